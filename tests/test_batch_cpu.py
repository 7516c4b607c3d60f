"""How fe_batch groups instances, without a device (fe_batch_plan): equal nx x ny x h stacked along z in order when
the law couples nothing along z, every instance a lattice of its own otherwise."""
import ctypes
import os

import pytest

from conftest import ROOT


def plan(law, lattices):
    from fieldcuda import _lib
    descs = (_lib.fe_batch_desc * len(lattices))()
    for d, (nx, ny, nz, h) in zip(descs, lattices):
        d.nx, d.ny, d.nz, d.h = nx, ny, nz, h
    n, stacked = ctypes.c_int(), ctypes.c_int()
    where, z0 = (ctypes.c_int * len(lattices))(), (ctypes.c_int * len(lattices))()
    _lib.check(_lib.lib().fe_batch_plan(law.encode(), descs, len(lattices), ctypes.byref(n), ctypes.byref(stacked), where, z0))
    return n.value, bool(stacked.value), list(where), list(z0)


def text(name):
    return open(os.path.join(ROOT, "tests", "laws", name)).read()


UNEVEN = [(32, 32, 3, 0.1), (32, 32, 5, 0.1), (16, 16, 2, 0.1), (32, 32, 1, 0.1), (32, 32, 2, 0.05)]


def test_plane_independent_laws_stack_equal_shapes():
    for law in ("fhn_rk4.law", "heston_douglas.law", "heston_hv.law"):
        assert plan(text(law), UNEVEN) == (3, True, [0, 0, 1, 0, 2], [0, 3, 0, 8, 0]), law


@pytest.mark.parametrize("law", [
    text("heat.law"),                                                     # reads across planes
    "field T init 0 range -1 1\nterm t\n  d T = -T * rim\n",              # `rim` marks the lattice's z faces
    "field T init 0 range -1 1\nterm t\n  d T = -T + maxof(T)\n",         # a lattice-wide reduction
    text("ops_fields.law"),                                               # distance and poisson
    # A pointwise classical term whose learned equations read across planes (ldiffuse's faces along z): learned
    # schemes may be turned on after planning, so the instances stay apart.
    "field T init 290 range 0 6000\nparam k = 1\nnet lh in 5 hidden 8 out 4 act tanh file none\n"
    "term t\n  d T = -k * T\n  learned d T = ldiffuse(lh, k, T)\n",
    # A pointwise learned term whose learned step limit reduces over the lattice.
    "field T init 1 range -10 10\nterm t\n  d T = -T\n  learned d T = -2 * T\n"
    "  learned max_dt = 0.1 / (maxof(T) + 1)\n",
])
def test_laws_that_couple_planes_keep_instances_apart(law):
    assert plan(law, UNEVEN) == (5, False, [0, 1, 2, 3, 4], [0, 0, 0, 0, 0])


def test_bad_instances_are_refused():
    from fieldcuda import _lib
    with pytest.raises(_lib.FeError, match="bad lattice"):
        plan(text("fhn_rk4.law"), [(4, 4, 0, 0.1)])
    with pytest.raises(_lib.FeError, match="unknown"):
        plan("field T init 0\nterm t\n  d T = sprinkle(T)\n", [(4, 4, 1, 0.1)])
