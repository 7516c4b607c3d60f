"""One law on many uneven lattices (fe_batch_*): every instance's fields equal, to the bit, those of the same instance
run alone; instances of equal nx x ny are stacked along z only when the law couples nothing along z; broken contracts
come back with their instance."""
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def text(name):
    return open(os.path.join(ROOT, "tests", "laws", name)).read()


def alone(law, lattice, fields, dt, steps):
    from fieldcuda.solver import Solver
    nx, ny, nz, h = lattice
    s = Solver(law, nx, ny, nz, h)
    for k, v in fields.items():
        s.set_field(k, v)
    for _ in range(steps):
        s.step(dt)
    out = {k: s.values(k) for k in s.field_names}
    s.close()
    return out


@pytest.mark.parametrize("law_name,lattices,stacked,count", [
    # FHN (2-D stencils, a sample a plane): equal shapes stacked, uneven depths.
    ("fhn_rk4.law", [(32, 32, 3, 2 / 32), (32, 32, 5, 2 / 32), (16, 16, 2, 2 / 16), (32, 32, 1, 2 / 32)], True, 2),
    # Heat in 3-D reads across planes: every instance a lattice of its own.
    ("heat.law", [(24, 20, 6, 0.05), (16, 16, 4, 0.1), (24, 20, 6, 0.05)], False, 3),
])
def test_batch_matches_each_instance_alone(cuda, law_name, lattices, stacked, count):
    from fieldcuda.batch import LawBatch
    law = text(law_name)
    rng = np.random.default_rng(5)
    b = LawBatch(law, lattices)
    assert b.info() == (count, stacked)
    starts = []
    for i, (nx, ny, nz, h) in enumerate(lattices):
        f = {}
        for name in b.field_names:
            f[name] = rng.normal(size=(nz, ny, nx)).astype(np.float32) * (300.0 if law_name == "heat.law" else 1.0)
            b.set_field(i, name, f[name])
        starts.append(f)
    dt = 1e-4 if law_name == "heat.law" else 0.05
    for _ in range(3):
        b.step(dt)
        assert b.violations() == []
    for i, lattice in enumerate(lattices):
        want = alone(law, lattice, starts[i], dt, 3)
        for name in b.field_names:
            got = b.values(i, name)
            assert np.array_equal(got.view(np.uint32), want[name].view(np.uint32)), (i, name)
    b.close()


def test_a_broken_range_names_its_instance(cuda):
    from fieldcuda.batch import LawBatch
    law = "field T init 0 range 0 100\nparam k = 0.1\nterm decay\n  d T = -k * T\n"
    b = LawBatch(law, [(8, 8, 2, 1.0), (8, 8, 3, 1.0), (4, 4, 1, 1.0)])
    assert b.info() == (2, True)
    hot = np.full((3, 8, 8), 50.0, np.float32)
    hot[1, 2, 3] = 500.0
    b.set_field(1, "T", hot)
    b.step(0.1)
    found = [(i, v.kind, v.first_cell) for i, v in b.violations()]
    assert found == [(1, "range", 3 + 8 * (2 + 8 * 1))], found
    b.set_param("k", 0.0)
    b.set_field(1, "T", np.full((3, 8, 8), 50.0, np.float32))
    b.step(0.1)
    assert b.violations() == []
    assert np.all(b.values(1, "T") == 50.0) and np.all(b.values(0, "T") == 0.0)
    b.close()
