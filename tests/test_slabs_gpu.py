"""A lattice split into z-slabs (fieldcuda.slabs), the slabs stepped on one GPU with their halo planes copied between
them (SlabGroup: the same kernels, plane layout and judge as one process a GPU, with device copies standing in for
NCCL): bit-identical to the whole lattice on one handle, conservation judged over the slabs, range cells reported at
their place in the lattice."""
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

HEAT = "field T init 0 range -1e6 1e6\nparam D = 1\nparam leak = 0\nterm conduction\n  d T = diffuse(D, T) - leak * T\n  conserves T\n"


def whole(law, shape, h, fields, steps, dt, params=()):
    from fieldcuda.solver import Solver
    nz, ny, nx = shape
    s = Solver(law, nx, ny, nz, h)
    for k, v in fields.items():
        s.set_field(k, v)
    for k, v in params:
        s.set_param(k, v)
    for _ in range(steps):
        s.step(dt)
    out = {k: s.values(k) for k in s.field_names}
    s.close()
    return out


@pytest.mark.parametrize("size,nx", [(2, 128), (3, 128), (2, 16)])
def test_heat_slabs_match_the_whole_lattice_bit_for_bit(cuda, size, nx):
    from fieldcuda.slabs import SlabGroup
    shape = (30, 20, nx)
    h = 1.0 / 32
    T0 = np.random.default_rng(3).uniform(0, 1, shape).astype(np.float32)
    dt = 0.4 * h * h / 6
    want = whole(HEAT, shape, h, {"T": T0}, 6, dt)["T"]
    g = SlabGroup(HEAT, nx, 20, 30, h, size)
    assert all(s.layout.halo == 1 for s in g.slabs)
    g.set_field("T", T0)
    for _ in range(6):
        g.step(dt)
    assert g.sync() == []
    got = g.values("T")
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    g.close()


def test_slabs_whose_planes_are_not_whole_float4s(cuda):
    """A 5 x 7 plane (35 cells): a slab's owned planes start inside a 16-byte word, and the lattice's cell count is not
    a multiple of 4. The totals before the first step (a fixed-grid float4 reduction) must count every owned cell once:
    no conservation break on the slabs or on the whole lattice, and the same bits."""
    from fieldcuda.slabs import SlabGroup
    from fieldcuda.solver import Solver
    shape = (30, 7, 5)
    h = 1.0 / 32
    T0 = np.random.default_rng(9).uniform(0, 1, shape).astype(np.float32)
    dt = 0.4 * h * h / 6
    s = Solver(HEAT, 5, 7, 30, h)
    s.set_field("T", T0)
    for _ in range(4):
        s.step(dt)
        assert s.violations() == []
    want = s.values("T")
    s.close()
    g = SlabGroup(HEAT, 5, 7, 30, h, 3)
    g.set_field("T", T0)
    for _ in range(4):
        g.step(dt)
    assert g.sync() == []
    assert np.array_equal(g.values("T").view(np.uint32), want.view(np.uint32))
    g.close()


def test_a_leak_is_judged_over_the_slabs_with_the_whole_lattices_totals(cuda):
    from fieldcuda.slabs import SlabGroup
    from fieldcuda.solver import Solver
    shape = (24, 12, 128)
    h = 0.1
    T0 = np.random.default_rng(4).uniform(1, 2, shape).astype(np.float32)
    s = Solver(HEAT, 128, 12, 24, h)
    s.set_field("T", T0)
    s.set_param("leak", 0.5)
    s.step(0.001)
    one = [v for v in s.violations() if v.kind == "conservation"]
    s.close()
    g = SlabGroup(HEAT, 128, 12, 24, h, 2)
    g.set_field("T", T0)
    g.set_param("leak", 0.5)
    g.step(0.001)
    v = g.sync()
    assert len(one) == 1 and len(v) == 1 and v[0]["kind"] == "conservation" and v[0]["term"] == "conduction"
    assert abs(v[0]["before"] - one[0].before) <= 1e-12 * abs(one[0].before)
    assert abs(v[0]["after"] - one[0].after) <= 1e-12 * abs(one[0].after)
    g.set_param("leak", 0.0)
    g.step(0.001)
    g.step(0.001)
    assert g.sync() == []
    g.close()


def test_deep_halo_of_a_43_term_law(cuda):
    """The 43-term law reads 17 planes along z in one step (its terms in turn): 17-plane halos keep the slabs exact."""
    from fieldcuda.slabs import SlabGroup
    law = open(os.path.join(ROOT, "tests", "laws", "multifield43.law")).read()
    shape = (40, 8, 128)
    h = 1.0 / 64
    g = SlabGroup(law, 128, 8, 40, h, 2)
    assert g.slabs[0].layout.halo == 17
    rng = np.random.default_rng(5)
    fields = {f: rng.uniform(0.2, 0.8, shape).astype(np.float32) for f in g.slabs[0].solver.field_names}
    for k, v in fields.items():
        g.set_field(k, v)
    dt = 1e-6
    want = whole(law, shape, h, fields, 3, dt)
    for _ in range(3):
        g.step(dt)
    g.sync()
    for k in fields:
        got = g.values(k)
        assert np.array_equal(got.view(np.uint32), want[k].view(np.uint32)), k
    g.close()


def test_range_cells_are_reported_at_their_place_in_the_lattice(cuda):
    from fieldcuda.slabs import SlabGroup
    law = "field a init 0 range -1 1\nfield b init 0 range -1e30 1e30 static\nterm t\n  d a = b\n"
    shape = (20, 6, 128)
    b = np.zeros(shape, np.float32)
    b[14, 2, 9] = 5.0
    b[17, 0, 1] = 5.0
    g = SlabGroup(law, 128, 6, 20, 1.0, 2)
    g.set_field("b", b)
    g.step(1.0)
    v = g.sync()
    assert len(v) == 1 and v[0]["kind"] == "range" and v[0]["count"] == 2
    assert v[0]["first_cell"] == 9 + 128 * (2 + 6 * 14)
    g.close()


def test_laws_that_do_not_split_are_refused(cuda):
    from fieldcuda.slabs import SlabGroup
    law = open(os.path.join(ROOT, "tests", "laws", "heston_explicit.law")).read()  # max_dt reads maxof(...)
    with pytest.raises(ValueError):
        SlabGroup(law, 128, 16, 8, 0.05, 2)


def _slab_worker(rank, size, port, steps, out):
    import sys
    from conftest import PKG
    sys.path[:0] = [ROOT, PKG]
    import torch
    import torch.distributed as dist
    from fieldcuda.slabs import DistComm, SlabLaw
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    try:
        nz, ny, nx = 30, 20, 128
        h = 1.0 / 32
        T0 = np.random.default_rng(3).uniform(0, 1, (nz, ny, nx)).astype(np.float32)
        s = SlabLaw(HEAT, nx, ny, nz, h, rank, size, DistComm(), source_name="heat.law")
        s.set_field("T", T0[s.layout.z0:s.layout.z1])
        for _ in range(steps):
            s.step(0.4 * h * h / 6)
        v = s.sync()
        out.put((rank, s.layout.z0, s.values("T").tobytes(), v))
        s.close()
    finally:
        dist.destroy_process_group()


def test_two_processes_step_one_lattice_through_the_distributed_path(cuda):
    """SlabLaw with DistComm as bench.py --gpus N runs it, here as two processes on the one GPU over gloo (host copies
    of the halo planes instead of NCCL; the kernels of the two processes never wait on each other)."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_slab_worker, args=(r, 2, port, 5, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in procs], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
    nz, ny, nx = 30, 20, 128
    h = 1.0 / 32
    T0 = np.random.default_rng(3).uniform(0, 1, (nz, ny, nx)).astype(np.float32)
    want = whole(HEAT, (nz, ny, nx), h, {"T": T0}, 5, 0.4 * h * h / 6)["T"]
    got = np.concatenate([np.frombuffer(b, np.float32).reshape(-1, ny, nx) for _, _, b, _ in res])
    assert all(v == [] for _, _, _, v in res)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
