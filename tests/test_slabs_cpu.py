"""The z-slab split of one lattice over ranks, on the CPU: the layout, the halo exchange protocol over gloo ranks
(world size 3, so a middle rank has both neighbours), and the conservation judge over the ranks' totals."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import PKG, ROOT


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_layout_covers_the_lattice_once_with_halos_only_between_ranks():
    from fieldcuda.slabs import SlabLayout
    for nz, size, halo in ((40, 2, 1), (41, 3, 2), (512, 8, 17), (7, 1, 3)):
        owned = []
        for r in range(size):
            L = SlabLayout(nz, size, r, halo)
            assert L.below == (halo if r > 0 else 0) and L.above == (halo if r < size - 1 else 0)
            lo, hi = L.own()
            assert hi - lo == L.z1 - L.z0 and L.local_nz == L.below + L.owned + L.above
            owned.extend(range(L.z0, L.z1))
            # a local index maps to the same (x, y) and the owned plane's global z
            nx, ny = 5, 3
            assert L.global_index(lo * nx * ny + 7, nx, ny) == L.z0 * nx * ny + 7
        assert owned == list(range(nz))
    with pytest.raises(ValueError):
        SlabLayout(10, 4, 0, 3)  # slabs of 2 or 3 planes cannot hold a 3-plane halo


def test_judge_sums_over_ranks_in_rank_order_and_applies_the_tolerance():
    from fieldcuda.slabs import judge_totals, pack_totals
    a = [{"step": 0, "term": 0, "group": 0, "substeps": 1, "before": 100.0, "after": 99.0, "scale": 100.0},
         {"step": 1, "term": 0, "group": 0, "substeps": 4, "before": 50.0, "after": 50.0005, "scale": 50.0}]
    b = [{"step": 0, "term": 0, "group": 0, "substeps": 1, "before": 20.0, "after": 21.0, "scale": 20.0},
         {"step": 1, "term": 0, "group": 0, "substeps": 4, "before": 10.0, "after": 10.0, "scale": 10.0}]
    assert judge_totals([pack_totals(a), pack_totals(b)]) == []  # flux across the slab face: conserved as a whole
    b[0]["after"] = 21.01
    v = judge_totals([pack_totals(a), pack_totals(b)])
    assert len(v) == 1 and v[0]["step"] == 0 and abs(v[0]["after"] - 120.01) < 1e-9
    assert abs(v[0]["tolerance"] - 1e-5 * 121.0) < 1e-15
    b[1]["after"] = 10.0 + 1e-5 * 61.0 * 2.0 * 1.01 - 0.0005  # just over 1e-5 (scale + 1) sqrt(4)
    v = judge_totals([pack_totals(a), pack_totals(b)])
    assert [x["step"] for x in v] == [0, 1]
    with pytest.raises(RuntimeError):
        judge_totals([pack_totals(a), pack_totals(b[:1])])


def _worker(rank, size, port, out):
    import sys
    sys.path[:0] = [ROOT, PKG]
    import torch
    import torch.distributed as dist
    from fieldcuda.slabs import DistComm, SlabLayout, exchange_halos, judge_totals, pack_totals
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    try:
        nz, ny, nx, halo = 13, 3, 4, 2
        L = SlabLayout(nz, size, rank, halo)
        comm = DistComm()
        lattice = np.arange(nz * ny * nx, dtype=np.float32).reshape(nz, ny, nx)
        bufs = []
        for k in range(2):  # two fields, exchanged in one round
            b = torch.full((L.local_nz, ny, nx), -1.0)
            lo, hi = L.own()
            b[lo:hi] = torch.from_numpy(lattice[L.z0:L.z1] * (k + 1))
            bufs.append(b)
        exchange_halos(bufs, L, comm)
        # every local plane now holds the lattice's plane it stands for
        got = [b.numpy().copy() for b in bufs]
        want = [lattice[L.z0 - L.below:L.z1 + L.above] * (k + 1) for k in range(2)]
        ok = all(np.array_equal(g, w) for g, w in zip(got, want))
        entries = [{"step": 0, "term": 0, "group": 0, "substeps": 1, "before": 1.0 + rank, "after": 1.5 - rank * 0.25, "scale": 3.0}]
        per_rank = comm.gather(pack_totals(entries))
        verdict = judge_totals(per_rank)
        out.put((rank, ok, [p.tobytes() for p in per_rank], verdict))
    finally:
        dist.destroy_process_group()


def test_halo_exchange_and_totals_gather_over_three_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    size = 3
    procs = [ctx.Process(target=_worker, args=(r, size, port, q)) for r in range(size)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=180) for _ in procs], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
    assert all(ok for _, ok, _, _ in res)
    assert res[0][2] == res[1][2] == res[2][2]  # the same gathered bytes on every rank
    # before 1 + 2 + 3 = 6, after 1.5 + 1.25 + 1.0 = 3.75: a leak, seen by every rank alike
    assert all(len(v) == 1 and abs(v[0]["before"] - 6.0) < 1e-12 and abs(v[0]["after"] - 3.75) < 1e-12 for _, _, _, v in res)
