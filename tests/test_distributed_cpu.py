"""The multi-process host logic on the CPU (gloo, world size 2): instance shards and the rank-ordered sums the sharded
forms use."""
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


def _worker(rank, size, port, out):
    import sys
    sys.path[:0] = [ROOT, PKG]
    import torch
    import torch.distributed as dist
    from fieldcuda import distributed as fd
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    try:
        rng = np.random.default_rng(rank)
        mine = rng.normal(size=7) * 10.0 ** rng.integers(-8, 8, 7)
        total = fd.fixed_order_sum(mine).numpy()
        lo, hi = fd.shard_range(11, rank, size)
        peak = fd.max_over_ranks(float(rank) * 2.5)
        out.put((rank, total.tobytes(), (lo, hi), peak))
    finally:
        dist.destroy_process_group()


def test_shards_cover_every_item_once():
    from fieldcuda.distributed import shard_range
    for n in (0, 1, 7, 2048, 2049):
        for size in (1, 2, 3, 8):
            seen = []
            for r in range(size):
                lo, hi = shard_range(n, r, size)
                assert 0 <= lo <= hi <= n
                seen.extend(range(lo, hi))
            assert seen == list(range(n))


def test_rank_ordered_sums_agree_on_every_rank_and_with_a_local_sum():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    totals = [np.frombuffer(b, np.float64) for _, b, _, _ in res]
    assert totals[0].tobytes() == totals[1].tobytes()
    want = np.zeros(7)
    for r in range(2):
        rng = np.random.default_rng(r)
        want = want + rng.normal(size=7) * 10.0 ** rng.integers(-8, 8, 7)
    assert totals[0].tobytes() == want.tobytes()
    assert [s for _, _, s, _ in res] == [(0, 6), (6, 11)]
    assert all(p == 2.5 for _, _, _, p in res)
