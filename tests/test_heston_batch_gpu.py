"""Batched Heston ADI (fe_heston_batch_*) against the law oracle option by option, the FP64 characteristic-function
price, and itself (graph replay, schedule independence, tile splits)."""
import json
import math
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

# Relative to the option's largest value, after `steps` ADI steps: the oracle does every op in double and stores float,
# the batch kernel computes in fp32 with the tridiagonal lines split between lanes (PCR), so the two round differently.
ORACLE_TOL = 1e-4

SMALL = ((16, 8), (32, 16), (64, 16), (32, 32), (128, 32))


def cell_payoff(strike, nx, ny):
    """The put payoff averaged over each cell (FP64, stored as float), rows identical."""
    h = 6.0 / nx
    lk = math.log(strike)
    x = lk - 3.0 + (np.arange(nx) + 0.5) * h
    lo = x - 0.5 * h
    hi = np.minimum(x + 0.5 * h, lk)
    v = np.where(hi > lo, (strike * (hi - lo) - (np.exp(hi) - np.exp(lo))) / h, 0.0)
    return np.broadcast_to(v.astype(np.float32)[None, :], (ny, nx)).copy()


def oracle_grid(o, steps, law_name):
    from oracle import law_cpu
    ir = json.load(open(os.path.join(ROOT, "tests", "golden", "ir", law_name + ".json")))
    nx, ny = o["nx"], o["ny"]
    h = 6.0 / nx
    s = law_cpu.Solver(law_cpu.Law(ir), (1, ny, nx), h)
    f32 = np.float32
    s.fields["V"] = cell_payoff(o["strike"], nx, ny)[None]
    s.fields["var"] = np.broadcast_to((o["sigma"] * (np.arange(ny) + 0.5) * h).astype(f32)[None, :, None], (1, ny, nx)).copy()
    for k, name in (("kappa", "kappa"), ("theta", "theta"), ("sig_v", "sigma"), ("rho", "rho"), ("r", "r")):
        s.fields[k] = np.full((1, ny, nx), f32(o[name]), f32)
    dt = o["maturity"] / steps
    for _ in range(steps):
        s.step(dt)
    return s.fields["V"][0]


def small_options(seed):
    from fieldcuda.heston import sample_options
    return sample_options(len(SMALL), seed, sizes=SMALL)


@pytest.mark.parametrize("scheme,law_name", [(0, "heston_douglas"), (1, "heston_hv")])
@pytest.mark.parametrize("split", [(16, 4, 384), (4, 1, 512), (8, 16, 256)])
def test_batch_matches_the_law_oracle(cuda, scheme, law_name, split):
    from fieldcuda.heston import HestonBatch
    opts = small_options(3)
    for i, (nx, ny) in enumerate(SMALL):
        opts[i]["nx"], opts[i]["ny"] = nx, ny
    steps = 12
    with HestonBatch(opts, steps, scheme) as b:
        b.set_split(*split)
        b.run()
        for i, o in enumerate(opts):
            got = b.grid(i).astype(np.float64)
            want = oracle_grid(o, steps, law_name).astype(np.float64)
            rel = np.abs(got - want).max() / np.abs(want).max()
            assert rel <= ORACLE_TOL, f"option {i} ({o['nx']}x{o['ny']}): relative difference {rel:.3g}"


@pytest.mark.parametrize("scheme,law_name", [(0, "heston_douglas"), (1, "heston_hv")])
def test_options_split_over_several_ctas_match_the_law_oracle(cuda, scheme, law_name):
    """Options of more than 16K cells or 128 rows are split by rows over 2, 4 or 8 CTAs of a cluster: the rows above and
    below a CTA's block come from its neighbours' shared memory and the y lines are solved across the CTAs."""
    from fieldcuda.heston import HestonBatch, sample_options
    sizes = ((256, 128), (512, 256), (64, 256), (512, 64), (128, 256), (32, 16))
    opts = sample_options(len(sizes), 11, sizes=sizes)
    for o, (nx, ny) in zip(opts, sizes):
        o["nx"], o["ny"] = nx, ny
    steps = 10
    with HestonBatch(opts, steps, scheme) as b:
        for split in ((16, 1, 512), (16, 16, 256), (16, 4, 384)):
            b.set_split(*split)
            b.run(use_graph=True)
            for i, o in enumerate(opts):
                got = b.grid(i).astype(np.float64)
                want = oracle_grid(o, steps, law_name).astype(np.float64)
                rel = np.abs(got - want).max() / np.abs(want).max()
                assert rel <= ORACLE_TOL, f"split {split} option {i} ({o['nx']}x{o['ny']}): relative difference {rel:.3g}"


def test_graph_replay_and_schedule_do_not_change_results(cuda):
    from fieldcuda.heston import HestonBatch, sample_options
    opts = sample_options(40, 5, sizes=((32, 16), (64, 32), (128, 64)))
    with HestonBatch(opts, 32) as b:
        b.run(use_graph=False)
        plain = b.prices()
        g0 = b.grid(7)
        b.run(use_graph=True)
        b.run(use_graph=True)
        assert np.array_equal(plain.view(np.uint32), b.prices().view(np.uint32))
        assert np.array_equal(g0.view(np.uint32), b.grid(7).view(np.uint32))
    # The same option alone: one CTA, another place in the queue, the same bits.
    with HestonBatch([opts[7]], 32) as one:
        one.run()
        assert np.array_equal(g0.view(np.uint32), one.grid(0).view(np.uint32))


def test_splits_agree_and_autotune_picks_one_that_fits(cuda):
    from fieldcuda.heston import HestonBatch, sample_options
    opts = sample_options(24, 9, sizes=((64, 32), (128, 64)))
    with HestonBatch(opts, 24, 1) as b:
        b.set_split(16, 16, 512)
        b.run()
        ref = b.prices().astype(np.float64)
        mx, sy, nt = b.autotune()
        assert mx in (4, 8, 16) and sy in (1, 2, 4, 8, 16) and nt in (256, 384, 512)
        assert 128 // mx <= 32
        b.run(use_graph=True)
        got = b.prices().astype(np.float64)
        assert np.abs(got - ref).max() <= 1e-4 * np.abs(ref).max()
        with pytest.raises(Exception):
            b.set_split(2, 8, 384)
        with pytest.raises(Exception):
            b.set_split(16, 8, 320)


def cf_price(o):
    from oracle import heston_cf
    return heston_cf.put(o["spot"], o["strike"], o["maturity"], o["v0"], o["kappa"], o["theta"], o["sigma"], o["rho"], o["r"])


@pytest.mark.parametrize("scheme", [0, 1])
def test_prices_converge_to_the_characteristic_function_price(cuda, scheme):
    """Grid refinement (h and dt halved together) brings the price toward the FP64 closed form."""
    from fieldcuda.heston import HestonBatch, sample_options
    base = sample_options(6, 21, sizes=((128, 64),))
    errs = []
    for level, (nx, ny, steps) in enumerate(((128, 64, 128), (256, 128, 256), (512, 256, 512))):
        opts = [dict(o, nx=nx, ny=ny) for o in base]
        with HestonBatch(opts, steps, scheme) as b:
            b.run(use_graph=True)
            p = b.prices().astype(np.float64)
        errs.append(np.array([abs(p[i] - cf_price(o)) for i, o in enumerate(opts)]))
    # Roughly second order for most options; one whose Feller condition fails badly (sigma^2 >> 2 kappa theta, option 0
    # here) has its error from the reflecting first variance rows and converges at first order, so the worst error
    # halves at least.
    worst = [float(e.max()) for e in errs]
    assert 2 * worst[2] < worst[1] and 2 * worst[1] < worst[0], worst
    median = [float(np.median(e)) for e in errs]
    assert median[2] < 2e-3 and median[2] < median[0] / 8, median
