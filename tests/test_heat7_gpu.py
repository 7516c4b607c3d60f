"""The hand-written 7-point heat kernel (TMA z-marching and plain) against the oracle's restatements."""
import numpy as np
import pytest

from oracle import heat as oh

pytestmark = pytest.mark.gpu

SHAPES = [(9, 14, 20), (11, 20, 132), (5, 3, 4), (1, 1, 4), (33, 40, 256)]  # (nz, ny, nx)


def _run(T0, k, h, dt, variant, zchunk, steps=1, check=0):
    import torch
    from fieldcuda import kernels
    a = torch.from_numpy(T0).cuda()
    b = torch.empty_like(a)
    ws = kernels.heat7_workspace(T0.shape, variant, zchunk)
    recs = []
    for _ in range(steps):
        if check:
            kernels.check_reset(ws)
        kernels.heat7_step(a, b, k, h, dt, variant=variant, zchunk=zchunk, check=check, workspace=ws)
        if check:
            recs.append(kernels.check_read(ws))
        a, b = b, a
    torch.cuda.synchronize()
    return a.cpu().numpy(), recs


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("variant", [-1, 0, 1, 2, 3])
def test_bit_identical_to_fp32_restatement(cuda, shape, variant):
    if variant >= 0 and shape[2] % 4:
        pytest.skip("TMA variants need nx % 4 == 0")
    rng = np.random.default_rng(7)
    T0 = rng.uniform(-1, 1, size=shape).astype(np.float32)
    k, h, dt = 0.7, 0.125, 0.002
    want = T0
    for _ in range(3):
        want = oh.gpu_order_step(want, k, h, dt)
    for zchunk in (1, 2, 7, 64):
        got, _ = _run(T0, k, h, dt, variant, zchunk, steps=3)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (shape, variant, zchunk)


def test_within_1e6_of_cpu_reference_heat_128(cuda):
    n, h = 128, 1.0 / 128
    dt = 0.4 * h * h / 6.0
    T0 = oh.gaussian_blobs(n, h, seed=0)
    cpu = T0
    for _ in range(20):
        cpu = oh.cpu_step(cpu, 1.0, h, dt)
    got, _ = _run(T0, 1.0, h, dt, 0, 64, steps=20)
    rel = np.abs(got.astype(np.float64) - cpu).max() / np.abs(cpu).max()
    assert rel <= 1e-6, rel


def test_contracts_fused(cuda):
    import torch
    from fieldcuda import kernels, _lib
    rng = np.random.default_rng(3)
    shape = (17, 24, 64)
    T0 = rng.uniform(0, 2, size=shape).astype(np.float32)
    k, h, dt = 1.0, 0.1, 0.001
    want = oh.gpu_order_step(T0, k, h, dt)
    for variant in (-1, 0, 1):
        a = torch.from_numpy(T0).cuda()
        b = torch.empty_like(a)
        ws = kernels.heat7_workspace(shape, variant, 4)
        kernels.check_reset(ws)
        kernels.heat7_step(a, b, k, h, dt, lo=0.5, hi=1.5, variant=variant, zchunk=4,
                           check=_lib.FE_HEAT7_BEFORE | _lib.FE_HEAT7_AFTER, workspace=ws)
        rec = kernels.check_read(ws)
        s0, m0 = oh.totals(T0)
        s1, m1 = oh.totals(want)
        # FP64 totals of fp32 sums of 4 cells: within a few 1e-8 of the exact total, far inside the contract's 1e-5.
        assert rec.before == pytest.approx(s0, rel=1e-7) and rec.before_abs == pytest.approx(m0, rel=1e-7)
        assert rec.after == pytest.approx(s1, rel=1e-7)
        lib = _lib.lib()
        assert np.float32(lib.fe_key_to_float(~rec.lo_inv & 0xFFFFFFFF)) == want.min()
        assert np.float32(lib.fe_key_to_float(rec.hi_key)) == want.max()
        bad = (want < 0.5) | (want > 1.5)
        assert rec.out_of_range == int(bad.sum()) and rec.not_finite == 0
        assert (~rec.first_bad & 0xFFFFFFFF) == int(np.flatnonzero(bad.ravel())[0])
        assert rec.changed == 1
        # Two runs: the FP64 totals agree to the bit (fixed order).
        kernels.check_reset(ws)
        kernels.heat7_step(a, b, k, h, dt, lo=0.5, hi=1.5, variant=variant, zchunk=4,
                           check=_lib.FE_HEAT7_BEFORE | _lib.FE_HEAT7_AFTER, workspace=ws)
        rec2 = kernels.check_read(ws)
        assert (rec2.before, rec2.before_abs, rec2.after) == (rec.before, rec.before_abs, rec.after)


def test_totals_are_compensated(cuda):
    """Planes alternating +1e20, 1, -1e20, 1 (each constant, k = 0: nothing moves), four planes a z-chunk, so every
    thread's run of planes cancels: the exact total is the 1-planes' cell count. Plain FP64 accumulation across a
    thread's planes loses each 1 added next to 1e20 (its ulp there is 2^14), half of them; the compensated sum (Neumaier
    from the plane partials on) keeps them, in every kernel variant. Each level of the fixed tree is compensated by
    itself and hands its sum on as one double, so the guarantee is the sum of each level's rounding, not cancellation
    across blocks: the case keeps the large values' cancellation inside a thread."""
    import torch
    from fieldcuda import kernels, _lib
    nz, ny, nx = 16, 24, 128
    T0 = np.empty((nz, ny, nx), np.float32)
    for z in range(nz):
        T0[z] = (1e20 if z % 4 == 0 else -1e20) if z % 2 == 0 else 1.0
    exact = float(nx * ny * (nz // 2))
    for variant in (-1, 0, 1):
        a = torch.from_numpy(T0).cuda()
        b = torch.empty_like(a)
        ws = kernels.heat7_workspace(T0.shape, variant, 4)
        kernels.check_reset(ws)
        kernels.heat7_step(a, b, 0.0, 0.1, 0.001, lo=-1e30, hi=1e30, variant=variant, zchunk=4,
                           check=_lib.FE_HEAT7_BEFORE | _lib.FE_HEAT7_AFTER, workspace=ws)
        rec = kernels.check_read(ws)
        assert rec.before == exact and rec.after == exact, (variant, rec.before, rec.after, exact)


def test_not_finite_is_counted(cuda):
    import torch
    from fieldcuda import kernels, _lib
    T0 = np.ones((6, 8, 16), dtype=np.float32)
    T0[2, 3, 5] = np.nan
    a = torch.from_numpy(T0).cuda()
    b = torch.empty_like(a)
    ws = kernels.heat7_workspace(T0.shape, 0, 2)
    kernels.check_reset(ws)
    kernels.heat7_step(a, b, 1.0, 0.5, 0.01, variant=0, zchunk=2, check=_lib.FE_HEAT7_AFTER, workspace=ws)
    rec = kernels.check_read(ws)
    out = b.cpu().numpy()
    assert rec.not_finite == int((~np.isfinite(out)).sum()) > 0
