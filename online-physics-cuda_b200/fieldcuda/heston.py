"""Batched Heston ADI on the GPU (include/fe.h, fe_heston_batch_*): many European puts, each on its own grid, stepped
to maturity by one persistent kernel.

The reference prices a batch as the z-planes of one lattice, all options on one grid, through its law solver
(bench/finance.py:253-288 with bench/laws/heston_adi.law). Here the options keep their own (nx, ny) and the whole
batch is one launch sequence (payoffs, the persistent ADI kernel of 8-CTA clusters that holds every option's state in
shared memory from its first step to its last, the price read-out), optionally replayed as a CUDA graph. The
discretisation is the law's: tests/laws/heston_douglas.law and heston_hv.law.
"""
import ctypes

import numpy as np

from . import _lib

DOUGLAS = _lib.FE_ADI_DOUGLAS
HV = _lib.FE_ADI_HV

FIELDS = ("nx", "ny", "strike", "maturity", "spot", "v0", "kappa", "theta", "sigma", "rho", "r")


def option_array(options):
    """A ctypes array of fe_heston_option from dicts (or objects with those attributes)."""
    arr = (_lib.fe_heston_option * len(options))()
    for i, o in enumerate(options):
        for f in FIELDS:
            setattr(arr[i], f, o[f] if isinstance(o, dict) else getattr(o, f))
    return arr


class HestonBatch:
    """One batch of options: ``run`` prices them all, ``prices`` and ``grid`` read the results back."""

    def __init__(self, options, steps, scheme=DOUGLAS):
        self.options = list(options)
        self.steps = int(steps)
        self.scheme = scheme
        self._arr = option_array(self.options)
        handle = ctypes.c_void_p()
        _lib.call("fe_heston_batch_create", self._arr, len(self.options), self.steps, scheme, ctypes.byref(handle))
        self._h = handle

    def close(self):
        if self._h:
            _lib.lib().fe_heston_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_split(self, mx, sy, threads=384):
        """Cells a lane holds in the x solves (4, 8 or 16), the most row blocks a CTA cuts a column into for the y
        solves (1 .. 16), and threads a CTA (256, 384 or 512)."""
        _lib.call("fe_heston_batch_set_split", self._h, mx, sy, threads)

    def autotune(self):
        """Times every split that fits and keeps the fastest; returns it as (mx, sy, threads)."""
        mx, sy, nt = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.call("fe_heston_batch_autotune", self._h, ctypes.byref(mx), ctypes.byref(sy), ctypes.byref(nt))
        return mx.value, sy.value, nt.value

    def layout(self):
        """(clusters of the persistent grid, tasks of the batch)."""
        c, t = ctypes.c_int(), ctypes.c_int()
        _lib.call("fe_heston_batch_layout", self._h, ctypes.byref(c), ctypes.byref(t))
        return c.value, t.value

    def run(self, use_graph=False):
        """Prices the batch (asynchronous on the batch's stream)."""
        _lib.call("fe_heston_batch_run", self._h, int(bool(use_graph)))

    def time(self, use_graph=True):
        """Device time of one run, in ms."""
        ms = ctypes.c_float()
        _lib.call("fe_heston_batch_time", self._h, int(bool(use_graph)), ctypes.byref(ms))
        return ms.value

    def prices(self):
        out = np.empty(len(self.options), np.float32)
        _lib.call("fe_heston_batch_prices", self._h, out.ctypes.data_as(ctypes.c_void_p))
        return out

    def grid(self, i):
        """Option i's grid after the last run, shape (ny, nx)."""
        o = self._arr[i]
        out = np.empty((o.ny, o.nx), np.float32)
        _lib.call("fe_heston_batch_grid", self._h, i, out.ctypes.data_as(ctypes.c_void_p))
        return out


def sample_options(n, seed, sizes=((128, 64), (256, 128), (512, 256))):
    """Seeded options with the batch benchmark's parameter ranges: strike U[80, 120], T U[0.25, 2], kappa U[0.5, 5],
    theta U[0.01, 0.1], sigma U[0.1, 1], rho U[-0.9, -0.1], v0 U[0.01, 0.1], r U[0, 0.05], spot 100; grid sizes
    drawn from ``sizes``."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx, ny = sizes[int(rng.integers(len(sizes)))]
        out.append(dict(nx=nx, ny=ny, strike=float(rng.uniform(80, 120)), maturity=float(rng.uniform(0.25, 2.0)),
                        spot=100.0, v0=float(rng.uniform(0.01, 0.1)), kappa=float(rng.uniform(0.5, 5)),
                        theta=float(rng.uniform(0.01, 0.1)), sigma=float(rng.uniform(0.1, 1.0)),
                        rho=float(rng.uniform(-0.9, -0.1)), r=float(rng.uniform(0.0, 0.05))))
    return out


def cell_payoff(strike, nx):
    """The put payoff averaged over each of nx cells of x = ln S on [ln K - 3, ln K + 3] (FP64, stored as float)."""
    h = 6.0 / nx
    lk = np.log(strike)
    x = lk - 3.0 + (np.arange(nx) + 0.5) * h
    lo = x - 0.5 * h
    hi = np.minimum(x + 0.5 * h, lk)
    v = np.where(hi > lo, (strike * (hi - lo) - (np.exp(hi) - np.exp(lo))) / h, 0.0)
    return v.astype(np.float32)


def lattice_fields(options, nx, ny):
    """The fields of the Heston laws (tests/laws/heston_*.law) for options of one grid size as the z-planes of one
    lattice, the reference's way of batching (bench/finance.py:253-267): V the cell-averaged payoff, var the rows'
    variances sigma (j + 1/2) h, the model numbers as per-plane constants. Returns (fields, h)."""
    nz = len(options)
    h = 6.0 / nx
    f32 = np.float32
    shape = (nz, ny, nx)
    out = {k: np.empty(shape, f32) for k in ("V", "var", "kappa", "theta", "sig_v", "rho", "r")}
    for z, o in enumerate(options):
        out["V"][z] = cell_payoff(o["strike"], nx)[None, :]
        out["var"][z] = (o["sigma"] * (np.arange(ny) + 0.5) * h).astype(f32)[:, None]
        for k, name in (("kappa", "kappa"), ("theta", "theta"), ("sig_v", "sigma"), ("rho", "rho"), ("r", "r")):
            out[k][z] = f32(o[name])
    return out, h


def _cubic(f, n):
    """First of the four cell centres of a cubic read at fractional centre index f on an axis of n, and the Lagrange
    weights at f (offsets -1, 0, 1, 2 from the second centre; below the first centre it extrapolates)."""
    s = int(max(0, min(n - 4, np.floor(f) - 1)))
    t = f - (s + 1)
    return s, np.array([-t * (t - 1) * (t - 2) / 6, (t + 1) * (t - 1) * (t - 2) / 2, -(t + 1) * t * (t - 2) / 2,
                        (t + 1) * t * (t - 1) / 6])


def price_at(grid, option):
    """Bicubic price at (ln spot, v0) through the 4 x 4 cell centres around it of one option's (ny, nx) grid, as the
    batch's read-out (a local Lagrange cubic along each axis)."""
    ny, nx = grid.shape
    h = 6.0 / nx
    x0 = np.log(option["strike"]) - 3.0 + 0.5 * h
    fx = (np.log(option["spot"]) - x0) / h
    fy = option["v0"] / (option["sigma"] * h) - 0.5
    i0, wx = _cubic(fx, nx)
    j0, wy = _cubic(fy, ny)
    g = grid.astype(np.float64)[j0:j0 + 4, i0:i0 + 4]
    return float(wy @ g @ wx)


def price_bilinear(grid, option):
    """Bilinear price at (ln spot, v0) between the four cell centres around it (clamped to the grid): the calibration's
    read-out (Calibration.prices), kept bilinear so its gradient through autograd is the read-out's own."""
    ny, nx = grid.shape
    h = 6.0 / nx
    x0 = np.log(option["strike"]) - 3.0 + 0.5 * h
    fx = (np.log(option["spot"]) - x0) / h
    fy = option["v0"] / (option["sigma"] * h) - 0.5
    i0 = int(max(0, min(nx - 2, np.floor(fx))))
    j0 = int(max(0, min(ny - 2, np.floor(fy))))
    tx = min(max(fx - i0, 0.0), 1.0)
    ty = min(max(fy - j0, 0.0), 1.0)
    g = grid.astype(np.float64)
    return float((1 - ty) * ((1 - tx) * g[j0, i0] + tx * g[j0, i0 + 1]) + ty * ((1 - tx) * g[j0 + 1, i0] + tx * g[j0 + 1, i0 + 1]))


class Calibration:
    """The Heston calibration's loss and its gradient by reverse mode through the ADI law (the reference's adjoint
    calibration, bench/calibrate.py, there through the explicit law): the options of one maturity as the z-planes of
    one (nx, ny) lattice, stepped by tests/laws/heston_douglas.law's scheme (`law_text`), the price read off each plane
    by bilinear interpolation (price_bilinear), loss = sum (price - target)^2, gradient with respect to (kappa, theta,
    sigma, rho, v0) through LawSteps (the IR-generated adjoint law, sqrt(N) checkpoints) and torch autograd for the
    rest (the variance rows sigma (j + 1/2) h and the read-out at v0)."""

    NAMES = ("kappa", "theta", "sigma", "rho", "v0")

    def __init__(self, law_text, strikes, maturity, spot, r, targets, nx, ny, steps):
        import torch
        from .adjoint import LawVJP
        self.n = len(strikes)
        self.nx, self.ny, self.steps = nx, ny, steps
        self.h = 6.0 / nx
        self.dt = maturity / steps
        self.spot = spot
        self.r = r
        self.strikes = np.asarray(strikes, np.float64)
        self.targets = torch.tensor(np.asarray(targets, np.float64), device="cuda")
        self.vjp = LawVJP(law_text, nx, ny, self.n, self.h, name="heston_calibration")
        payoff = np.stack([cell_payoff(k, nx) for k in self.strikes])
        self.V0 = torch.tensor(np.broadcast_to(payoff[:, None, :], (self.n, ny, nx)).copy(), device="cuda")
        self.rows = torch.tensor(((np.arange(ny) + 0.5) * self.h)[None, :, None], dtype=torch.float32, device="cuda")
        x0 = np.log(self.strikes) - 3.0 + 0.5 * self.h
        self.fx = torch.tensor((np.log(spot) - x0) / self.h, dtype=torch.float64, device="cuda")

    def close(self):
        self.vjp.close()

    def prices(self, params):
        """Prices (float64 tensor) of every option under params = (kappa, theta, sigma, rho, v0) tensors."""
        import torch
        from .adjoint import LawSteps
        kappa, theta, sigma, rho, v0 = params
        shape = (self.n, self.ny, self.nx)
        f32 = torch.float32
        full = lambda v: v.to(f32).reshape(1, 1, 1).expand(shape).contiguous()
        var = (sigma.to(f32) * self.rows).expand(shape).contiguous()
        names = ("V", "var", "kappa", "theta", "sig_v", "rho", "r")
        r = torch.full(shape, self.r, dtype=f32, device="cuda")
        (VT,) = LawSteps.apply(self.vjp, self.dt, self.steps, names, self.V0, var, full(kappa), full(theta), full(sigma), full(rho), r)
        fx = self.fx
        fy = v0.double() / (sigma.double() * self.h) - 0.5
        i0 = torch.clamp(torch.floor(fx), 0, self.nx - 2).long()
        j0 = torch.clamp(torch.floor(fy.detach()), 0, self.ny - 2).long().expand(self.n)
        tx = torch.clamp(fx - i0, 0.0, 1.0)
        ty = torch.clamp(fy - j0, 0.0, 1.0)
        z = torch.arange(self.n, device="cuda")
        U = VT.double()
        a, b = U[z, j0, i0], U[z, j0, i0 + 1]
        c, d = U[z, j0 + 1, i0], U[z, j0 + 1, i0 + 1]
        return (1 - ty) * ((1 - tx) * a + tx * b) + ty * ((1 - tx) * c + tx * d)

    def loss(self, params):
        p = self.prices(params)
        return ((p - self.targets) ** 2).sum()

    def loss_and_grad(self, values):
        """(loss, gradient) at values = (kappa, theta, sigma, rho, v0) floats."""
        import torch
        params = [torch.tensor(float(v), dtype=torch.float64, device="cuda", requires_grad=True) for v in values]
        L = self.loss(params)
        L.backward()
        return float(L.detach()), np.array([float(p.grad) for p in params])

    def loss_only(self, values):
        import torch
        with torch.no_grad():
            params = [torch.tensor(float(v), dtype=torch.float64, device="cuda") for v in values]
            return float(self.loss(params))


def calibration_options(n, seed):
    """The calibration set: n strikes U[80, 120] at one maturity (T = 1, spot 100, r = 0.02), and a seeded ground-truth
    parameter set (kappa U[0.5, 5], theta U[0.01, 0.1], sigma U[0.1, 1], rho U[-0.9, -0.1], v0 U[0.01, 0.1])."""
    rng = np.random.default_rng(seed)
    strikes = rng.uniform(80, 120, n)
    truth = dict(kappa=rng.uniform(0.5, 5), theta=rng.uniform(0.01, 0.1), sigma=rng.uniform(0.1, 1.0),
                 rho=rng.uniform(-0.9, -0.1), v0=rng.uniform(0.01, 0.1))
    return strikes, dict(maturity=1.0, spot=100.0, r=0.02), truth
