"""The learned coarse-lattice correction (include/fe.h, fe_corr_*): a 3x3-conv/pointwise network on the tensor cores
that corrects a coarse plain step, trained on the GPU against fine solutions the engine itself generates.

The workflow of the FitzHugh-Nagumo form: fine trajectories (128 x 128, every z-plane a sample) from the plain law
(tests/laws/fhn_rk4.law) through the law backend, averaged 4 x 4 onto the 32 x 32 lattice; the coarse plain step
(the same law on 32 x 32) from each averaged frame; the network trained so that coarse step + correction lands on the
next averaged frame; then the learned solve: coarse step, guarded correction, frame after frame. The plain fine law
stays the judge of the error and the fallback: a correction that leaves a cell outside the range, or not finite, is
not applied (decided on the card).
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .solver import Solver

W_SIZES = (32 * 64, 80 * 64, 80 * 16)


def pack(W1, b1, W2, b2, W3, b3, Wt=None):
    """The flat weight vector from layer matrices (inputs x outputs) and biases: W1 18 x 64, W2 64 x 64, W3 64 x 2, and
    Wt (64) the first layer's weights of the time input (zero when None)."""
    w1 = np.zeros((32, 64), np.float32)
    w1[:18] = W1
    w1[18] = b1
    if Wt is not None:
        w1[19] = Wt
    w2 = np.zeros((80, 64), np.float32)
    w2[:64] = W2
    w2[64] = b2
    w3 = np.zeros((80, 16), np.float32)
    w3[:64, :2] = W3
    w3[64, :2] = b3
    return np.concatenate([w1.reshape(-1), w2.reshape(-1), w3.reshape(-1)])


def init_weights(seed, out_scale=1e-3):
    """He-initialised hidden layers, a small last layer (the correction starts near zero), zero biases."""
    rng = np.random.default_rng(seed)
    W1 = rng.normal(0.0, np.sqrt(2.0 / 19), (18, 64))
    W2 = rng.normal(0.0, np.sqrt(2.0 / 64), (64, 64))
    W3 = rng.normal(0.0, out_scale, (64, 2))
    Wt = rng.normal(0.0, np.sqrt(2.0 / 19), 64)
    return pack(W1, np.zeros(64), W2, np.zeros(64), W3, np.zeros(2), Wt)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class Corrector:
    """The network's weights on the card, its training step and its guarded application."""

    def __init__(self, weights=None):
        self._lib = _lib.lib()
        h = ctypes.c_void_p()
        _lib.check(self._lib.fe_corr_create(ctypes.byref(h)))
        self._h = h
        self.count = self._lib.fe_corr_weight_count()
        self.time_scale = 1.0   # the time input is the state's time times this (set by train_correction)
        self.set_weights(init_weights(0) if weights is None else weights)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.fe_corr_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        assert w.size == self.count
        _lib.check(self._lib.fe_corr_set_weights(self._h, w.ctypes.data_as(ctypes.c_void_p)))

    def weights(self):
        out = np.empty(self.count, np.float32)
        _lib.check(self._lib.fe_corr_get_weights(self._h, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    @staticmethod
    def _check(*ts):
        for t in ts:
            assert t.is_cuda and t.dtype == torch.float32 and t.is_contiguous() and t.dim() == 3

    def grads(self, u, v, tu, tv, time=0.0):
        """(loss, gradient) on (nz, ny, nx) CUDA float32 tensors; `time` the time of the state being corrected."""
        self._check(u, v, tu, tv)
        nz, ny, nx = u.shape
        torch.cuda.current_stream().synchronize()
        loss = ctypes.c_double()
        g = np.empty(self.count, np.float32)
        _lib.check(self._lib.fe_corr_grads(self._h, _ptr(u), _ptr(v), _ptr(tu), _ptr(tv), nx, ny, nz, float(time), None,
                                           ctypes.byref(loss), g.ctypes.data_as(ctypes.c_void_p)))
        return loss.value, g

    def train_step(self, u, v, tu, tv, lr, time=0.0, want_loss=False):
        self._check(u, v, tu, tv)
        nz, ny, nx = u.shape
        torch.cuda.current_stream().synchronize()
        loss = ctypes.c_double()
        _lib.check(self._lib.fe_corr_train_step(self._h, _ptr(u), _ptr(v), _ptr(tu), _ptr(tv), nx, ny, nz, float(time), None,
                                                float(lr), ctypes.byref(loss) if want_loss else None))
        return loss.value if want_loss else None

    def apply(self, u, v, lo=-1000.0, hi=1000.0, time=0.0, wait=True, stream=None):
        """(u, v) += correction in place, guarded; returns whether the plain step was kept (None when not waited)."""
        self._check(u, v)
        nz, ny, nx = u.shape
        rev = ctypes.c_int(0)
        _lib.check(self._lib.fe_corr_apply(self._h, _ptr(u), _ptr(v), nx, ny, nz, float(time), float(lo), float(hi),
                                           ctypes.c_void_p(stream) if stream else None, ctypes.byref(rev) if wait else None))
        return bool(rev.value) if wait else None


    def apply_solver(self, solver, time=0.0, lo=-1000.0, hi=1000.0):
        """Corrects the fields u and v of a law backend handle in place on its own stream, after its step, guarded; no
        host wait (the verdict stays on the card). `time` is the solve's time (scaled by time_scale for the network)."""
        nz, ny, nx = solver.shape
        u, v = solver.device_ptr("u"), solver.device_ptr("v")
        _lib.check(self._lib.fe_corr_apply(self._h, ctypes.c_void_p(u), ctypes.c_void_p(v), nx, ny, nz, float(time * self.time_scale), float(lo),
                                           float(hi), ctypes.c_void_p(solver.stream), None))
        solver.mark_edited("u")
        solver.mark_edited("v")


FHN_LAW_FILE = "fhn_rk4.law"


def fhn_initial(seeds, n):
    """PDEBench's diffusion-reaction start: u0 then v0 drawn N(0, 1) per cell from default_rng(seed), per sample."""
    u = np.empty((len(seeds), n, n), np.float32)
    v = np.empty((len(seeds), n, n), np.float32)
    for i, s in enumerate(seeds):
        rng = np.random.default_rng(s)
        u[i] = rng.normal(size=(n, n))
        v[i] = rng.normal(size=(n, n))
    return u, v


def block_mean(x, f):
    """(nz, n, n) -> (nz, n/f, n/f) block means."""
    nz, ny, nx = x.shape
    return x.reshape(nz, ny // f, f, nx // f, f).mean(axis=(2, 4))


class PlainFHN:
    """The plain law on an n x n lattice of `samples` z-planes over [-1, 1]^2, stepped frame by frame (dt = frame)."""

    def __init__(self, law_text, n, samples, frame=0.05):
        self.n = n
        self.samples = samples
        self.frame = frame
        self.solver = Solver(law_text, n, n, samples, 2.0 / n, "fhn_rk4.law")
        self.solver.set_deferred(True)

    def close(self):
        self.solver.close()

    def set(self, u, v):
        if isinstance(u, torch.Tensor):
            torch.cuda.current_stream().synchronize()
            self.solver.set_field_device("u", u.contiguous())
            self.solver.set_field_device("v", v.contiguous())
        else:
            self.solver.set_field("u", u)
            self.solver.set_field("v", v)

    def step(self):
        self.solver.step(self.frame)

    def get(self):
        u = torch.empty((self.samples, self.n, self.n), dtype=torch.float32, device="cuda")
        v = torch.empty_like(u)
        self.solver.fetch_device("u", u)
        self.solver.fetch_device("v", v)
        return u, v

    def substeps(self):
        return max(self.solver.last_substeps())


def fine_frames(law_text, seeds, frames, fine=128, coarse=32, frame=0.05):
    """The plain law's solves at `fine` resolution from fhn_initial(seeds), each frame averaged onto `coarse`: a list of
    frames + 1 (u, v) CUDA tensor pairs (nz = len(seeds))."""
    import torch.nn.functional as F
    u0, v0 = fhn_initial(seeds, fine)
    s = PlainFHN(law_text, fine, len(seeds), frame)
    s.set(u0, v0)
    f = fine // coarse
    out = []
    for t in range(frames + 1):
        if t:
            s.step()
        u, v = s.get()
        out.append((F.avg_pool2d(u[:, None], f)[:, 0].contiguous(), F.avg_pool2d(v[:, None], f)[:, 0].contiguous()))
    s.close()
    return out


def train_correction(corr, law_text, targets, iters=3000, rounds=2, lr=2e-3, frame=0.05, horizon=None):
    """Trains `corr` so that the coarse plain step + correction lands on the next target frame. First on the targets'
    own frames (teacher forcing), then `rounds` times on the states the learned solver itself reaches from the first
    frame (its rollouts), so it learns to correct what it will see. After each phase the rollout error on the training
    targets is measured and the best weights are kept. The time input is the state's time over `horizon` (the
    targets' span by default). Returns (best rollout RMSE, RMSE of the plain coarse rollout) on the training targets."""
    frames = len(targets) - 1
    nz, n, _ = targets[0][0].shape
    horizon = horizon or frames * frame
    corr.time_scale = 1.0 / horizon
    coarse = PlainFHN(law_text, n, nz, frame)

    def pairs_from(states):
        out = []
        for k in range(frames):
            coarse.set(*states[k])
            coarse.step()
            out.append((*coarse.get(), *targets[k + 1], (k + 1) * frame / horizon))
        return out

    def fit(pairs, steps, rate):
        for it in range(steps):
            u, v, tu, tv, t = pairs[it % frames]
            corr.train_step(u, v, tu, tv, rate if it < 2 * steps // 3 else rate / 4, time=t)

    def rollout(correct):
        states = [targets[0]]
        u, v = targets[0]
        err = 0.0
        for k in range(frames):
            coarse.set(u, v)
            coarse.step()
            u, v = coarse.get()
            if correct:
                corr.apply(u, v, time=(k + 1) * frame / horizon)
            states.append((u, v))
            tu, tv = targets[k + 1]
            err += float(((u - tu) ** 2 + (v - tv) ** 2).mean() / 2)
        return states, (err / frames) ** 0.5

    _, plain = rollout(False)
    pairs = pairs_from(targets)
    fit(pairs, iters, lr)
    states, best = rollout(True)
    best_w = corr.weights()
    for _ in range(rounds):
        mixed = pairs_from(states)
        fit([mixed[k] if k % 2 else pairs[k] for k in range(frames)], iters, lr / 2)
        states, err = rollout(True)
        if err < best:
            best, best_w = err, corr.weights()
    corr.set_weights(best_w)
    coarse.close()
    return best, plain
