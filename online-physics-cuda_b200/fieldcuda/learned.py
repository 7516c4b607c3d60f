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


def pack(W1, b1, W2, b2, W3, b3):
    """The flat weight vector from layer matrices (inputs x outputs) and biases: W1 18 x 64, W2 64 x 64, W3 64 x 2."""
    w1 = np.zeros((32, 64), np.float32)
    w1[:18] = W1
    w1[18] = b1
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
    W1 = rng.normal(0.0, np.sqrt(2.0 / 18), (18, 64))
    W2 = rng.normal(0.0, np.sqrt(2.0 / 64), (64, 64))
    W3 = rng.normal(0.0, out_scale, (64, 2))
    return pack(W1, np.zeros(64), W2, np.zeros(64), W3, np.zeros(2))


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

    def grads(self, u, v, tu, tv):
        """(loss, gradient) on (nz, ny, nx) CUDA float32 tensors."""
        self._check(u, v, tu, tv)
        nz, ny, nx = u.shape
        torch.cuda.current_stream().synchronize()
        loss = ctypes.c_double()
        g = np.empty(self.count, np.float32)
        _lib.check(self._lib.fe_corr_grads(self._h, _ptr(u), _ptr(v), _ptr(tu), _ptr(tv), nx, ny, nz, None, ctypes.byref(loss),
                                           g.ctypes.data_as(ctypes.c_void_p)))
        return loss.value, g

    def train_step(self, u, v, tu, tv, lr, want_loss=False):
        self._check(u, v, tu, tv)
        nz, ny, nx = u.shape
        torch.cuda.current_stream().synchronize()
        loss = ctypes.c_double()
        _lib.check(self._lib.fe_corr_train_step(self._h, _ptr(u), _ptr(v), _ptr(tu), _ptr(tv), nx, ny, nz, None, float(lr),
                                                ctypes.byref(loss) if want_loss else None))
        return loss.value if want_loss else None

    def apply(self, u, v, lo=-1000.0, hi=1000.0, wait=True, stream=None):
        """(u, v) += correction in place, guarded; returns whether the plain step was kept (None when not waited)."""
        self._check(u, v)
        nz, ny, nx = u.shape
        rev = ctypes.c_int(0)
        _lib.check(self._lib.fe_corr_apply(self._h, _ptr(u), _ptr(v), nx, ny, nz, float(lo), float(hi),
                                           ctypes.c_void_p(stream) if stream else None, ctypes.byref(rev) if wait else None))
        return bool(rev.value) if wait else None


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
