"""Reverse mode through a law's steps: the IR-generated adjoint law, the native sqrt(N)-checkpointed VJP driver
(fe_vjp_*) and a torch.autograd.Function over it.

The reference differentiates one term of a law by generating an adjoint law from its IR (src/field/ir/Adjoint.cpp) and
running it backward over every state the forward kept on the host (tools/lawc/main.cpp:274-361). Here the adjoint law
comes from this backend's IR (fe_law_adjoint: transposed stencils, and tridiagonal solves by their transposes, which the
reference refuses), both laws run as generated sm_100a kernels, and the driver (csrc/vjp.cpp) keeps only every K-th
state on the device (K = ceil(sqrt(N))): the backward pass recomputes each segment's K states from its checkpoint, then
steps the adjoint law back over them. Memory: about 2 sqrt(N) copies of the moving fields; work: about two forward
passes and one adjoint pass.
"""
import ctypes

import torch

from . import _lib
from .solver import Solver


def adjoint_law(law_text, term=None):
    """The adjoint law of `term` (the first when None) as text; raises FeError (FE_EUNSUP) with the reason when an op
    on the path has no adjoint."""
    return _lib.text_call("fe_law_adjoint", law_text.encode(), (term or "").encode())


class LawVJP:
    """N steps of one term of a law and their vector-Jacobian product (fe_vjp_*).

    The term must be the only one that moves anything, one substep a step (dt within its max_dt). Fields the term
    writes are the state; the others it reads are static inputs; their cotangents, and the params', accumulate over
    the backward pass (a param's cotangent is a field whose total is the gradient)."""

    def __init__(self, law_text, nx, ny, nz, h, term=None, name="law"):
        self._lib = _lib.lib()
        self.shape = (nz, ny, nx)
        self.h = h
        handle = ctypes.c_void_p()
        _lib.check(self._lib.fe_vjp_create(law_text.encode(), (term or "").encode(), nx, ny, nz, float(h), ctypes.byref(handle)))
        self._v = handle
        primal, adj = ctypes.c_void_p(), ctypes.c_void_p()
        _lib.check(self._lib.fe_vjp_laws(self._v, ctypes.byref(primal), ctypes.byref(adj)))
        self.primal = Solver.borrow(primal, self.shape, h)
        self.adj = Solver.borrow(adj, self.shape, h)
        self.adjoint_text = adjoint_law(law_text, term)
        adj_static = [f for f in self.adj.field_names if self.adj.field_info(f)["static"]]
        self.state = [f for f in self.primal.field_names if f + "__adj" in self.adj.field_names and
                      not self.primal.field_info(f)["static"]]
        self.inputs = [f for f in adj_static if f in self.primal.field_names]
        self.statics = [f for f in self.inputs if f not in self.state]
        self.params = [f[:-5] for f in self.adj.field_names if f.endswith("__adj") and f[:-5] not in self.primal.field_names]
        self.steps = 0
        self.dt = 0.0

    def close(self):
        if getattr(self, "_v", None) is not None and self._v.value:
            for view in (getattr(self, "primal", None), getattr(self, "adj", None)):
                if view is not None:
                    view.close()  # a borrowed view: forgets the handle, which fe_vjp_destroy frees
            self._lib.fe_vjp_destroy(self._v)
            self._v = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _snapshot(self):
        out = {}
        for f in self.state:
            t = torch.empty(self.shape, dtype=torch.float32, device="cuda")
            self.primal.fetch_device(f, t)
            out[f] = t
        return out

    def set_param(self, name, value):
        _lib.check(self._lib.fe_vjp_set_param(self._v, name.encode(), float(value)))

    def forward(self, fields, dt, steps, every=None):
        """Steps the law `steps` times from `fields` (name -> CUDA float32 tensor of the lattice; missing fields keep
        their values) and returns the state fields at the end. Keeps every `every`-th state (default ceil(sqrt(N)))."""
        torch.cuda.current_stream().synchronize()
        for f, t in fields.items():
            self.primal.set_field_device(f, t.detach().contiguous())
        self.steps = int(steps)
        self.dt = float(dt)
        _lib.check(self._lib.fe_vjp_forward(self._v, self.dt, self.steps, int(every or 0)))
        return self._snapshot()

    def backward(self, seeds):
        """Cotangents of the forward's inputs given those of its outputs (name -> tensor; missing state seeds are zero).
        Returns name -> tensor for every state and static field and every param (a param's tensor sums to its
        gradient)."""
        torch.cuda.current_stream().synchronize()
        zero = torch.zeros(self.shape, dtype=torch.float32, device="cuda")
        for f in self.adj.field_names:
            if f.endswith("__adj"):
                seed = seeds.get(f[:-5]) if f[:-5] in self.state else None
                self.adj.set_field_device(f, seed.detach().contiguous() if seed is not None else zero)
        _lib.check(self._lib.fe_vjp_backward(self._v))
        out = {}
        for f in self.adj.field_names:
            if f.endswith("__adj"):
                t = torch.empty(self.shape, dtype=torch.float32, device="cuda")
                self.adj.fetch_device(f, t)
                out[f[:-5]] = t
        return out

    def param_grad(self, name):
        """A param's gradient after backward(): the FP64 total of its cotangent field."""
        g = ctypes.c_double()
        _lib.check(self._lib.fe_vjp_param_grad(self._v, name.encode(), ctypes.byref(g)))
        return g.value


class LawSteps(torch.autograd.Function):
    """``LawSteps.apply(vjp, dt, steps, names, *tensors)``: the state fields after `steps` steps of the law from the
    given fields (names[i] -> tensors[i], CUDA float32 lattices), differentiable in every given field."""

    @staticmethod
    def forward(ctx, vjp, dt, steps, names, *tensors):
        out = vjp.forward(dict(zip(names, tensors)), dt, steps)
        ctx.vjp = vjp
        ctx.names = names
        return tuple(out[f] for f in vjp.state)

    @staticmethod
    def backward(ctx, *grads):
        vjp = ctx.vjp
        seeds = {f: g for f, g in zip(vjp.state, grads) if g is not None}
        cot = vjp.backward(seeds)
        ctx.param_grads = {p: float(cot[p].double().sum()) for p in vjp.params if p in cot}
        vjp.param_grads = ctx.param_grads
        return (None, None, None, None) + tuple(cot.get(n) for n in ctx.names)
