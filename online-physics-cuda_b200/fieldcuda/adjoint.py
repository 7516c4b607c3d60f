"""Reverse mode through a law's steps: the IR-generated adjoint law, a sqrt(N)-checkpointed VJP driver and a
torch.autograd.Function over it.

The reference differentiates one term of a law by generating an adjoint law from its IR (src/field/ir/Adjoint.cpp) and
running it backward over every state the forward kept on the host (tools/lawc/main.cpp:274-361). Here the adjoint law
comes from this backend's IR (fe_law_adjoint: transposed stencils, and tridiagonal solves by their transposes, which the
reference refuses), both laws run as generated sm_100a kernels, and the forward keeps only every K-th state on the
device (K = ceil(sqrt(N))): the backward pass recomputes each segment's K states from its checkpoint, then steps the
adjoint law back over them. Memory: about 2 sqrt(N) copies of the moving fields; work: about two forward passes and
one adjoint pass.
"""
import math

import torch

from . import _lib
from .solver import Solver


def adjoint_law(law_text, term=None):
    """The adjoint law of `term` (the first when None) as text; raises FeError (FE_EUNSUP) with the reason when an op
    on the path has no adjoint."""
    return _lib.text_call("fe_law_adjoint", law_text.encode(), (term or "").encode())


class LawVJP:
    """N steps of one term of a law and their vector-Jacobian product.

    The term must be the only one that moves anything, one substep a step (dt within its max_dt). Fields the term
    writes are the state; the others it reads are static inputs; their cotangents, and the params', accumulate over
    the backward pass (a param's cotangent is a field whose total is the gradient)."""

    def __init__(self, law_text, nx, ny, nz, h, term=None, name="law"):
        self.shape = (nz, ny, nx)
        self.h = h
        self.primal = Solver(law_text, nx, ny, nz, h, name)
        self.adjoint_text = adjoint_law(law_text, term)
        self.adj = Solver(self.adjoint_text, nx, ny, nz, h, name + "__adj")
        adj_static = [f for f in self.adj.field_names if self.adj.field_info(f)["static"]]
        self.state = [f for f in self.primal.field_names if f + "__adj" in self.adj.field_names and
                      not self.primal.field_info(f)["static"]]
        self.inputs = [f for f in adj_static if f in self.primal.field_names]
        self.statics = [f for f in self.inputs if f not in self.state]
        self.params = [f[:-5] for f in self.adj.field_names if f.endswith("__adj") and f[:-5] not in self.primal.field_names]
        for s in (self.primal, self.adj):
            s.set_deferred(True)
        self._fields = None
        self._checkpoints = []
        self.steps = 0
        self.dt = 0.0

    def close(self):
        self.primal.close()
        self.adj.close()

    def _snapshot(self):
        out = {}
        for f in self.state:
            t = torch.empty(self.shape, dtype=torch.float32, device="cuda")
            self.primal.fetch_device(f, t)
            out[f] = t
        return out

    def _restore(self, snap):
        for f, t in snap.items():
            self.primal.set_field_device(f, t)

    def set_param(self, name, value):
        self.primal.set_param(name, value)
        self.adj.set_param(name, value)

    def forward(self, fields, dt, steps, every=None):
        """Steps the law `steps` times from `fields` (name -> CUDA float32 tensor of the lattice; missing fields keep
        their values) and returns the state fields at the end. Keeps every `every`-th state (default ceil(sqrt(N)))."""
        torch.cuda.current_stream().synchronize()
        self._fields = {k: v.detach().contiguous() for k, v in fields.items()}
        for f, t in self._fields.items():
            self.primal.set_field_device(f, t)
        self.steps = int(steps)
        self.dt = float(dt)
        self.every = int(every or max(1, math.ceil(math.sqrt(self.steps))))
        self._checkpoints = []
        for s in range(self.steps):
            if s % self.every == 0:
                self._checkpoints.append(self._snapshot())
            self.primal.step(self.dt)
            if max(self.primal.last_substeps()) != 1:
                raise RuntimeError("the differentiated term took more than one substep: give a dt within its max_dt")
        self.primal.sync()
        if self.primal.violations():
            raise RuntimeError(f"the forward broke a contract: {self.primal.violations()}")
        return self._snapshot()

    def backward(self, seeds):
        """Cotangents of the forward's inputs given those of its outputs (name -> tensor; missing state seeds are zero).
        Returns name -> tensor for every state and static field and every param (a param's tensor sums to its
        gradient)."""
        if not self._checkpoints:
            raise RuntimeError("backward before forward")
        torch.cuda.current_stream().synchronize()
        zero = torch.zeros(self.shape, dtype=torch.float32, device="cuda")
        for f in self.adj.field_names:
            if f.endswith("__adj"):
                seed = seeds.get(f[:-5]) if f[:-5] in self.state else None
                self.adj.set_field_device(f, seed.detach().contiguous() if seed is not None else zero)
        for f in self.statics:
            if f in self._fields:
                self.adj.set_field_device(f, self._fields[f])
            else:
                t = torch.empty(self.shape, dtype=torch.float32, device="cuda")
                self.primal.fetch_device(f, t)
                self.adj.set_field_device(f, t)
        for seg in range(len(self._checkpoints) - 1, -1, -1):
            start = seg * self.every
            end = min(self.steps, start + self.every)
            self._restore(self._checkpoints[seg])
            states = []
            for s in range(start, end):
                states.append(self._snapshot())
                if s + 1 < end:
                    self.primal.step(self.dt)
            for s in range(end - 1, start - 1, -1):
                for f, t in states[s - start].items():
                    self.adj.set_field_device(f, t)
                self.adj.step(self.dt)
        self.adj.sync()
        out = {}
        for f in self.adj.field_names:
            if f.endswith("__adj"):
                t = torch.empty(self.shape, dtype=torch.float32, device="cuda")
                self.adj.fetch_device(f, t)
                out[f[:-5]] = t
        return out


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
