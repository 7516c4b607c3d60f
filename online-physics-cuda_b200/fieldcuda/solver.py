"""The reference's field API on the B200 backend.

:class:`Solver` mirrors the reference's ``Solver`` (src/field/Solver.hpp:23-129): construct it from law text and a
lattice, write fields, ``step(dt)``, read fields, read the violations of the contracts. Under it every call goes to
libfe_b200.so through include/fe.h; there is no CPU path (the reference's CPU solver is the oracle, not a fallback).
Fields are numpy arrays shaped (nz, ny, nx), x fastest, float32 — the reference's FieldSet order (Grid.hpp:25-30).

Lazy readback is how this backend always works: a step leaves the fields on the card, and ``values``/``fields`` bring
them back when asked (the reference's ``set_lazy_readback(true)``, Solver.hpp:49-53).
"""
import ctypes

import numpy as np

from . import _lib

KIND_NAMES = {0: "range", 1: "not-finite", 2: "conservation", 3: "substep-cap"}


class Violation:
    """A broken contract (Backend.hpp:16-22): kind, term and field names, the step, and the numbers behind it."""

    def __init__(self, raw, solver):
        self.kind = KIND_NAMES.get(raw.kind, "?")
        self.term = solver.term_names[raw.term] if 0 <= raw.term < len(solver.term_names) else ""
        self.field = solver.field_names[raw.field] if 0 <= raw.field < len(solver.field_names) else ""
        self.count = raw.count
        self.first_cell = raw.first_cell
        self.before, self.after, self.tolerance = raw.before, raw.after, raw.tolerance
        self.step = raw.step
        self.detail = raw.detail.decode(errors="replace")

    def __repr__(self):
        return f"Violation({self.kind}, term={self.term!r}, field={self.field!r}, step={self.step}, {self.detail})"


class Solver:
    """A compiled law integrated on one lattice of nx*ny*nz cells of edge h, on the current CUDA device."""

    def __init__(self, law_text, nx, ny, nz, h, source_name="law"):
        self._lib = _lib.lib()
        handle = ctypes.c_void_p()
        _lib.check(self._lib.fe_law_create(law_text.encode(), source_name.encode(), nx, ny, nz, float(h),
                                           ctypes.byref(handle)))
        self._attach(handle, (nz, ny, nx), h, owned=True)

    @classmethod
    def borrow(cls, handle, shape, h):
        """A view of a law handle another object owns (a VJP's primal or adjoint law): close() leaves it alone."""
        s = cls.__new__(cls)
        s._lib = _lib.lib()
        s._attach(handle, shape, h, owned=False)
        return s

    def _attach(self, handle, shape, h, owned):
        self._h = handle
        self._owned = owned
        self.shape = tuple(shape)
        self.h = h
        self.respect_max_dt = True
        n = self._lib.fe_law_field_count(self._h)
        self.field_names = []
        for f in range(n):
            buf = ctypes.create_string_buffer(256)
            _lib.check(self._lib.fe_law_field_name(self._h, f, buf, 256))
            self.field_names.append(buf.value.decode())
        self.term_names = []
        for t in range(self._lib.fe_law_term_count(self._h)):
            buf = ctypes.create_string_buffer(256)
            _lib.check(self._lib.fe_law_term_name(self._h, t, buf, 256))
            self.term_names.append(buf.value.decode())
        self._info = _lib.fe_step_info()

    # ---- lifetime ------------------------------------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            if self._owned:
                self._lib.fe_law_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- fields and params ---------------------------------------------------------------------------------------
    def field(self, name):
        """A field's id (Solver::field), -1 if the law has none of that name."""
        return self._lib.fe_law_field_id(self._h, name.encode())

    def _id(self, field):
        if isinstance(field, str):
            f = self.field(field)
            if f < 0:
                raise KeyError(f"the law has no field {field!r}")
            return f
        return int(field)

    def field_info(self, field):
        info = _lib.fe_field_info()
        _lib.check(self._lib.fe_law_field_info(self._h, self._id(field), ctypes.byref(info)))
        return {"init": info.init, "lo": info.lo, "hi": info.hi, "static": bool(info.is_static),
                "derived": bool(info.derived), "clamp": bool(info.clamp)}

    def set_param(self, name, value):
        p = self._lib.fe_law_param_id(self._h, name.encode())
        if p < 0:
            return False
        _lib.check(self._lib.fe_law_set_param(self._h, p, float(value)))
        return True

    def param(self, name):
        p = self._lib.fe_law_param_id(self._h, name.encode())
        if p < 0:
            return None
        v = ctypes.c_double()
        _lib.check(self._lib.fe_law_get_param(self._h, p, ctypes.byref(v)))
        return v.value

    def set_field(self, field, values):
        """Writes a whole field from the host (the reference's edit of fields(); FieldEdits::all)."""
        a = np.ascontiguousarray(values, dtype=np.float32)
        if a.size != np.prod(self.shape):
            raise ValueError(f"field holds {np.prod(self.shape)} cells, got {a.size}")
        _lib.check(self._lib.fe_law_upload(self._h, self._id(field), a.ctypes.data_as(ctypes.c_void_p)))

    def set_field_device(self, field, tensor):
        """Writes a whole field from a CUDA tensor of nx*ny*nz float32."""
        _lib.check(self._lib.fe_law_upload_device(self._h, self._id(field), ctypes.c_void_p(tensor.data_ptr())))

    def values(self, field):
        """One field's cells, brought back from the card (Solver::values)."""
        out = np.empty(self.shape, dtype=np.float32)
        _lib.check(self._lib.fe_law_fetch(self._h, self._id(field), out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def mark_edited(self, field):
        """The field's device buffer (device_ptr) was changed in place on this solver's stream."""
        _lib.check(self._lib.fe_law_mark_edited(self._h, self._id(field)))

    def fetch_device(self, field, tensor):
        _lib.check(self._lib.fe_law_fetch_device(self._h, self._id(field), ctypes.c_void_p(tensor.data_ptr())))

    def fields(self):
        """Every field by name (Solver::fields)."""
        return {n: self.values(i) for i, n in enumerate(self.field_names)}

    def device_ptr(self, field):
        p = ctypes.c_void_p()
        _lib.check(self._lib.fe_law_field_device_ptr(self._h, self._id(field), ctypes.byref(p)))
        return p.value

    @property
    def stream(self):
        s = ctypes.c_void_p()
        _lib.check(self._lib.fe_law_stream(self._h, ctypes.byref(s)))
        return s.value

    # ---- stepping ------------------------------------------------------------------------------------------------
    def set_respect_max_dt(self, respect):
        """The falsification hook (Solver.hpp:91-93): ignore every max_dt."""
        self.respect_max_dt = bool(respect)

    def check_contracts_every(self, steps):
        _lib.check(self._lib.fe_law_check_every(self._h, int(steps)))

    def set_learned(self, on):
        """Learned schemes under guard (Solver::set_learned): a term's learned equations run first; a step that breaks a
        contract is undone and taken classically."""
        _lib.check(self._lib.fe_law_set_learned(self._h, 1 if on else 0))

    def term_learned(self):
        """Per term in the last step: "learned" (its learned scheme kept), "fell back" (undone), or "classical"."""
        names = {0: "classical", 1: "learned", 2: "fell back"}
        return [names.get(self._lib.fe_law_term_learned(self._h, t), "?") for t in range(len(self.term_names))]

    def set_deferred(self, on):
        """Judge the contracts at sync() instead of after every checked step."""
        _lib.check(self._lib.fe_law_set_deferred(self._h, 1 if on else 0))

    def step(self, dt):
        flags = 0 if self.respect_max_dt else _lib.FE_STEP_IGNORE_MAX_DT
        _lib.check(self._lib.fe_law_step(self._h, float(dt), flags, ctypes.byref(self._info)))

    def sync(self):
        _lib.check(self._lib.fe_law_sync(self._h, ctypes.byref(self._info)))

    def refresh_derived(self):
        _lib.check(self._lib.fe_law_derive(self._h))

    def violations(self):
        n = self._info.violations
        out = []
        for i in range(n):
            raw = _lib.fe_violation()
            if self._lib.fe_law_violation(self._h, i, ctypes.byref(raw)) == 0:
                out.append(Violation(raw, self))
        return out

    def last_substeps(self):
        return [self._lib.fe_law_substeps(self._h, t) for t in range(len(self.term_names))]

    def idle_terms(self):
        return [bool(self._lib.fe_law_term_idle(self._h, t)) for t in range(len(self.term_names))]

    def profile(self):
        return {"launches": self._info.launches, "gpu_ms": self._info.gpu_ms, "fallbacks": self._info.fallbacks}

    def digest(self):
        """FNV-1a over every field's bits in declaration order (FieldSet::digest)."""
        d = ctypes.c_uint64()
        _lib.check(self._lib.fe_law_digest(self._h, ctypes.byref(d)))
        return d.value

    # ---- one slab of a lattice split along z over ranks (fieldcuda.slabs) ---------------------------------------------
    def set_owned_z(self, z0, z1):
        """Contracts cover planes [z0, z1) of this handle only; the rest are halo planes another rank owns."""
        _lib.check(self._lib.fe_law_set_owned_z(self._h, int(z0), int(z1)))

    def mark_halo(self, field):
        """The field's halo planes were written in place (on this solver's stream): its bounds are forgotten."""
        _lib.check(self._lib.fe_law_mark_halo(self._h, self._id(field)))

    def set_external_conservation(self, on):
        """Checked steps log each conserves group's totals (take_totals) instead of judging them."""
        _lib.check(self._lib.fe_law_set_external_conservation(self._h, 1 if on else 0))

    def take_totals(self, room=4096):
        """The logged group totals since the last call, oldest first: dicts of step, term, group, substeps, before,
        after, scale."""
        buf = (_lib.fe_group_totals * room)()
        n = ctypes.c_int()
        _lib.check(self._lib.fe_law_take_totals(self._h, buf, room, ctypes.byref(n)))
        return [{"step": e.step, "term": e.term, "group": e.group, "substeps": e.substeps, "before": e.before, "after": e.after,
                 "scale": e.scale} for e in buf[:n.value]]

    def time_stage(self, term=0, stage=0, launches=10, dt=0.0):
        """(kernel name, ms for `launches` back-to-back launches of the term's stage `stage`)."""
        ms = ctypes.c_float()
        name = ctypes.create_string_buffer(128)
        _lib.check(self._lib.fe_law_time_stage(self._h, term, stage, launches, float(dt), ctypes.byref(ms), name, 128))
        return name.value.decode(), ms.value

    def time_gather(self, term=0, launches=10):
        ms = ctypes.c_float()
        _lib.check(self._lib.fe_law_time_gather(self._h, term, launches, ctypes.byref(ms)))
        return ms.value


def ir_json(law_text):
    """The IR as the reference's JSON (lawc --ir-json)."""
    return _lib.text_call("fe_law_ir_json", law_text.encode())


def ir_listing(law_text):
    return _lib.text_call("fe_law_ir_listing", law_text.encode())


def cuda_source(law_text, nx, ny, nz, h):
    """The generated CUDA translation unit (lawc --cuda)."""
    return _lib.text_call("fe_law_source", law_text.encode(), nx, ny, nz, float(h))


def plan_z_reach(law_text, nx, ny, nz, h):
    """(planes along z one step reads beyond a cell, reduces over the lattice, solves along z) for the planned law."""
    reach, flags = ctypes.c_int(), ctypes.c_int()
    _lib.check(_lib.lib().fe_law_plan_z_reach(law_text.encode(), nx, ny, nz, float(h), ctypes.byref(reach), ctypes.byref(flags)))
    return reach.value, bool(flags.value & 1), bool(flags.value & 2)


def compile_check(law_text, nx, ny, nz, h):
    """Lowers, generates and NVRTC-compiles the law for sm_100a (no GPU needed); raises on failure."""
    _lib.check(_lib.lib().fe_law_compile_check(law_text.encode(), nx, ny, nz, float(h)))
