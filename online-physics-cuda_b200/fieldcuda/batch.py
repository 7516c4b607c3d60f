"""One law on many uneven lattices, stepped together (fe_batch_*).

The reference batches instances as the z-planes of one lattice of one nx x ny (bench/finance.py:253-288,
bench/pdebench.py:71-92). A LawBatch takes instances of any extents: those of equal (nx, ny, h) are stacked along z
into one lattice when the law couples nothing along z, every other instance is a lattice of its own, and a step
launches all lattices on their own streams before judging their contracts.

    b = LawBatch(law_text, [(64, 64, 10, 1/64), (128, 128, 3, 1/128), (64, 64, 5, 1/64)])
    b.set_field(0, "u", u0)           # (nz, ny, nx) float32 of instance 0
    b.step(dt)
    u = b.values(2, "u")
"""
import ctypes

import numpy as np

from . import _lib
from .solver import Solver, Violation


class LawBatch:
    def __init__(self, law_text, lattices):
        self._lib = _lib.lib()
        descs = (_lib.fe_batch_desc * len(lattices))()
        for d, (nx, ny, nz, h) in zip(descs, lattices):
            d.nx, d.ny, d.nz, d.h = int(nx), int(ny), int(nz), float(h)
        self.shapes = [(int(nz), int(ny), int(nx)) for nx, ny, nz, _ in lattices]
        handle = ctypes.c_void_p()
        _lib.check(self._lib.fe_batch_create(law_text.encode(), descs, len(lattices), ctypes.byref(handle)))
        self._b = handle
        law = ctypes.c_void_p()
        _lib.check(self._lib.fe_batch_law(self._b, 0, ctypes.byref(law), None))
        nx, ny, nz, h = lattices[0]
        self._names = Solver.borrow(law, (nz, ny, nx), h)
        self.field_names = self._names.field_names
        self.term_names = self._names.term_names
        self._violations = []

    def close(self):
        if getattr(self, "_b", None) is not None and self._b.value:
            if getattr(self, "_names", None) is not None:
                self._names.close()  # a borrowed view: forgets the handle, which fe_batch_destroy frees
            self._lib.fe_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        """(lattices, stacked): how many law handles the instances went into, and whether equal shapes were stacked."""
        n, stacked = ctypes.c_int(), ctypes.c_int()
        _lib.check(self._lib.fe_batch_info(self._b, ctypes.byref(n), ctypes.byref(stacked)))
        return n.value, bool(stacked.value)

    def _field(self, name):
        if name not in self.field_names:
            raise KeyError(f"the law has no field '{name}'")
        return self.field_names.index(name)

    def set_param(self, name, value):
        p = self._lib.fe_law_param_id(self._names._h, name.encode())
        if p < 0:
            raise KeyError(f"the law has no param '{name}'")
        _lib.check(self._lib.fe_batch_set_param(self._b, p, float(value)))

    def set_field(self, instance, name, values):
        v = np.ascontiguousarray(values, np.float32)
        if v.shape != self.shapes[instance]:
            raise ValueError(f"instance {instance} is {self.shapes[instance]}, not {v.shape}")
        _lib.check(self._lib.fe_batch_upload(self._b, instance, self._field(name), v.ctypes.data_as(ctypes.c_void_p)))

    def values(self, instance, name):
        out = np.empty(self.shapes[instance], np.float32)
        _lib.check(self._lib.fe_batch_fetch(self._b, instance, self._field(name), out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def step(self, dt, respect_max_dt=True):
        n = ctypes.c_int()
        flags = 0 if respect_max_dt else _lib.FE_STEP_IGNORE_MAX_DT
        _lib.check(self._lib.fe_batch_step(self._b, float(dt), flags, ctypes.byref(n)))
        self._violations = []
        for i in range(n.value):
            raw, inst = _lib.fe_violation(), ctypes.c_int()
            _lib.check(self._lib.fe_batch_violation(self._b, i, ctypes.byref(inst), ctypes.byref(raw)))
            self._violations.append((inst.value, Violation(raw, self._names)))

    def violations(self):
        """(instance, Violation) of the last step; instance -1 for a conserved total of a lattice of several."""
        return list(self._violations)
