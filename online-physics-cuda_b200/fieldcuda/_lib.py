"""ctypes binding of libfe_b200.so (include/fe.h).

The shared library is built in-tree (``make -C online-physics-cuda_b200``). Loading it needs no GPU; every compute
entry point checks for an sm_100 device itself and returns FE_ENODEV without one. There is no CPU fallback: if the
library is missing, :func:`lib` raises.
"""
import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
PACKAGE = os.path.dirname(HERE)
LIB_PATH = os.path.join(PACKAGE, "libfe_b200.so")

FE_OK = 0
FE_EINVAL = 1
FE_ENODEV = 2
FE_ECUDA = 3
FE_ELAW = 4
FE_EUNSUP = 5
FE_EKERNEL = 6

FE_HEAT7_BEFORE = 1
FE_HEAT7_AFTER = 2

_c = ctypes
_lock = threading.Lock()
_lib = None


class FeError(RuntimeError):
    """A failing fe_* call: ``code`` is its status, the message is fe_last_error()."""

    def __init__(self, code, message):
        super().__init__(f"[fe status {code}] {message}")
        self.code = code


class fe_check(ctypes.Structure):
    """Mirror of ``fe_check`` (include/fe.h)."""

    _fields_ = [
        ("before", _c.c_double),
        ("before_abs", _c.c_double),
        ("after", _c.c_double),
        ("after_abs", _c.c_double),
        ("out_of_range", _c.c_uint32),
        ("not_finite", _c.c_uint32),
        ("first_bad", _c.c_uint32),
        ("lo_inv", _c.c_uint32),
        ("hi_key", _c.c_uint32),
        ("changed", _c.c_uint32),
        ("pad", _c.c_uint32 * 2),
    ]


# name -> (restype, argtypes). Every symbol include/fe.h declares is listed here (a CPU test checks both ways).
SIGNATURES = {
    "fe_version": (_c.c_int, []),
    "fe_last_error": (_c.c_char_p, []),
    "fe_device_check": (_c.c_int, []),
    "fe_key_to_float": (_c.c_float, [_c.c_uint32]),
    "fe_heat7_workspace_bytes": (_c.c_size_t, [_c.c_int, _c.c_int, _c.c_int, _c.c_int, _c.c_int]),
    "fe_heat7_rows": (_c.c_int, [_c.c_int]),
    "fe_heat7_step": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_int, _c.c_int, _c.c_int, _c.c_float, _c.c_float,
                                 _c.c_float, _c.c_float, _c.c_float, _c.c_int, _c.c_int, _c.c_int, _c.c_void_p,
                                 _c.c_void_p]),
    "fe_check_reset": (_c.c_int, [_c.c_void_p, _c.c_void_p]),
    "fe_check_read": (_c.c_int, [_c.c_void_p, _c.POINTER(fe_check), _c.c_void_p]),
    "fe_copy_f32": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_size_t, _c.c_void_p]),
}


def lib():
    """The loaded library (raises if it was not built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise FeError(FE_ENODEV, f"{LIB_PATH} is not built: run `make -C {PACKAGE}`")
            handle = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(handle, name)
                fn.restype = res
                fn.argtypes = args
            _lib = handle
        return _lib


def last_error():
    msg = lib().fe_last_error()
    return msg.decode() if msg else ""


def check(status):
    """Raises FeError for a non-zero status."""
    if status != FE_OK:
        raise FeError(status, last_error())
    return status


def call(name, *args):
    """Calls fe_<name> and raises on a non-zero status."""
    return check(getattr(lib(), name)(*args))
