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


class fe_violation(ctypes.Structure):
    _fields_ = [
        ("kind", _c.c_int), ("term", _c.c_int), ("field", _c.c_int), ("count", _c.c_uint32), ("first_cell", _c.c_uint32),
        ("before", _c.c_double), ("after", _c.c_double), ("tolerance", _c.c_double), ("step", _c.c_longlong),
        ("detail", _c.c_char * 160),
    ]


class fe_heston_option(ctypes.Structure):
    """Mirror of ``fe_heston_option`` (include/fe.h)."""

    _fields_ = [("nx", _c.c_int), ("ny", _c.c_int), ("strike", _c.c_float), ("maturity", _c.c_float),
                ("spot", _c.c_float), ("v0", _c.c_float), ("kappa", _c.c_float), ("theta", _c.c_float),
                ("sigma", _c.c_float), ("rho", _c.c_float), ("r", _c.c_float)]


class fe_group_totals(ctypes.Structure):
    """Mirror of ``fe_group_totals`` (include/fe.h)."""

    _fields_ = [("step", _c.c_longlong), ("term", _c.c_int), ("group", _c.c_int), ("substeps", _c.c_int), ("reserved", _c.c_int),
                ("before", _c.c_double), ("after", _c.c_double), ("scale", _c.c_double)]


class fe_step_info(ctypes.Structure):
    _fields_ = [("violations", _c.c_int), ("launches", _c.c_int), ("gpu_ms", _c.c_double), ("fallbacks", _c.c_int)]


class fe_field_info(ctypes.Structure):
    _fields_ = [("init", _c.c_double), ("lo", _c.c_double), ("hi", _c.c_double), ("is_static", _c.c_int),
                ("derived", _c.c_int), ("clamp", _c.c_int)]


FE_RANGE, FE_NOT_FINITE, FE_CONSERVATION, FE_SUBSTEP_CAP = 0, 1, 2, 3
class fe_batch_desc(_c.Structure):
    _fields_ = [("nx", _c.c_int), ("ny", _c.c_int), ("nz", _c.c_int), ("h", _c.c_double)]


FE_STEP_IGNORE_MAX_DT = 1
FE_ADI_DOUGLAS, FE_ADI_HV = 0, 1

_p = _c.c_void_p
_s = _c.c_size_t
_i = _c.c_int
_d = _c.c_double
_cs = _c.c_char_p

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
    "fe_heat7_step_noalloc": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_int, _c.c_int, _c.c_int, _c.c_float, _c.c_float,
                                         _c.c_float, _c.c_float, _c.c_float, _c.c_int, _c.c_int, _c.c_int, _c.c_void_p,
                                         _c.c_void_p]),
    "fe_law_create": (_i, [_cs, _cs, _i, _i, _i, _d, _c.POINTER(_p)]),
    "fe_law_destroy": (None, [_p]),
    "fe_law_create_ir": (_i, [_cs, _i, _i, _i, _d, _c.POINTER(_p)]),
    "fe_law_ir_check": (_i, [_cs, _p, _s, _c.POINTER(_s)]),
    "fe_law_source_ir": (_i, [_cs, _i, _i, _i, _d, _p, _s, _c.POINTER(_s)]),
    "fe_law_shift": (_i, [_p, _i, _i, _i]),
    "fe_law_upload_box": (_i, [_p, _i, _p, _i, _i, _i, _i, _i, _i]),
    "fe_law_upload_planes": (_i, [_p, _i, _p, _p]),
    "fe_law_ir_json": (_i, [_cs, _p, _s, _c.POINTER(_s)]),
    "fe_law_ir_listing": (_i, [_cs, _p, _s, _c.POINTER(_s)]),
    "fe_law_adjoint": (_i, [_cs, _cs, _p, _s, _c.POINTER(_s)]),
    "fe_law_source": (_i, [_cs, _i, _i, _i, _d, _p, _s, _c.POINTER(_s)]),
    "fe_law_compile_check": (_i, [_cs, _i, _i, _i, _d]),
    "fe_law_field_count": (_i, [_p]),
    "fe_law_field_id": (_i, [_p, _cs]),
    "fe_law_field_name": (_i, [_p, _i, _p, _s]),
    "fe_law_field_info": (_i, [_p, _i, _c.POINTER(fe_field_info)]),
    "fe_law_term_count": (_i, [_p]),
    "fe_law_term_name": (_i, [_p, _i, _p, _s]),
    "fe_law_param_count": (_i, [_p]),
    "fe_law_param_id": (_i, [_p, _cs]),
    "fe_law_set_param": (_i, [_p, _i, _d]),
    "fe_law_get_param": (_i, [_p, _i, _c.POINTER(_d)]),
    "fe_law_upload": (_i, [_p, _i, _p]),
    "fe_law_upload_device": (_i, [_p, _i, _p]),
    "fe_law_fetch": (_i, [_p, _i, _p]),
    "fe_law_fetch_device": (_i, [_p, _i, _p]),
    "fe_law_field_device_ptr": (_i, [_p, _i, _c.POINTER(_p)]),
    "fe_law_mark_edited": (_i, [_p, _i]),
    "fe_law_set_owned_z": (_i, [_p, _i, _i]),
    "fe_law_set_learned": (_i, [_p, _i]),
    "fe_law_term_learned": (_i, [_p, _i]),
    "fe_law_mark_halo": (_i, [_p, _i]),
    "fe_law_set_external_conservation": (_i, [_p, _i]),
    "fe_law_take_totals": (_i, [_p, _c.POINTER(fe_group_totals), _i, _c.POINTER(_i)]),
    "fe_law_plan_z_reach": (_i, [_c.c_char_p, _i, _i, _i, _c.c_double, _c.POINTER(_i), _c.POINTER(_i)]),
    "fe_law_step": (_i, [_p, _d, _i, _c.POINTER(fe_step_info)]),
    "fe_law_derive": (_i, [_p]),
    "fe_law_check_every": (_i, [_p, _i]),
    "fe_law_set_deferred": (_i, [_p, _i]),
    "fe_law_sync": (_i, [_p, _c.POINTER(fe_step_info)]),
    "fe_law_violation": (_i, [_p, _i, _c.POINTER(fe_violation)]),
    "fe_law_substeps": (_i, [_p, _i]),
    "fe_law_term_idle": (_i, [_p, _i]),
    "fe_law_digest": (_i, [_p, _c.POINTER(_c.c_uint64)]),
    "fe_law_stream": (_i, [_p, _c.POINTER(_p)]),
    "fe_law_time_gather": (_i, [_p, _i, _i, _c.POINTER(_c.c_float)]),
    "fe_law_time_stage": (_i, [_p, _i, _i, _i, _d, _c.POINTER(_c.c_float), _p, _s]),
    "fe_batch_create": (_i, [_cs, _c.POINTER(fe_batch_desc), _i, _c.POINTER(_p)]),
    "fe_batch_destroy": (None, [_p]),
    "fe_batch_plan": (_i, [_cs, _c.POINTER(fe_batch_desc), _i, _c.POINTER(_i), _c.POINTER(_i), _p, _p]),
    "fe_batch_info": (_i, [_p, _c.POINTER(_i), _c.POINTER(_i)]),
    "fe_batch_law": (_i, [_p, _i, _c.POINTER(_p), _c.POINTER(_i)]),
    "fe_batch_set_param": (_i, [_p, _i, _d]),
    "fe_batch_upload": (_i, [_p, _i, _i, _p]),
    "fe_batch_fetch": (_i, [_p, _i, _i, _p]),
    "fe_batch_step": (_i, [_p, _d, _i, _c.POINTER(_i)]),
    "fe_batch_violation": (_i, [_p, _i, _c.POINTER(_i), _c.POINTER(fe_violation)]),
    "fe_vjp_create": (_i, [_cs, _cs, _i, _i, _i, _d, _c.POINTER(_p)]),
    "fe_vjp_destroy": (None, [_p]),
    "fe_vjp_laws": (_i, [_p, _c.POINTER(_p), _c.POINTER(_p)]),
    "fe_vjp_set_param": (_i, [_p, _cs, _d]),
    "fe_vjp_forward": (_i, [_p, _d, _i, _i]),
    "fe_vjp_backward": (_i, [_p]),
    "fe_vjp_param_grad": (_i, [_p, _cs, _c.POINTER(_d)]),
    "fe_heston_batch_create": (_i, [_c.POINTER(fe_heston_option), _i, _i, _i, _c.POINTER(_p)]),
    "fe_heston_batch_destroy": (None, [_p]),
    "fe_heston_batch_set_split": (_i, [_p, _i, _i, _i]),
    "fe_heston_batch_autotune": (_i, [_p, _c.POINTER(_i), _c.POINTER(_i), _c.POINTER(_i)]),
    "fe_heston_batch_layout": (_i, [_p, _c.POINTER(_i), _c.POINTER(_i)]),
    "fe_heston_batch_run": (_i, [_p, _i]),
    "fe_heston_batch_time": (_i, [_p, _i, _c.POINTER(_c.c_float)]),
    "fe_heston_batch_prices": (_i, [_p, _p]),
    "fe_heston_batch_grid": (_i, [_p, _i, _p]),
    "fe_corr_create": (_i, [_c.POINTER(_p)]),
    "fe_corr_destroy": (None, [_p]),
    "fe_corr_weight_count": (_i, []),
    "fe_corr_set_weights": (_i, [_p, _p]),
    "fe_corr_get_weights": (_i, [_p, _p]),
    "fe_corr_grads": (_i, [_p, _p, _p, _p, _p, _i, _i, _i, _c.c_float, _p, _c.POINTER(_d), _p]),
    "fe_corr_train_step": (_i, [_p, _p, _p, _p, _p, _i, _i, _i, _c.c_float, _p, _c.c_float, _c.POINTER(_d)]),
    "fe_corr_apply": (_i, [_p, _p, _p, _i, _i, _i, _c.c_float, _c.c_float, _c.c_float, _p, _c.POINTER(_i)]),
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


def text_call(name, *args):
    """Calls a text-returning fe_* function (buf, cap, needed at the end) and returns the text."""
    needed = ctypes.c_size_t(0)
    check(getattr(lib(), name)(*args, None, 0, ctypes.byref(needed)))
    buf = ctypes.create_string_buffer(needed.value)
    check(getattr(lib(), name)(*args, buf, needed.value, ctypes.byref(needed)))
    return buf.value.decode()
