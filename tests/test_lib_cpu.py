"""The C ABI library loads without a GPU and exports exactly what include/fe.h declares."""
import os
import re

from conftest import ROOT


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "fe.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(fe_[a-z0-9_]+)\s*\(", text))


def test_library_loads_and_exports_every_declared_symbol():
    from fieldcuda import _lib
    lib = _lib.lib()
    declared = declared_symbols()
    assert declared, "no declarations found in include/fe.h"
    missing = [s for s in sorted(declared) if not hasattr(lib, s)]
    assert not missing, f"declared but not exported: {missing}"
    assert declared == set(_lib.SIGNATURES), (
        f"binding table differs from the header: only in header {sorted(declared - set(_lib.SIGNATURES))}, "
        f"only in binding {sorted(set(_lib.SIGNATURES) - declared)}")


def test_version_and_no_device_status():
    from fieldcuda import _lib
    lib = _lib.lib()
    assert lib.fe_version() >= 1000
    status = lib.fe_device_check()
    if status != _lib.FE_OK:
        assert status == _lib.FE_ENODEV
        assert _lib.last_error()


def test_key_to_float_roundtrip():
    import numpy as np
    from fieldcuda import _lib
    lib = _lib.lib()
    for v in (-3.5, -0.0, 0.0, 1e-30, 7.25, 1e30):
        b = np.array([v], dtype=np.float32).view(np.uint32)[0]
        key = (~b & 0xFFFFFFFF) if (b & 0x80000000) else (b | 0x80000000)
        assert np.float32(lib.fe_key_to_float(int(key))) == np.float32(v)


def test_heston_batch_rejects_bad_options_before_touching_a_device():
    import ctypes
    from fieldcuda import _lib
    from fieldcuda.heston import option_array, sample_options
    lib = _lib.lib()
    good = sample_options(3, 1)
    for bad in (dict(nx=96), dict(ny=512), dict(strike=-1.0), dict(sigma=0.0), dict(maturity=0.0), dict(spot=0.0)):
        opts = [dict(good[0]), dict(good[1], **bad), dict(good[2])]
        h = ctypes.c_void_p()
        assert lib.fe_heston_batch_create(option_array(opts), 3, 8, 0, ctypes.byref(h)) == _lib.FE_EINVAL
        assert "option 1" in _lib.last_error()
        assert not h.value
    h = ctypes.c_void_p()
    assert lib.fe_heston_batch_create(option_array(good), 3, 8, 2, ctypes.byref(h)) == _lib.FE_EINVAL
    status = lib.fe_heston_batch_create(option_array(good), 3, 8, 0, ctypes.byref(h))
    if status == _lib.FE_OK:
        lib.fe_heston_batch_destroy(h)
    else:
        assert status == _lib.FE_ENODEV
