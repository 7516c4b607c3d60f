"""Python calls of the hand-written kernels (the bit-identity witness and the copy roof) on torch CUDA tensors.

torch is only the allocator and the stream here; the work is the library's (include/fe.h)."""
import ctypes

from . import _lib


def _stream(stream):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def heat7_workspace(shape, variant=0, zchunk=64, device="cuda"):
    """A workspace tensor (bytes) for fe_heat7_step with contracts."""
    import torch
    nz, ny, nx = shape
    n = _lib.lib().fe_heat7_workspace_bytes(nx, ny, nz, variant, zchunk)
    if n == 0:
        raise _lib.FeError(_lib.FE_EINVAL, "bad heat7 shape")
    return torch.zeros(n, dtype=torch.uint8, device=device)


def heat7_step(T, out, k, h, dt, lo=-1e30, hi=1e30, variant=0, zchunk=64, check=0, workspace=None, stream=None):
    """out <- one 7-point heat step of T (both (nz, ny, nx) float32 CUDA tensors)."""
    nz, ny, nx = T.shape
    ws = ctypes.c_void_p(workspace.data_ptr()) if workspace is not None else None
    _lib.call("fe_heat7_step", ctypes.c_void_p(T.data_ptr()), ctypes.c_void_p(out.data_ptr()), nx, ny, nz, k, h, dt, lo,
              hi, variant, zchunk, check, ws, _stream(stream))


def check_reset(workspace, stream=None):
    _lib.call("fe_check_reset", ctypes.c_void_p(workspace.data_ptr()), _stream(stream))


def check_read(workspace, stream=None):
    rec = _lib.fe_check()
    _lib.call("fe_check_read", ctypes.c_void_p(workspace.data_ptr()), ctypes.byref(rec), _stream(stream))
    return rec


def copy_f32(src, dst, stream=None):
    _lib.call("fe_copy_f32", ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(dst.data_ptr()), src.numel(),
              _stream(stream))
