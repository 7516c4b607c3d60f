"""fe_heat7_step_noalloc: the heat step for callers that cannot allocate device memory (their memory belongs to another
allocator or a fixed pool, or they run inside a process that forbids new device allocations). Its contract scratch lives
in a fixed array inside the library instead of a caller-allocated workspace; everything else is the same step, so it
must give what fe_heat7_step gives. Collected last on purpose (the file name), so a failure here stops a run only after
every other test has run; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_matches_workspace_step_two_calls_in_a_row(cuda):
    import torch
    from fieldcuda import _lib, kernels
    lib = _lib.lib()
    shape = (24, 40, 64)  # (nz, ny, nx)
    nz, ny, nx = shape
    T0 = np.random.default_rng(11).uniform(0.0, 2.0, shape).astype(np.float32)
    k, h, dt, lo, hi = 0.8, 0.125, 0.001, 0.25, 1.75
    check = _lib.FE_HEAT7_BEFORE | _lib.FE_HEAT7_AFTER
    stream = torch.cuda.current_stream()
    s = ctypes.c_void_p(stream.cuda_stream)
    for variant, zchunk in ((0, 8), (-1, 6)):
        # The existing entry point, with a workspace.
        a = torch.from_numpy(T0).cuda()
        b = torch.empty_like(a)
        ws = kernels.heat7_workspace(shape, variant, zchunk)
        want = []
        for _ in range(2):
            kernels.check_reset(ws)
            kernels.heat7_step(a, b, k, h, dt, lo=lo, hi=hi, variant=variant, zchunk=zchunk, check=check, workspace=ws)
            want.append((b.clone(), kernels.check_read(ws)))
            a, b = b, a
        # The allocation-free one, twice in a row on the same buffers; its record is a device fe_check of the caller's.
        c = torch.from_numpy(T0).cuda()
        d = torch.empty_like(c)
        rec_dev = torch.zeros(ctypes.sizeof(_lib.fe_check), dtype=torch.uint8, device="cuda")
        for i in range(2):
            _lib.check(lib.fe_heat7_step_noalloc(_ptr(c), _ptr(d), nx, ny, nz, k, h, dt, lo, hi, variant, zchunk, check,
                                                 _ptr(rec_dev), s))
            torch.cuda.synchronize()
            got = _lib.fe_check.from_buffer_copy(bytes(rec_dev.cpu().numpy()))
            field, ref = want[i]
            assert torch.equal(d.view(torch.int32), field.view(torch.int32)), (variant, i)
            # Same per-block partials in the same order: the FP64 totals agree to the bit.
            assert (got.before, got.before_abs, got.after) == (ref.before, ref.before_abs, ref.after), (variant, i)
            assert (got.out_of_range, got.not_finite, got.first_bad) == (ref.out_of_range, ref.not_finite, ref.first_bad)
            assert (got.lo_inv, got.hi_key, got.changed) == (ref.lo_inv, ref.hi_key, ref.changed)
            assert got.pad[0] == 0  # no kernel error word
            c, d = d, c


def test_noalloc_without_contracts_matches_and_reports_into_its_record(cuda):
    """check == 0: the field must still equal fe_heat7_step's bit for bit. A TMA variant still takes a record, for the
    kernel's error word: the call clears whatever the record held before (here stale nonzero bytes) and a clean pass
    leaves it all zero. Without a record a TMA variant is refused; the plain kernel (no waits) runs without one."""
    import torch
    from fieldcuda import _lib, kernels
    lib = _lib.lib()
    shape = (20, 36, 128)  # (nz, ny, nx)
    nz, ny, nx = shape
    T0 = np.random.default_rng(12).uniform(-1.0, 3.0, shape).astype(np.float32)
    k, h, dt = 1.3, 0.25, 0.004
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for variant, zchunk in ((1, 5), (0, 8), (-1, 7)):
        a = torch.from_numpy(T0).cuda()
        b = torch.empty_like(a)
        ws = kernels.heat7_workspace(shape, variant, zchunk)
        want = []
        for _ in range(2):
            kernels.check_reset(ws)
            kernels.heat7_step(a, b, k, h, dt, variant=variant, zchunk=zchunk, check=0, workspace=ws)
            want.append(b.clone())
            a, b = b, a
        c = torch.from_numpy(T0).cuda()
        d = torch.empty_like(c)
        rec_dev = torch.full((ctypes.sizeof(_lib.fe_check),), 0xA5, dtype=torch.uint8, device="cuda")
        for i in range(2):
            _lib.check(lib.fe_heat7_step_noalloc(_ptr(c), _ptr(d), nx, ny, nz, k, h, dt, -1e30, 1e30, variant, zchunk,
                                                 0, _ptr(rec_dev), s))
            torch.cuda.synchronize()
            assert torch.equal(d.view(torch.int32), want[i].view(torch.int32)), (variant, i)
            assert int(rec_dev.count_nonzero()) == 0, (variant, i)  # cleared, and no error word
            rec_dev.fill_(0x5A)
            c, d = d, c
        if variant >= 0:
            status = lib.fe_heat7_step_noalloc(_ptr(c), _ptr(d), nx, ny, nz, k, h, dt, -1e30, 1e30, variant, zchunk, 0,
                                               None, s)
            assert status == _lib.FE_EINVAL and "record" in _lib.last_error()
        else:
            # A third step from the second's result, without a record, against the workspace form of that step.
            third = torch.empty_like(c)
            kernels.heat7_step(c, third, k, h, dt, variant=variant, zchunk=zchunk, check=0, workspace=None)
            _lib.check(lib.fe_heat7_step_noalloc(_ptr(c), _ptr(d), nx, ny, nz, k, h, dt, -1e30, 1e30, variant, zchunk,
                                                 0, None, s))
            torch.cuda.synchronize()
            assert torch.equal(d.view(torch.int32), third.view(torch.int32))


def test_noalloc_refuses_sizes_beyond_its_scratch(cuda):
    import torch
    from fieldcuda import _lib
    lib = _lib.lib()
    # 4096 x 256 x 17 with one plane a CTA: 32 x 16 x 17 = 8704 thread blocks, more than the fixed scratch holds.
    nx, ny, nz = 4096, 256, 17
    a = torch.zeros((nz, ny, nx), dtype=torch.float32, device="cuda")
    b = torch.empty_like(a)
    rec = torch.zeros(ctypes.sizeof(_lib.fe_check), dtype=torch.uint8, device="cuda")
    status = lib.fe_heat7_step_noalloc(_ptr(a), _ptr(b), nx, ny, nz, 1.0, 1.0, 0.1, -1e30, 1e30, 0, 1, 3, _ptr(rec),
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert status == _lib.FE_EINVAL
    assert "8192" in _lib.last_error()
