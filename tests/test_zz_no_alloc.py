"""The allocation-free TV-gradient entry point, for callers that may not let
a library allocate device memory (a service that reserves its whole budget up
front, a host application whose allocator owns the device memory).

It is called through the C ABI on several calls in a row and must equal the
allocating entry point (ct2_dev_totalvar_total_var_grad3d) bit for bit each
time: both run the same kernels with the same fixed reduction order.  The
calls share one scratch array, so the sequence includes a call that needs
more reduction blocks than the one before it (stale sums from the earlier
call lie in the range the later one reads, unless every block writes its own
entry first) and the same input twice.  It also checks the property the
entry point exists for: a call moves neither the device's stream-ordered
memory pool (used or reserved bytes, high-water mark included) nor the free
device memory.  This file is collected last, so a run stopping at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# cudaMemPoolAttr values (cuda_runtime_api / driver_types.h)
RESERVED_CURRENT, RESERVED_HIGH, USED_CURRENT, USED_HIGH = 0x5, 0x6, 0x7, 0x8


def _run(fn, lam, x, normalizeq, torch):
    nx, ny, nz = x.shape
    out = torch.empty_like(x)
    bobo = torch.empty(1, dtype=torch.float32, device=x.device)
    stream = ctypes.c_void_p(torch.cuda.current_stream(x.device).cuda_stream)
    rc = fn(ctypes.c_float(lam), ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(x.data_ptr()),
            nx, ny, nz, normalizeq, ctypes.c_void_p(bobo.data_ptr()), stream)
    return rc, out, bobo


class _Pool:
    """The current device's default stream-ordered memory pool, read through
    the CUDA runtime the library links."""

    def __init__(self, torch):
        self.rt = ctypes.CDLL("libcudart.so.12")
        self.pool = ctypes.c_void_p()
        dev = torch.cuda.current_device()
        assert self.rt.cudaDeviceGetDefaultMemPool(ctypes.byref(self.pool), dev) == 0

    def get(self, attr):
        v = ctypes.c_uint64()
        assert self.rt.cudaMemPoolGetAttribute(self.pool, attr, ctypes.byref(v)) == 0
        return v.value

    def reset_high(self):
        zero = ctypes.c_uint64(0)
        for attr in (RESERVED_HIGH, USED_HIGH):
            assert self.rt.cudaMemPoolSetAttribute(self.pool, attr, ctypes.byref(zero)) == 0

    def free_bytes(self):
        free, total = ctypes.c_size_t(), ctypes.c_size_t()
        assert self.rt.cudaMemGetInfo(ctypes.byref(free), ctypes.byref(total)) == 0
        return free.value


def test_noalloc_tv_grad_matches_allocating_entry_point(cuda):
    import torch

    from ct2b200 import _lib
    L = _lib.lib()
    new = L.ct2_dev_totalvar_total_var_grad3d_noalloc
    ref = L.ct2_dev_totalvar_total_var_grad3d
    gen = torch.Generator(device="cpu").manual_seed(0)
    big = torch.rand((40, 36, 48), generator=gen)        # 270 reduction blocks
    small = torch.rand((33, 17, 29), generator=gen) * 3   # 64 blocks
    bigger = torch.rand((64, 60, 70), generator=gen)     # 1050 blocks (8 * 148 caps at 1184)
    cases = [(0.0, big, 1), (0.02, small, 0), (0.0, bigger, 1), (0.0, bigger, 1),
             (0.01, small, 1)]
    for lam, xc, normalizeq in cases:
        x = xc.to(cuda).contiguous()
        rc_n, out_n, b_n = _run(new, lam, x, normalizeq, torch)
        _lib.check(rc_n, "ct2_dev_totalvar_total_var_grad3d_noalloc")
        rc_r, out_r, b_r = _run(ref, lam, x, normalizeq, torch)
        _lib.check(rc_r, "ct2_dev_totalvar_total_var_grad3d")
        torch.cuda.synchronize()
        assert float(b_n.item()) == float(b_r.item())
        assert np.array_equal(out_n.cpu().numpy(), out_r.cpu().numpy())


def test_noalloc_tv_grad_allocates_nothing(cuda):
    import torch

    from ct2b200 import _lib
    fn = _lib.lib().ct2_dev_totalvar_total_var_grad3d_noalloc
    x = torch.rand((64, 60, 70), device=cuda)
    out = torch.empty_like(x)
    bobo = torch.empty(1, dtype=torch.float32, device=cuda)
    stream = ctypes.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)

    def call():
        rc = fn(ctypes.c_float(0.0), ctypes.c_void_p(out.data_ptr()),
                ctypes.c_void_p(x.data_ptr()), *x.shape, 1, ctypes.c_void_p(bobo.data_ptr()),
                stream)
        _lib.check(rc, "ct2_dev_totalvar_total_var_grad3d_noalloc")

    call()  # the first call on a device looks up the array's address
    torch.cuda.synchronize()
    pool = _Pool(torch)
    pool.reset_high()
    before = {a: pool.get(a) for a in (RESERVED_CURRENT, RESERVED_HIGH, USED_CURRENT, USED_HIGH)}
    free_before = pool.free_bytes()
    for _ in range(3):
        call()
    torch.cuda.synchronize()
    after = {a: pool.get(a) for a in before}
    assert after == before, (before, after)
    assert pool.free_bytes() == free_before


def test_noalloc_tv_grad_rejects_what_the_allocating_entry_point_rejects(cuda):
    import torch

    from ct2b200 import _lib
    L = _lib.lib()
    dummy = torch.empty(1, device=cuda)
    p = ctypes.c_void_p(dummy.data_ptr())
    s = ctypes.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    for dims in ((-1, 4, 4), (1 << 14, 1 << 14, 1 << 13)):  # negative; 2^41 voxels
        for fn in (L.ct2_dev_totalvar_total_var_grad3d_noalloc,
                   L.ct2_dev_totalvar_total_var_grad3d):
            assert fn(ctypes.c_float(0.0), p, p, *dims, 0, p, s) == _lib.CT2_EINVAL
