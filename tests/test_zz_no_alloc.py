"""naja_backmap_noalloc: the tensor-core backmap without device allocations (GPU).

Callers that must not allocate device memory where they call the backmap
(a service that reserves its device memory up front and forbids allocations
on its request path, or a framework whose allocator owns the device) use
this entry point; its split operands live in a fixed 64 MiB array inside the
library.  The test calls it through the C ABI twice in a row with different
inputs (the array is reused, so the second call must not see the first
call's data) and compares each result with the allocating entry point,
naja_backmap, in the same mode, within the backmap tests' tolerance
(2^-15 of |T||y| + |shift| for BF16X3, 2^-17 for TF32X3), and checks around
warm calls that no device memory is taken: free device memory, torch's
allocator and the default stream-ordered pool stay as they were.  It runs
alone in a fresh process as well as after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"bf16x3": 2.0 ** -15, "tf32x3": 2.0 ** -17}
MODE = {"bf16x3": 1, "tf32x3": 2}


def _inputs(seed, N, n, d):
    import torch

    rng = np.random.default_rng(seed)
    T = np.where(rng.random((n, d)) < 0.3, rng.standard_normal((n, d)), 0.0)
    Y = (rng.standard_normal((N, d)) * 10 ** rng.uniform(-1, 1, (1, d))).astype(np.float32)
    shift = rng.standard_normal(n)
    dev = torch.device("cuda", 0)
    Tc = torch.from_numpy(np.asfortranarray(T).T.copy()).to(dev)  # column-major n x d == row-major d x n
    return (T, Y, shift, Tc, torch.from_numpy(Y).to(dev), torch.from_numpy(shift).to(dev))


@pytest.mark.parametrize("mode", ["bf16x3", "tf32x3"])
def test_noalloc_matches_allocating_backmap(cuda, mode):
    import torch

    from naja_b200 import _lib

    lib = _lib.load()
    N, n, d = 3000, 700, 130
    for seed in (11, 12):  # two calls in a row on the shared scratch
        T, Y, shift, Tc, Yd, sd = _inputs(seed, N, n, d)
        out_na = torch.full((N, n), float("nan"), dtype=torch.float32, device=cuda)
        out_ref = torch.empty((N, n), dtype=torch.float32, device=cuda)
        stream = C.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
        st = lib.naja_backmap_noalloc(n, d, N, C.c_void_p(Tc.data_ptr()), n, C.c_void_p(sd.data_ptr()),
                                      C.c_void_p(Yd.data_ptr()), _lib.DTYPE_F32, C.c_void_p(out_na.data_ptr()),
                                      _lib.DTYPE_F32, MODE[mode], stream)
        _lib.check(st)
        st = lib.naja_backmap(n, d, N, C.c_void_p(Tc.data_ptr()), n, C.c_void_p(sd.data_ptr()),
                              C.c_void_p(Yd.data_ptr()), _lib.DTYPE_F32, C.c_void_p(out_ref.data_ptr()),
                              _lib.DTYPE_F32, MODE[mode], stream)
        _lib.check(st)
        torch.cuda.synchronize()
        got, ref = out_na.cpu().numpy().astype(np.float64), out_ref.cpu().numpy().astype(np.float64)
        scale = np.abs(Y.astype(np.float64)) @ np.abs(T).T + np.abs(shift)
        assert np.isfinite(got).all()
        assert np.max(np.abs(got - ref) / scale) <= TOL[mode]
        exact = Y.astype(np.float64) @ T.T + shift
        assert np.max(np.abs(got - exact) / scale) <= TOL[mode]


def test_noalloc_rejects_oversized_and_host_buffers(cuda):
    import torch

    from naja_b200 import _lib

    lib = _lib.load()
    n, d = 64, 700
    T, Y, shift, Tc, Yd, sd = _inputs(3, 8, n, d)
    stream = C.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    big_N = 100000  # 2 * 100000 * 704 * 4 bytes of split operands > 64 MiB
    out = torch.empty((8, n), dtype=torch.float32, device=cuda)
    st = lib.naja_backmap_noalloc(n, d, big_N, C.c_void_p(Tc.data_ptr()), n, C.c_void_p(sd.data_ptr()),
                                  C.c_void_p(Yd.data_ptr()), _lib.DTYPE_F32, C.c_void_p(out.data_ptr()),
                                  _lib.DTYPE_F32, MODE["tf32x3"], stream)
    assert st == _lib.NAJA_ERR_INVALID_ARGUMENT
    assert b"scratch" in lib.naja_last_error()
    host_out = np.empty((8, n), dtype=np.float32)
    st = lib.naja_backmap_noalloc(n, d, 8, C.c_void_p(Tc.data_ptr()), n, C.c_void_p(sd.data_ptr()),
                                  C.c_void_p(Yd.data_ptr()), _lib.DTYPE_F32, C.c_void_p(host_out.ctypes.data),
                                  _lib.DTYPE_F32, MODE["tf32x3"], stream)
    assert st == _lib.NAJA_ERR_INVALID_ARGUMENT


def _pool_usage(dev_index):
    """(used, reserved) bytes of the device's default memory pool (the pool
    cudaMallocAsync draws from), read through the driver API."""
    cu = C.CDLL("libcuda.so.1")
    dev = C.c_int()
    assert cu.cuDeviceGet(C.byref(dev), dev_index) == 0
    pool = C.c_void_p()
    assert cu.cuDeviceGetDefaultMemPool(C.byref(pool), dev) == 0
    used, reserved = C.c_uint64(), C.c_uint64()
    assert cu.cuMemPoolGetAttribute(pool, 7, C.byref(used)) == 0  # CU_MEMPOOL_ATTR_USED_MEM_CURRENT
    assert cu.cuMemPoolGetAttribute(pool, 5, C.byref(reserved)) == 0  # CU_MEMPOOL_ATTR_RESERVED_MEM_CURRENT
    return used.value, reserved.value


def test_noalloc_allocates_no_device_memory(cuda):
    """Around a warm call: the device's free memory, torch's allocator and the
    default stream-ordered pool are unchanged, while the allocating entry
    point in the same place draws from that pool."""
    import torch

    from naja_b200 import _lib

    lib = _lib.load()
    N, n, d = 2000, 500, 100
    T, Y, shift, Tc, Yd, sd = _inputs(5, N, n, d)
    out = torch.empty((N, n), dtype=torch.float32, device=cuda)
    stream = C.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    args = (n, d, N, C.c_void_p(Tc.data_ptr()), n, C.c_void_p(sd.data_ptr()), C.c_void_p(Yd.data_ptr()),
            _lib.DTYPE_F32, C.c_void_p(out.data_ptr()), _lib.DTYPE_F32, MODE["bf16x3"], stream)
    _lib.check(lib.naja_backmap_noalloc(*args))  # warm: set-up done, kernels loaded
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(cuda)[0]
    torch0 = (torch.cuda.memory_allocated(cuda), torch.cuda.memory_reserved(cuda))
    pool0 = _pool_usage(cuda.index or 0)
    for _ in range(3):
        _lib.check(lib.naja_backmap_noalloc(*args))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(cuda)[0] == free0
    assert (torch.cuda.memory_allocated(cuda), torch.cuda.memory_reserved(cuda)) == torch0
    assert _pool_usage(cuda.index or 0) == pool0
    # the allocating entry point does draw its split operands from the pool
    # (its high-water mark must exceed them; current usage returns after the call)
    cu = C.CDLL("libcuda.so.1")
    dev = C.c_int()
    cu.cuDeviceGet(C.byref(dev), cuda.index or 0)
    pool = C.c_void_p()
    cu.cuDeviceGetDefaultMemPool(C.byref(pool), dev)
    zero = C.c_uint64(0)
    assert cu.cuMemPoolSetAttribute(pool, 8, C.byref(zero)) == 0  # reset CU_MEMPOOL_ATTR_USED_MEM_HIGH
    _lib.check(lib.naja_backmap(*args))
    torch.cuda.synchronize()
    high = C.c_uint64()
    assert cu.cuMemPoolGetAttribute(pool, 8, C.byref(high)) == 0
    assert high.value >= 2 * N * 128 * 2  # two BF16 halves of the samples, d padded to 128
