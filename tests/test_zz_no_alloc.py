"""naja_backmap_noalloc: the tensor-core backmap without device allocations (GPU).

Callers that must not allocate device memory where they call the backmap
(a service that reserves its device memory up front and forbids allocations
on its request path, or a framework whose allocator owns the device) use
this entry point; its split operands live in a fixed 64 MiB array inside the
library.  The test calls it through the C ABI twice in a row with different
inputs (the array is reused, so the second call must not see the first
call's data) and compares each result with the allocating entry point,
naja_backmap, in the same mode, within the backmap tests' tolerance
(2^-15 of |T||y| + |shift| for BF16X3, 2^-17 for TF32X3).  It runs alone in
a fresh process as well as after the other tests.
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
