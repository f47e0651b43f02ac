// Backmap V = T Y + shift (reduced -> original flux space), the reference's
// backmap_into (src/gpu/backmap.cu:20-48 of quothbonney/naja: cublasDgemm
// followed by add_shift_cols_kernel) as one kernel with the shift fused into
// the epilogue.
//
// Layouts: T is n x d column-major (leading dimension ldt).  Y holds N
// samples as rows of d values (the sampler's output, row = sample), V
// receives N rows of n values -- the `samples.npy` layout of the
// back-transformed file.  In GEMM terms V (N x n) = Y (N x d) T^T (d x n).
//
// Modes (NAJA_BACKMAP_*):
//   FP64    SIMT FP64 tiles (the reference's arithmetic, different
//           summation order than cuBLAS).
//   BF16X3  / TF32X3: split-precision tensor-core products on tcgen05,
//           in backmap_tc.cu.
#include <cuda_runtime.h>

#include <string>

#include "../../include/naja_chr.h"
#include "capi_internal.cuh"

namespace naja {

namespace {

constexpr int kBM = 64;  // samples per CTA tile
constexpr int kBN = 64;  // outputs (rows of T) per CTA tile
constexpr int kBK = 16;

template <class YT, class VT>
__global__ void __launch_bounds__(256) backmap_fp64_kernel(int n, int d, long long N, const double* __restrict__ T,
                                                           int ldt, const double* __restrict__ shift,
                                                           const YT* __restrict__ Y, VT* __restrict__ V) {
  __shared__ double Ys[kBK][kBM + 1];
  __shared__ double Ts[kBK][kBN + 1];
  const long long s0 = static_cast<long long>(blockIdx.x) * kBM;
  const int i0 = blockIdx.y * kBN;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;  // 16 x 16 threads, 4 x 4 outputs each
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  for (int k0 = 0; k0 < d; k0 += kBK) {
    for (int e = threadIdx.x; e < kBK * kBM; e += 256) {
      const int kk = e % kBK, ss = e / kBK;
      const long long s = s0 + ss;
      Ys[kk][ss] = (s < N && k0 + kk < d) ? static_cast<double>(Y[s * d + k0 + kk]) : 0.0;
    }
    for (int e = threadIdx.x; e < kBK * kBN; e += 256) {
      const int ii = e % kBN, kk = e / kBN;
      const int i = i0 + ii;
      Ts[kk][ii] = (i < n && k0 + kk < d) ? T[static_cast<long long>(k0 + kk) * ldt + i] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kBK; ++kk) {
      double yv[4], tv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) yv[a] = Ys[kk][ty * 4 + a];
#pragma unroll
      for (int b = 0; b < 4; ++b) tv[b] = Ts[kk][tx * 4 + b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = __fma_rn(yv[a], tv[b], acc[a][b]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const long long s = s0 + ty * 4 + a;
    if (s >= N) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int i = i0 + tx * 4 + b;
      if (i < n) V[s * n + i] = static_cast<VT>(acc[a][b] + shift[i]);
    }
  }
}

template <class YT, class VT>
int launch_fp64(int n, int d, long long N, const double* T, int ldt, const double* shift, const void* Y, void* V,
                cudaStream_t stream) {
  dim3 grid(static_cast<unsigned>((N + kBM - 1) / kBM), static_cast<unsigned>((n + kBN - 1) / kBN));
  backmap_fp64_kernel<YT, VT><<<grid, 256, 0, stream>>>(n, d, N, T, ldt, shift, static_cast<const YT*>(Y),
                                                        static_cast<VT*>(V));
  return cudaGetLastError() == cudaSuccess ? NAJA_OK : NAJA_ERR_CUDA;
}

}  // namespace

int backmap_fp64_enqueue(int n, int d, long long N, const double* T, int ldt, const double* shift, const void* Y,
                         int y_dtype, void* V, int v_dtype, cudaStream_t stream) {
  int st;
  if (y_dtype == NAJA_DTYPE_F32)
    st = v_dtype == NAJA_DTYPE_F32 ? launch_fp64<float, float>(n, d, N, T, ldt, shift, Y, V, stream)
                                   : launch_fp64<float, double>(n, d, N, T, ldt, shift, Y, V, stream);
  else
    st = v_dtype == NAJA_DTYPE_F32 ? launch_fp64<double, float>(n, d, N, T, ldt, shift, Y, V, stream)
                                   : launch_fp64<double, double>(n, d, N, T, ldt, shift, Y, V, stream);
  if (st) return fail(st, std::string("backmap: launch failed: ") + cudaGetErrorString(cudaGetLastError()));
  return NAJA_OK;
}

}  // namespace naja

using namespace naja;

extern "C" int naja_backmap(int n, int d, long long N, const double* T, int ldt, const double* shift, const void* Y,
                            int y_dtype, void* V, int v_dtype, int mode, void* stream_ptr) {
  if (n <= 0 || d <= 0 || N < 0) return fail(NAJA_ERR_INVALID_ARGUMENT, "backmap_into: bad shape");
  if (!T || !shift || !Y || !V) return fail(NAJA_ERR_INVALID_ARGUMENT, "backmap_into: null argument");
  if (ldt < n) return fail(NAJA_ERR_INVALID_ARGUMENT, "backmap_into: transformation shape mismatch with samples");
  if ((y_dtype != NAJA_DTYPE_F32 && y_dtype != NAJA_DTYPE_F64) || (v_dtype != NAJA_DTYPE_F32 && v_dtype != NAJA_DTYPE_F64))
    return fail(NAJA_ERR_INVALID_ARGUMENT, "backmap_into: unknown dtype");
  if (int st = require_local("backmap_into", {T, shift, Y, V})) return st;
  if (N == 0) return NAJA_OK;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  const size_t ybytes = static_cast<size_t>(N) * d * (y_dtype == NAJA_DTYPE_F64 ? 8 : 4);
  const size_t vbytes = static_cast<size_t>(N) * n * (v_dtype == NAJA_DTYPE_F64 ? 8 : 4);
  DeviceBuffer bT, bs, bY, bV;
  const void *dT = nullptr, *dS = nullptr, *dY = nullptr;
  int st;
  if ((st = device_view(T, static_cast<size_t>(ldt) * (d - 1) * 8 + static_cast<size_t>(n) * 8, stream, bT, &dT)))
    return st;
  if ((st = device_view(shift, static_cast<size_t>(n) * 8, stream, bs, &dS))) return st;
  if ((st = device_view(Y, ybytes, stream, bY, &dY))) return st;
  void* dV = V;
  const bool host_v = !is_device_ptr(V);
  if (host_v) {
    if ((st = bV.alloc(vbytes, stream))) return st;
    dV = bV.ptr;
  }
  const double* Td = static_cast<const double*>(dT);
  const double* Sd = static_cast<const double*>(dS);
  if (mode == NAJA_BACKMAP_FP64) {
    if ((st = backmap_fp64_enqueue(n, d, N, Td, ldt, Sd, dY, y_dtype, dV, v_dtype, stream))) return st;
  } else if (mode == NAJA_BACKMAP_BF16X3 || mode == NAJA_BACKMAP_TF32X3) {
    st = backmap_tc(n, d, N, Td, ldt, Sd, dY, y_dtype, dV, v_dtype, mode, stream);
    if (st) return st;
  } else {
    return fail(NAJA_ERR_INVALID_ARGUMENT, "backmap: unknown mode");
  }
  cudaError_t e = cudaSuccess;
  if (host_v) e = cudaMemcpyAsync(V, dV, vbytes, cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess && (host_v || bT.ptr || bs.ptr || bY.ptr)) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("backmap: ") + cudaGetErrorString(e));
  return NAJA_OK;
}

extern "C" int naja_backmap_noalloc(int n, int d, long long N, const double* T, int ldt, const double* shift,
                                    const void* Y, int y_dtype, void* V, int v_dtype, int mode, void* stream_ptr) {
  if (n <= 0 || d <= 0 || N < 0) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_backmap_noalloc: bad shape");
  if (!T || !shift || !Y || !V) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_backmap_noalloc: null argument");
  if (ldt < n) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_backmap_noalloc: ldt < n");
  if ((y_dtype != NAJA_DTYPE_F32 && y_dtype != NAJA_DTYPE_F64) || (v_dtype != NAJA_DTYPE_F32 && v_dtype != NAJA_DTYPE_F64))
    return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_backmap_noalloc: unknown dtype");
  if (mode != NAJA_BACKMAP_BF16X3 && mode != NAJA_BACKMAP_TF32X3)
    return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_backmap_noalloc: mode must be NAJA_BACKMAP_BF16X3 or NAJA_BACKMAP_TF32X3");
  // Host buffers would need staging copies, i.e. allocations: every buffer must be device memory.
  if (!is_device_ptr(T) || !is_device_ptr(shift) || !is_device_ptr(Y) || !is_device_ptr(V))
    return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_backmap_noalloc: T, shift, Y and V must be device memory");
  if (int st = require_local("naja_backmap_noalloc", {T, shift, Y, V})) return st;
  if (N == 0) return NAJA_OK;
  return backmap_tc_noalloc(n, d, N, T, ldt, shift, Y, y_dtype, V, v_dtype, mode, static_cast<cudaStream_t>(stream_ptr));
}
