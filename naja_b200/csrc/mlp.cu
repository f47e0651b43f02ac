// Kernels of the learned-rounding network (see include/naja_mlp.h).
//
// GEMM: D (M x N) = A (M x K) B (N x K)^T with BF16 operands and an FP32
// accumulator in tensor memory, persistent over 128 x 128 output tiles
// (n fastest), one CTA per SM:
//   warp 4, one thread : TMA producer, 2-D tiled loads (128-byte swizzle) of
//                        a 128-row x 64-value K slice of A and of B per stage
//                        into a 4-stage shared-memory ring; loads past the
//                        matrix edges read zeros, so M, N and K need no padding.
//   warp 5, one thread : MMA issuer, 4 tcgen05.mma (K = 16 each) per stage;
//                        the stage is released with tcgen05.commit.
//   warps 0-3          : epilogue, tcgen05.ld of their 32 accumulator lanes
//                        (one output row per thread), bias, GELU, and the
//                        FP32 / BF16 / transposed-BF16 stores.
// Every wait is bounded by the global timer; on expiry the CTA records an
// error in a device word (read by naja_mlp_check), stops issuing, drains its
// own copies and MMAs and frees its tensor memory.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "../../include/naja_chr.h"
#include "../../include/naja_mlp.h"
#include "capi_internal.cuh"
#include "common.cuh"
#include "tc_common.cuh"

namespace naja {
namespace {

constexpr int kTileM = 128;
constexpr int kTileN = 128;
constexpr int kStages = 4;
constexpr int kThreads = 192;
constexpr uint32_t kTmemCols = 128;
constexpr uint64_t kTimeoutNs = 5ull * 1000 * 1000 * 1000;
constexpr uint32_t kATile = kTileM * 128;  // bytes of one 128-row x 128-byte slice
constexpr uint32_t kBTile = kTileN * 128;
constexpr uint32_t kStageBytes = kATile + kBTile;

enum GemmError : int { kGemmTimeoutLoad = 21, kGemmTimeoutSlot = 22, kGemmTimeoutAcc = 23, kGemmTimeoutEpi = 24 };

__device__ int g_gemm_err[4];

struct GemmArgs {
  int M, N, kslices, tiles_n;
  long long tiles;
  naja_gemm_epilogue epi;
};

__device__ __forceinline__ float gelu_f(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad_f(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * expf(-0.5f * x * x) * 0.39894228040143268f;
}

__global__ void __launch_bounds__(kThreads, 1)
    gemm_bf16_kernel(const __grid_constant__ CUtensorMap mA, const __grid_constant__ CUtensorMap mB,
                     const __grid_constant__ GemmArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* acc_full = empty + kStages;
  uint64_t* acc_empty = acc_full + 1;
  uint64_t* drain_bar = acc_empty + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain_bar + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  int* err = g_gemm_err;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, 4);
    mbar_init(drain_bar, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0) tc::tmem_alloc(tmem_slot, kTmemCols);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = *tmem_slot;
  const int K = a.kslices;

  if (warp == 4) {
    if (lane == 0) {
      int stage = 0;
      uint32_t round = 0, last_parity = 0, used = 0;
      for (long long tile = blockIdx.x; tile < a.tiles && !*abort_flag; tile += gridDim.x) {
        const int tm = static_cast<int>(tile / a.tiles_n), tn = static_cast<int>(tile % a.tiles_n);
        for (int ks = 0; ks < K; ++ks) {
          if (round >= 1 && !mbar_wait_bounded(&empty[stage], (round - 1) & 1u, kTimeoutNs)) {
            set_error(err, kGemmTimeoutSlot, static_cast<int>(blockIdx.x), stage, ks);
            *abort_flag = 1;
            break;
          }
          unsigned char* st = smem + stage * kStageBytes;
          mbar_arrive_expect_tx(&full[stage], kStageBytes);
          tc::tma_load_2d(st, &mA, ks * 64, tm * kTileM, &full[stage]);
          tc::tma_load_2d(st + kATile, &mB, ks * 64, tn * kTileN, &full[stage]);
          used |= 1u << stage;
          last_parity = (last_parity & ~(1u << stage)) | ((round & 1u) << stage);
          if (++stage == kStages) {
            stage = 0;
            ++round;
          }
        }
      }
      for (int s = 0; s < kStages; ++s)
        if (((used >> s) & 1u) && !mbar_wait_bounded(&full[s], (last_parity >> s) & 1u, kTimeoutNs))
          set_error(err, kGemmTimeoutLoad, static_cast<int>(blockIdx.x), s, -1);
    }
  } else if (warp == 5) {
    if (lane == 0) {
      constexpr uint32_t idesc = tc::idesc_bf16_f32(kTileM, kTileN);
      int stage = 0;
      uint32_t parity = 0, acc_round = 0;
      bool issued = false;
      for (long long tile = blockIdx.x; tile < a.tiles && !*abort_flag; tile += gridDim.x) {
        if (acc_round >= 1 && !mbar_wait_bounded(acc_empty, (acc_round - 1) & 1u, kTimeoutNs)) {
          set_error(err, kGemmTimeoutEpi, static_cast<int>(blockIdx.x), static_cast<int>(acc_round), -1);
          *abort_flag = 1;
          break;
        }
        tc::fence_after();
        bool ok = true;
        for (int ks = 0; ks < K; ++ks) {
          if (!mbar_wait_bounded(&full[stage], parity, kTimeoutNs)) {
            set_error(err, kGemmTimeoutLoad, static_cast<int>(blockIdx.x), stage, ks);
            *abort_flag = 1;
            ok = false;
            break;
          }
          tc::fence_after();
          const unsigned char* st = smem + stage * kStageBytes;
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            tc::mma_bf16(tmem, tc::desc_sw128(st + kk * 32), tc::desc_sw128(st + kATile + kk * 32), idesc,
                         (ks > 0 || kk > 0) ? 1u : 0u);
          }
          issued = true;
          tc::commit(&empty[stage]);
          if (++stage == kStages) {
            stage = 0;
            parity ^= 1u;
          }
        }
        if (!ok) break;
        tc::commit(acc_full);
        ++acc_round;
      }
      if (issued) {
        tc::commit(drain_bar);
        if (!mbar_wait_bounded(drain_bar, 0u, kTimeoutNs))
          set_error(err, kGemmTimeoutAcc, static_cast<int>(blockIdx.x), -1, -1);
      }
    }
  } else {
    const naja_gemm_epilogue& e = a.epi;
    uint32_t acc_round = 0;
    for (long long tile = blockIdx.x; tile < a.tiles; tile += gridDim.x) {
      const bool ok = mbar_wait_bounded(acc_full, acc_round & 1u, kTimeoutNs);
      if (!__all_sync(0xffffffffu, ok)) {
        if (lane == 0) set_error(err, kGemmTimeoutAcc, static_cast<int>(blockIdx.x), warp, static_cast<int>(acc_round));
        *abort_flag = 1;
        break;
      }
      tc::fence_after();
      const int tm = static_cast<int>(tile / a.tiles_n), tn = static_cast<int>(tile % a.tiles_n);
      const int row = tm * kTileM + warp * 32 + lane;
#pragma unroll 1
      for (int c = 0; c < kTileN; c += 32) {
        uint32_t r[32];
        tc::tmem_ld32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c), r);
        const int n0 = tn * kTileN + c;
        if (row < a.M) {
#pragma unroll
          for (int q = 0; q < 32; ++q) {
            const int n = n0 + q;
            if (n < a.N) {
              float v = __uint_as_float(r[q]);
              if (e.bias) v += e.bias[n];
              if (e.c_f32) {
                float* cp = e.c_f32 + static_cast<size_t>(row) * e.ldc + n;
                *cp = e.accumulate ? *cp + v : v;
              }
              const float g = e.gelu ? gelu_f(v) : v;
              if (e.act) reinterpret_cast<__nv_bfloat16*>(e.act)[static_cast<size_t>(row) * e.ld_act + n] = __float2bfloat16_rn(g);
              if (e.act_t)
                reinterpret_cast<__nv_bfloat16*>(e.act_t)[static_cast<size_t>(n) * e.ld_act_t + row] = __float2bfloat16_rn(g);
            }
          }
        }
      }
      tc::fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acc_empty);
      ++acc_round;
    }
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  if (warp == 0) tc::tmem_dealloc(tmem, kTmemCols);
}

// ------------------------------------------------------------ elementwise
__global__ void cast_bf16_kernel(int rows, int cols, const float* __restrict__ src, int ld_src,
                                 __nv_bfloat16* dst, int ld_dst, __nv_bfloat16* dst_t, int ld_dst_t) {
  const long long total = static_cast<long long>(rows) * cols;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(i / cols), c = static_cast<int>(i % cols);
    const __nv_bfloat16 v = __float2bfloat16_rn(src[static_cast<size_t>(r) * ld_src + c]);
    if (dst) dst[static_cast<size_t>(r) * ld_dst + c] = v;
    if (dst_t) dst_t[static_cast<size_t>(c) * ld_dst_t + r] = v;
  }
}

__global__ void gelu_backward_kernel(int rows, int cols, const float* __restrict__ dact, const float* __restrict__ pre,
                                     int ld, float* dpre, __nv_bfloat16* dpre_bf, int ld_bf, __nv_bfloat16* dpre_bf_t,
                                     int ld_bf_t) {
  const long long total = static_cast<long long>(rows) * cols;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(i / cols), c = static_cast<int>(i % cols);
    const size_t o = static_cast<size_t>(r) * ld + c;
    const float g = dact[o] * gelu_grad_f(pre[o]);
    if (dpre) dpre[o] = g;
    const __nv_bfloat16 b = __float2bfloat16_rn(g);
    if (dpre_bf) dpre_bf[static_cast<size_t>(r) * ld_bf + c] = b;
    if (dpre_bf_t) dpre_bf_t[static_cast<size_t>(c) * ld_bf_t + r] = b;
  }
}

__global__ void mse_grad_kernel(int rows, int cols, const float* __restrict__ out, const float* __restrict__ target,
                                int ld, const float* __restrict__ w, double* loss, float* grad, __nv_bfloat16* grad_bf,
                                int ld_bf, __nv_bfloat16* grad_bf_t, int ld_bf_t) {
  __shared__ double part[32];
  const long long total = static_cast<long long>(rows) * cols;
  double acc = 0.0;
  const float inv_rows = 1.0f / static_cast<float>(rows);
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(i / cols), c = static_cast<int>(i % cols);
    const size_t o = static_cast<size_t>(r) * ld + c;
    const float wc = w ? w[c] : 1.0f;
    const float diff = out[o] - target[o];
    acc += static_cast<double>(wc) * diff * diff;
    const float g = 2.0f * wc * diff * inv_rows;
    if (grad) grad[o] = g;
    const __nv_bfloat16 b = __float2bfloat16_rn(g);
    if (grad_bf) grad_bf[static_cast<size_t>(r) * ld_bf + c] = b;
    if (grad_bf_t) grad_bf_t[static_cast<size_t>(c) * ld_bf_t + r] = b;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < static_cast<int>(blockDim.x >> 5); ++k) s += part[k];
    atomicAdd(loss, s / rows);
  }
}

__global__ void col_sum_kernel(int rows, int cols, const float* __restrict__ d, int ld, float* db) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.0f;
  for (int r = 0; r < rows; ++r) s += d[static_cast<size_t>(r) * ld + c];
  db[c] = s;
}

__global__ void adam_kernel(int rows, int cols, float* W, const float* __restrict__ g, float* m, float* v, int ld,
                            float lr, float b1, float b2, float eps, float c1, float c2, __nv_bfloat16* w_bf, int ld_bf,
                            __nv_bfloat16* w_bf_t, int ld_bf_t) {
  const long long total = static_cast<long long>(rows) * cols;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(i / cols), c = static_cast<int>(i % cols);
    const size_t o = static_cast<size_t>(r) * ld + c;
    const float gi = g[o];
    const float mi = b1 * m[o] + (1.0f - b1) * gi;
    const float vi = b2 * v[o] + (1.0f - b2) * gi * gi;
    m[o] = mi;
    v[o] = vi;
    const float wi = W[o] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    W[o] = wi;
    const __nv_bfloat16 b = __float2bfloat16_rn(wi);
    if (w_bf) w_bf[static_cast<size_t>(r) * ld_bf + c] = b;
    if (w_bf_t) w_bf_t[static_cast<size_t>(c) * ld_bf_t + r] = b;
  }
}

int grid_for(long long total) {
  return static_cast<int>(std::min<long long>((total + 255) / 256, 148LL * 16));
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int launch_status(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return NAJA_OK;
}

}  // namespace
}  // namespace naja

using namespace naja;

extern "C" {

int naja_gemm_bf16(int M, int N, int K, const void* A, int lda, const void* B, int ldb,
                   const naja_gemm_epilogue* epi, void* stream) {
  if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !epi) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_gemm_bf16: bad arguments");
  if (lda < K || ldb < K || (lda % 8) || (ldb % 8) || !aligned16(A) || !aligned16(B))
    return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_gemm_bf16: BF16 rows must be 16-byte aligned with pitch >= K");
  if ((epi->c_f32 && epi->ldc < N) || (epi->act && epi->ld_act < N) || (epi->act_t && epi->ld_act_t < M))
    return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_gemm_bf16: epilogue pitch too small");
  if (int st = require_local("naja_gemm_bf16", {A, B, epi->bias, epi->c_f32, epi->act, epi->act_t})) return st;
  CUtensorMap mA, mB;
  if (!tc::make_map_bf16(&mA, A, M, K, lda, kTileM) || !tc::make_map_bf16(&mB, B, N, K, ldb, kTileN))
    return fail(NAJA_ERR_CUDA, "naja_gemm_bf16: cuTensorMapEncodeTiled failed");
  GemmArgs a;
  a.M = M;
  a.N = N;
  a.kslices = (K + 63) / 64;
  a.tiles_n = (N + kTileN - 1) / kTileN;
  a.tiles = static_cast<long long>((M + kTileM - 1) / kTileM) * a.tiles_n;
  a.epi = *epi;
  const size_t smem = kStages * kStageBytes + 1024 + 256;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = static_cast<int>(std::min<long long>(sms, a.tiles));
  cudaError_t e = cudaFuncSetAttribute(gemm_bf16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("naja_gemm_bf16: ") + cudaGetErrorString(e));
  gemm_bf16_kernel<<<grid, kThreads, smem, static_cast<cudaStream_t>(stream)>>>(mA, mB, a);
  return launch_status("naja_gemm_bf16");
}

int naja_mlp_check(void* stream) {
  int w[4] = {0, 0, 0, 0};
  cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
  if (e == cudaSuccess) e = cudaMemcpyFromSymbol(w, g_gemm_err, sizeof(w));
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("naja_mlp_check: ") + cudaGetErrorString(e));
  if (w[0] != 0) {
    const int z[4] = {0, 0, 0, 0};
    cudaMemcpyToSymbol(g_gemm_err, z, sizeof(z));
    return fail(NAJA_ERR_DEVICE, "naja_gemm_bf16: tensor-core pipeline gave up a bounded wait (code " +
                                     std::to_string(w[0]) + ", " + std::to_string(w[1]) + ", " + std::to_string(w[2]) +
                                     ", " + std::to_string(w[3]) + ")");
  }
  return NAJA_OK;
}

int naja_cast_bf16(int rows, int cols, const float* src, int ld_src, void* dst, int ld_dst, void* dst_t,
                   int ld_dst_t, void* stream) {
  if (rows <= 0 || cols <= 0 || !src || ld_src < cols || (dst && ld_dst < cols) || (dst_t && ld_dst_t < rows))
    return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_cast_bf16: bad arguments");
  if (int st = require_local("naja_cast_bf16", {src, dst, dst_t})) return st;
  const long long total = static_cast<long long>(rows) * cols;
  cast_bf16_kernel<<<grid_for(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      rows, cols, src, ld_src, static_cast<__nv_bfloat16*>(dst), ld_dst, static_cast<__nv_bfloat16*>(dst_t), ld_dst_t);
  return launch_status("naja_cast_bf16");
}

int naja_gelu_backward(int rows, int cols, const float* dact, const float* pre, int ld, float* dpre, void* dpre_bf,
                       int ld_bf, void* dpre_bf_t, int ld_bf_t, void* stream) {
  if (rows <= 0 || cols <= 0 || !dact || !pre || ld < cols || (dpre_bf && ld_bf < cols) || (dpre_bf_t && ld_bf_t < rows))
    return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_gelu_backward: bad arguments");
  if (int st = require_local("naja_gelu_backward", {dact, pre, dpre, dpre_bf, dpre_bf_t})) return st;
  const long long total = static_cast<long long>(rows) * cols;
  gelu_backward_kernel<<<grid_for(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      rows, cols, dact, pre, ld, dpre, static_cast<__nv_bfloat16*>(dpre_bf), ld_bf,
      static_cast<__nv_bfloat16*>(dpre_bf_t), ld_bf_t);
  return launch_status("naja_gelu_backward");
}

int naja_mse_grad(int rows, int cols, const float* out, const float* target, int ld, const float* w, double* loss,
                  float* grad, void* grad_bf, int ld_bf, void* grad_bf_t, int ld_bf_t, void* stream) {
  if (rows <= 0 || cols <= 0 || !out || !target || !loss || ld < cols || (grad_bf && ld_bf < cols) ||
      (grad_bf_t && ld_bf_t < rows))
    return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_mse_grad: bad arguments");
  if (int st = require_local("naja_mse_grad", {out, target, w, loss, grad, grad_bf, grad_bf_t})) return st;
  const long long total = static_cast<long long>(rows) * cols;
  mse_grad_kernel<<<grid_for(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      rows, cols, out, target, ld, w, loss, grad, static_cast<__nv_bfloat16*>(grad_bf), ld_bf,
      static_cast<__nv_bfloat16*>(grad_bf_t), ld_bf_t);
  return launch_status("naja_mse_grad");
}

int naja_col_sum(int rows, int cols, const float* d, int ld, float* db, void* stream) {
  if (rows <= 0 || cols <= 0 || !d || !db || ld < cols) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_col_sum: bad arguments");
  if (int st = require_local("naja_col_sum", {d, db})) return st;
  col_sum_kernel<<<(cols + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(rows, cols, d, ld, db);
  return launch_status("naja_col_sum");
}

int naja_adam(int rows, int cols, float* W, const float* g, float* m, float* v, int ld, float lr, float beta1,
              float beta2, float eps, int step, void* w_bf, int ld_bf, void* w_bf_t, int ld_bf_t, void* stream) {
  if (rows <= 0 || cols <= 0 || !W || !g || !m || !v || ld < cols || step < 1 || (w_bf && ld_bf < cols) ||
      (w_bf_t && ld_bf_t < rows))
    return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_adam: bad arguments");
  if (int st = require_local("naja_adam", {W, g, m, v, w_bf, w_bf_t})) return st;
  const float c1 = 1.0f / (1.0f - std::pow(beta1, static_cast<float>(step)));
  const float c2 = 1.0f / (1.0f - std::pow(beta2, static_cast<float>(step)));
  const long long total = static_cast<long long>(rows) * cols;
  adam_kernel<<<grid_for(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      rows, cols, W, g, m, v, ld, lr, beta1, beta2, eps, c1, c2, static_cast<__nv_bfloat16*>(w_bf), ld_bf,
      static_cast<__nv_bfloat16*>(w_bf_t), ld_bf_t);
  return launch_status("naja_adam");
}

}  // extern "C"
