// Device-side `naja validate` metrics: Geyer ESS per (dim, chain) and
// split-R-hat per dim, following src/validate/mcmc.cpp:17-194 of
// quothbonney/naja.
//
// ESS: one CTA per series.  The series is centred in shared memory, then
// autocovariances are summed directly (FP32 products, FP64 sums), one lag
// per thread, in blocks of lags until Geyer's initial positive sequence
// stops.  The reference obtains the same acov[k] = (1/n) sum (x_t-m)(x_{t+k}-m)
// from a float FFT of size 2n; the direct sum needs only the lags the rule
// reaches (a few blocks for a mixing chain) and has no FFT round-off.
//
// R-hat: one CTA per dim, half-chain sums in FP64 exactly as mcmc.cpp does.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/naja_chr.h"
#include "capi_internal.cuh"

namespace naja {
namespace {

constexpr int kEssThreads = 256;
constexpr long kEssMaxSeries = 48 * 1024;  // floats kept on chip per series

__device__ __forceinline__ long series_row(int layout, int c, long i, long spc, int nchains) {
  return layout == 0 ? static_cast<long>(c) * spc + i : i * nchains + c;
}

__device__ double block_sum(double v, double* scratch) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) scratch[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = (l < static_cast<int>(blockDim.x >> 5)) ? scratch[l] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (l == 0) scratch[0] = t;
  }
  __syncthreads();
  t = scratch[0];
  __syncthreads();
  return t;
}

__global__ void __launch_bounds__(kEssThreads) ess_kernel(const float* __restrict__ s, long N, int dim, int nchains,
                                                        int layout, double* __restrict__ ess) {
  extern __shared__ __align__(16) unsigned char sm[];
  __shared__ double scratch[32];
  __shared__ double acov_blk[2 * kEssThreads + 2];
  __shared__ int stop_flag;
  __shared__ double tau_sh;
  float* y = reinterpret_cast<float*>(sm);
  const long spc = N / nchains;
  const int series = blockIdx.x;
  const int dd = series / nchains, c = series % nchains;
  const long n = spc;
  if (n < 4) {
    if (threadIdx.x == 0) ess[series] = static_cast<double>(n);
    return;
  }
  double part = 0.0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) {
    const float v = s[series_row(layout, c, i, spc, nchains) * dim + dd];
    y[i] = v;
    part += static_cast<double>(v);
  }
  const double mean = block_sum(part, scratch) / static_cast<double>(n);
  for (long i = threadIdx.x; i < n; i += blockDim.x) y[i] = static_cast<float>(static_cast<double>(y[i]) - mean);
  __syncthreads();
  // acov[0]
  part = 0.0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) part += static_cast<double>(y[i]) * y[i];
  const double var = block_sum(part, scratch) / static_cast<double>(n);
  if (var < 1e-30) {
    if (threadIdx.x == 0) ess[series] = 1.0;
    return;
  }
  if (threadIdx.x == 0) {
    stop_flag = 0;
    tau_sh = 1.0;
  }
  __syncthreads();
  // Lags are evaluated in blocks [base, base + 2*T); pair k uses lags 2k-1, 2k.
  const long kmax = n / 2;  // pairs k = 1 .. kmax-1
  for (long base = 1; base <= 2 * (kmax - 1); base += 2 * kEssThreads) {
    for (int q = 0; q < 2; ++q) {
      const long lag = base + threadIdx.x + q * kEssThreads;
      double acc = 0.0;
      if (lag < n) {
        const float* yk = y + lag;
        const long len = n - lag;
        for (long t = 0; t < len; ++t) acc += static_cast<double>(y[t] * yk[t]);
      }
      acov_blk[threadIdx.x + q * kEssThreads] = acc / static_cast<double>(n);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double tau = tau_sh;
      // acov_blk[i] holds lag base + i; base is odd, so pairs are (i, i+1) for even i.
      for (int i = 0; i + 1 < 2 * kEssThreads; i += 2) {
        const long k = (base + i + 1) / 2;
        if (k >= kmax) {
          stop_flag = 1;
          break;
        }
        const double pair = acov_blk[i] / var + acov_blk[i + 1] / var;
        if (pair < 0.0) {
          stop_flag = 1;
          break;
        }
        tau += 2.0 * pair;
      }
      tau_sh = tau;
    }
    __syncthreads();
    if (stop_flag) break;
  }
  if (threadIdx.x == 0) {
    double tau = tau_sh < 1.0 ? 1.0 : tau_sh;
    ess[series] = static_cast<double>(n) / tau;
  }
}

__global__ void rhat_kernel(const float* __restrict__ s, long N, int dim, int nchains, int layout,
                            double* __restrict__ rhat) {
  __shared__ double scratch[32];
  const int dd = blockIdx.x;
  const long spc = N / nchains;
  const long half = spc / 2;
  const int m = 2 * nchains;
  double grand = 0.0, W = 0.0;
  // First pass: half-chain means and Bessel-corrected variances.
  for (int j = 0; j < m; ++j) {
    const int c = j / 2, h = j % 2;
    double ps = 0.0, ps2 = 0.0;
    for (long i = threadIdx.x; i < half; i += blockDim.x) {
      const double v = static_cast<double>(s[series_row(layout, c, h * half + i, spc, nchains) * dim + dd]);
      ps += v;
      ps2 += v * v;
    }
    const double S = block_sum(ps, scratch);
    const double S2 = block_sum(ps2, scratch);
    const double mean = S / half;
    double var = (S2 / half) - mean * mean;
    var = var * half / (half - 1);
    grand += mean;
    W += var;
  }
  // Second pass for B (sum of squared deviations from the grand mean).
  const double gm = grand / m;
  double B = 0.0;
  for (int j = 0; j < m; ++j) {
    const int c = j / 2, h = j % 2;
    double ps = 0.0;
    for (long i = threadIdx.x; i < half; i += blockDim.x)
      ps += static_cast<double>(s[series_row(layout, c, h * half + i, spc, nchains) * dim + dd]);
    const double mean = block_sum(ps, scratch) / half;
    B += (mean - gm) * (mean - gm);
  }
  if (threadIdx.x == 0) {
    B *= static_cast<double>(half) / (m - 1);
    W /= m;
    const double var_hat = ((half - 1.0) / half) * W + B / half;
    rhat[dd] = (W > 1e-30) ? sqrt(var_hat / W) : 1.0;
  }
}

}  // namespace
}  // namespace naja

using namespace naja;

extern "C" int naja_validate(const float* samples, long long N, int dim, int nchains, int layout, double* ess,
                             double* rhat, void* stream_ptr) {
  if (!samples || dim <= 0 || nchains <= 0 || N <= 0)
    return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_validate: bad arguments");
  if (layout != 0 && layout != 1) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_validate: layout must be 0 or 1");
  if (N % nchains != 0)
    return fail(NAJA_ERR_RUNTIME, "n_total (" + std::to_string(N) + ") not divisible by n_chains (" +
                                      std::to_string(nchains) + ")");
  const long spc = static_cast<long>(N / nchains);
  if (ess && spc < 4) return fail(NAJA_ERR_INVALID_ARGUMENT, "compute_ess: fewer than 4 samples per chain");
  if (rhat && spc / 2 < 2) return fail(NAJA_ERR_INVALID_ARGUMENT, "compute_split_rhat: chain too short to split");
  if (ess && spc > kEssMaxSeries)
    return fail(NAJA_ERR_UNSUPPORTED, "naja_validate: more than " + std::to_string(kEssMaxSeries) +
                                          " samples per chain");
  if (int st = require_local("naja_validate", {samples, ess, rhat})) return st;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  DeviceBuffer bs, be, br;
  const void* ds = nullptr;
  int st = device_view(samples, static_cast<size_t>(N) * dim * sizeof(float), stream, bs, &ds);
  if (st) return st;
  double* de = ess;
  double* dr = rhat;
  const bool host_e = ess && !is_device_ptr(ess), host_r = rhat && !is_device_ptr(rhat);
  if (host_e) {
    if ((st = be.alloc(static_cast<size_t>(dim) * nchains * sizeof(double), stream))) return st;
    de = static_cast<double*>(be.ptr);
  }
  if (host_r) {
    if ((st = br.alloc(static_cast<size_t>(dim) * sizeof(double), stream))) return st;
    dr = static_cast<double*>(br.ptr);
  }
  if (ess) {
    const size_t smem = static_cast<size_t>(spc) * sizeof(float);
    cudaFuncSetAttribute(ess_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    ess_kernel<<<dim * nchains, kEssThreads, smem, stream>>>(static_cast<const float*>(ds), static_cast<long>(N), dim,
                                                             nchains, layout, de);
  }
  if (rhat) {
    rhat_kernel<<<dim, 256, 0, stream>>>(static_cast<const float*>(ds), static_cast<long>(N), dim, nchains, layout, dr);
  }
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && host_e)
    e = cudaMemcpyAsync(ess, de, static_cast<size_t>(dim) * nchains * sizeof(double), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess && host_r)
    e = cudaMemcpyAsync(rhat, dr, static_cast<size_t>(dim) * sizeof(double), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess && (host_e || host_r || bs.ptr)) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("naja_validate: ") + cudaGetErrorString(e));
  return NAJA_OK;
}
