// Launch planning and dispatch for the CHR step kernel (see chr_kernel.cuh).
#include <curand_kernel.h>

#include "chr.cuh"
#include "chr_kernel.cuh"

namespace naja {
int chr_launch_float_32(const ChrArgs& a, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream);
int chr_launch_float_64(const ChrArgs& a, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream);
int chr_launch_float_128(const ChrArgs& a, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream);
int chr_launch_float_256(const ChrArgs& a, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream);
int chr_launch_float_448(const ChrArgs& a, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream);
int chr_launch_float_512(const ChrArgs& a, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream);
int chr_launch_float_992(const ChrArgs& a, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream);
int chr_launch_double_32(const ChrArgs& a, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream);
int chr_launch_double_64(const ChrArgs& a, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream);
int chr_launch_double_128(const ChrArgs& a, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream);
int chr_launch_double_256(const ChrArgs& a, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream);
int chr_launch_double_448(const ChrArgs& a, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream);
int chr_launch_double_512(const ChrArgs& a, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream);
int chr_launch_double_992(const ChrArgs& a, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream);

int chr_batch_dispatch_128(const ChrArgs* base, const ModelDesc* models, const int* im, const int* ic, int nitems,
                        const BatchConfig& cfg, cudaStream_t stream, int* occ_out);
int chr_batch_dispatch_256(const ChrArgs* base, const ModelDesc* models, const int* im, const int* ic, int nitems,
                        const BatchConfig& cfg, cudaStream_t stream, int* occ_out);
int chr_batch_dispatch_512(const ChrArgs* base, const ModelDesc* models, const int* im, const int* ic, int nitems,
                        const BatchConfig& cfg, cudaStream_t stream, int* occ_out);

using namespace chr_detail;
namespace {
__global__ void mrg_tape_kernel(unsigned long long seed, int chain_base, int nchains, long count, double* tape) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nchains) return;
  curandStateMRG32k3a st;
  curand_init(seed, static_cast<unsigned long long>(chain_base + c), 0ull, &st);
  for (long i = 0; i < count; ++i) tape[static_cast<size_t>(c) * count + i] = curand_uniform_double(&st);
}

__global__ void mrg_init_kernel(unsigned long long seed, int chain_base, int nchains, curandStateMRG32k3a* st) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < nchains) curand_init(seed, static_cast<unsigned long long>(chain_base + c), 0ull, &st[c]);
}

// slack[c][r] = b[r] - sum_j A64[r][j] x_c[j] for every chain c, in FP64
// with each row's fma chain over j in order from 0.0 (the step kernel's
// recompute), rounded to the tier's type.  One thread per row for kSlackCG
// chains (they share every load of A64), the CTA's chains' x in shared
// memory (XS) or read from global memory (every lane the same address).
// The loop is latency-bound, so each thread loads kSlackJB values of its row
// before their fmas: kSlackJB loads in flight per thread.
constexpr int kSlackCG = 2;
constexpr int kSlackJB = 16;
template <class Real, bool XS>
__global__ void __launch_bounds__(128) slack_recompute_kernel(const double* __restrict__ A64, int lda,
                                                              const double* __restrict__ b, int m, int d,
                                                              const double* __restrict__ X, int ldx, int nchains,
                                                              Real* __restrict__ slack) {
  extern __shared__ double xsh[];  // XS: kSlackCG x d
  const int c0 = blockIdx.y * kSlackCG;
  const int nc = nchains - c0 < kSlackCG ? nchains - c0 : kSlackCG;
  const double* xv = X + static_cast<size_t>(c0) * ldx;
  int ldv = ldx;
  if constexpr (XS) {
    for (int i = threadIdx.x; i < nc * d; i += blockDim.x) {
      const int c = i / d, j = i - c * d;
      xsh[c * d + j] = xv[static_cast<size_t>(c) * ldx + j];
    }
    __syncthreads();
    xv = xsh;
    ldv = d;
  }
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m) return;
  double acc[kSlackCG];
#pragma unroll
  for (int c = 0; c < kSlackCG; ++c) acc[c] = 0.0;
  const double* Ar = A64 + r;
  // a CTA with fewer than kSlackCG chains repeats its last one (not stored),
  // which keeps the loop free of branches
  const double* xc[kSlackCG];
#pragma unroll
  for (int c = 0; c < kSlackCG; ++c) xc[c] = xv + static_cast<size_t>(c < nc ? c : nc - 1) * ldv;
  int j = 0;
  for (; j + kSlackJB <= d; j += kSlackJB) {
    double av[kSlackJB];
#pragma unroll
    for (int u = 0; u < kSlackJB; ++u) av[u] = __ldg(Ar + static_cast<size_t>(j + u) * lda);
#pragma unroll
    for (int u = 0; u < kSlackJB; ++u)
#pragma unroll
      for (int c = 0; c < kSlackCG; ++c) acc[c] = __fma_rn(av[u], xc[c][j + u], acc[c]);
  }
  for (; j < d; ++j) {
    const double av = __ldg(Ar + static_cast<size_t>(j) * lda);
#pragma unroll
    for (int c = 0; c < kSlackCG; ++c) acc[c] = __fma_rn(av, xc[c][j], acc[c]);
  }
#pragma unroll
  for (int c = 0; c < kSlackCG; ++c)
    if (c < nc) slack[static_cast<size_t>(c0 + c) * m + r] = Tier<Real>::from64(__dsub_rn(b[r], acc[c]));
}

// Launches slack_recompute_kernel for every chain of x (leading dimension ldx).
template <class Real>
int slack_recompute(const ChrArgs& a, const double* x, int ldx, int nchains, Real* slack, cudaStream_t stream) {
  const dim3 grid((a.m + 127) / 128, (nchains + kSlackCG - 1) / kSlackCG);
  const size_t xs_bytes = static_cast<size_t>(kSlackCG) * a.d * sizeof(double);
  if (xs_bytes <= 48 * 1024) {
    slack_recompute_kernel<Real, true><<<grid, 128, xs_bytes, stream>>>(a.A64, a.lda, a.b, a.m, a.d, x, ldx,
                                                                         nchains, slack);
  } else {
    slack_recompute_kernel<Real, false><<<grid, 128, 0, stream>>>(a.A64, a.lda, a.b, a.m, a.d, x, ldx, nchains,
                                                                   slack);
  }
  return cudaGetLastError() == cudaSuccess ? NAJA_OK : NAJA_ERR_CUDA;
}

// Largest chunks-per-warp capacity used for a thread count (the slack of R
// chunks takes R * V registers per thread, V rows per lane and chunk).
int max_chunks_for(int threads, int v) { return (threads <= 512 ? 32 : 16) / v; }
// Largest chunk count of the uniform-chunk kernels (instantiated 1..8).
constexpr int kMaxUniformChunks = 8;

}  // namespace

namespace {
int plan_single(int precision, int m, int d, int lda, int tpb, int max_slots, ChrLaunchConfig* out) {
  const int elt = precision == NAJA_PREC_FP64 ? 8 : 4;
  int threads = 0;
  if (tpb > 0) {
    // The reference's thread counts (chr.cu:529-551).  A block also holds the
    // producer warp, so 1024 maps to 992 consumer threads.
    if (tpb != 32 && tpb != 64 && tpb != 128 && tpb != 256 && tpb != 512 && tpb != 1024) return NAJA_ERR_INVALID_ARGUMENT;
    threads = tpb == 1024 ? 992 : tpb;
  } else {
    // Automatic: at most 12 rows per thread, 992 threads only when 512 would
    // hold more than 16.  Fewer warps per chain carry less per-step fixed
    // work: at m = 5200 a step takes 2.07 us with 512 threads, 2.56 us with
    // 992 and 3.26 us with 256 (B200, 16 chains).
    threads = 32;
    while (threads < 512 && (m + threads - 1) / threads > 12) threads *= 2;
    if ((m + threads - 1) / threads > 16) threads = 992;
  }
  const int chunk = 32 * standalone_v(precision);
  const int chunks = (m + chunk - 1) / chunk, warps = threads / 32;
  int rows = 1;
  while (rows * warps < chunks) rows *= 2;
  if (rows > max_chunks_for(threads, standalone_v(precision))) return NAJA_ERR_UNSUPPORTED;
  int slots = kMaxSlots;
  if (max_slots > 0 && max_slots < slots) slots = max_slots;
  Layout L = make_layout(d, lda, elt, threads, slots);
  while (slots >= 3 && L.total > kSmemBudget) {
    --slots;
    L = make_layout(d, lda, elt, threads, slots);
  }
  if (L.total > kSmemBudget || slots < 3) {
    slots = 0;  // direct: columns straight from L2 / HBM
    L = make_layout(d, lda, elt, threads, 0);
    if (L.total > kSmemBudget) return NAJA_ERR_UNSUPPORTED;
  }
  out->threads = threads;
  out->rows = rows;
  out->slots = slots;
  out->smem = L.total;
  out->cluster = 1;
  out->slice_lda = lda;
  out->max_col = 0;
  out->pair_scatter = 0;
  out->uniform = 0;
  // Uniform chunks: every warp runs the same R = ceil(chunks / warps)
  // chunks as one straight-line row pass (rows past m repeat the last V).
  const int v = standalone_v(precision), exact = (chunks + warps - 1) / warps;
  if (m % v == 0 && m >= v && exact <= kMaxUniformChunks && exact <= max_chunks_for(threads, v)) {
    out->uniform = 1;
    out->rows = exact;
    // 14 warps where they hold the same chunks per warp as 16: fewer row
    // slots repeat (m 5200: 42 for 41 chunks instead of 48); the layout
    // depends on the thread count, so it is planned again
    if (tpb <= 0 && threads == 512 && 14 * exact >= chunks) {
      const Layout L448 = make_layout(d, lda, elt, 448, slots);
      if (L448.total <= kSmemBudget) {
        out->threads = 448;
        out->smem = L448.total;
      }
    }
  }
  return NAJA_OK;
}

// A chain over `cs` CTAs: 128 or 256 consumer threads per CTA (about 8 rows
// per thread of the CTA's slice), the slot ring sized for the slice.
int plan_cluster(int precision, int m, int d, int tpb, int max_slots, int cs, ChrLaunchConfig* out) {
  const int elt = precision == NAJA_PREC_FP64 ? 8 : 4;
  const int chunk = 32 * kClusterV;
  const int nc = (m + chunk - 1) / chunk;
  if (cs < 2 || cs > 8 || nc < cs) return NAJA_ERR_UNSUPPORTED;
  const int slice_chunks = (nc + cs - 1) / cs;
  const int slice_rows = slice_chunks * chunk;
  int threads;
  if (tpb > 0) {
    if (tpb != 128 && tpb != 256) return NAJA_ERR_UNSUPPORTED;
    threads = tpb;
  } else {
    threads = (slice_rows + 127) / 128 > 8 ? 256 : 128;
  }
  const int warps = threads / 32;
  int rows = 1;
  while (rows * warps < slice_chunks) rows *= 2;
  if (rows > max_chunks_for(threads, kClusterV)) return NAJA_ERR_UNSUPPORTED;
  const int slda = (slice_rows + 31) / 32 * 32;
  int slots = kMaxSlots;
  if (max_slots > 0 && max_slots < slots) slots = max_slots;
  Layout L = make_layout(d, slda, elt, threads, slots);
  // the cluster kernel also holds ~1 KB of static shared memory
  while (slots >= 3 && L.total + 1024 > kSmemBudget) {
    --slots;
    L = make_layout(d, slda, elt, threads, slots);
  }
  if (L.total + 1024 > kSmemBudget || slots < 3) return NAJA_ERR_UNSUPPORTED;
  out->threads = threads;
  out->rows = rows;
  out->slots = slots;
  out->smem = L.total;
  out->cluster = cs;
  out->slice_lda = slda;
  out->max_col = 0;
  out->pair_scatter = 0;
  out->uniform = 0;
  return NAJA_OK;
}
}  // namespace

int chr_plan(int precision, int m, int d, int lda, int tpb, int max_slots, int nchains, int cluster, int sms,
             ChrLaunchConfig* out) {
  if (cluster < 0 || cluster > 8) return NAJA_ERR_INVALID_ARGUMENT;
  // Automatic is one CTA per chain: splitting a chain over a cluster was
  // measured slower at every size tried (16 chains, m = 5200: 2.8-6.8 us per
  // step against 2.07 us), the cross-SM exchange costing more per step than
  // the split rows save.  The split stays available on request.
  (void)nchains;
  (void)sms;
  if (cluster >= 2) return plan_cluster(precision, m, d, tpb, max_slots, cluster, out);
  return plan_single(precision, m, d, lda, tpb, max_slots, out);
}

int chr_launch(int precision, const ChrArgs& args, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream) {
  if (nchains <= 0) return NAJA_OK;
  const bool f64 = precision == NAJA_PREC_FP64;
  switch (cfg.threads) {
    case 32: return f64 ? chr_launch_double_32(args, nchains, cfg, stream) : chr_launch_float_32(args, nchains, cfg, stream);
    case 64: return f64 ? chr_launch_double_64(args, nchains, cfg, stream) : chr_launch_float_64(args, nchains, cfg, stream);
    case 128: return f64 ? chr_launch_double_128(args, nchains, cfg, stream) : chr_launch_float_128(args, nchains, cfg, stream);
    case 256: return f64 ? chr_launch_double_256(args, nchains, cfg, stream) : chr_launch_float_256(args, nchains, cfg, stream);
    case 448: return f64 ? chr_launch_double_448(args, nchains, cfg, stream) : chr_launch_float_448(args, nchains, cfg, stream);
    case 512: return f64 ? chr_launch_double_512(args, nchains, cfg, stream) : chr_launch_float_512(args, nchains, cfg, stream);
    case 992: return f64 ? chr_launch_double_992(args, nchains, cfg, stream) : chr_launch_float_992(args, nchains, cfg, stream);
    default: return NAJA_ERR_UNSUPPORTED;
  }
}

int chr_run_segmented(int precision, const ChrArgs& a0, int nchains, const ChrLaunchConfig& cfg,
                      cudaStream_t stream, long long* launches, const SpArgs* sp) {
  if (launches) *launches = 0;
  if (nchains <= 0) return NAJA_OK;
  const long long K = a0.resync;
  const long long total = launch_steps_host(a0);
  if (K <= 0 || a0.t_first != 0 || a0.slack_in) return NAJA_ERR_INVALID_ARGUMENT;
  const long long nseg = (total + K - 1) / K;
  const int d = a0.d, m = a0.m;
  const size_t elt = precision == NAJA_PREC_FP64 ? sizeof(double) : sizeof(float);
  const size_t x_bytes = static_cast<size_t>(nchains) * d * sizeof(double);
  const size_t s_bytes = static_cast<size_t>(nchains) * m * elt;
  const bool own_states = a0.rng != 0 && !a0.rng_state;
  void *xb = nullptr, *sb = nullptr, *rs = nullptr;
  auto release = [&]() {
    if (xb) cudaFreeAsync(xb, stream);
    if (sb) cudaFreeAsync(sb, stream);
    if (rs) cudaFreeAsync(rs, stream);
  };
  cudaError_t e = cudaMallocAsync(&xb, 2 * x_bytes, stream);
  if (e == cudaSuccess) e = cudaMallocAsync(&sb, s_bytes, stream);
  if (e == cudaSuccess && own_states) e = cudaMallocAsync(&rs, nchains * sizeof(curandStateMRG32k3a), stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    release();
    return NAJA_ERR_NO_MEMORY;
  }
  double* xs[2] = {static_cast<double*>(xb), static_cast<double*>(xb) + static_cast<size_t>(nchains) * d};
  // positions travel between segments chain-major with leading dimension d
  e = cudaMemcpy2DAsync(xs[0], d * sizeof(double), a0.X0, static_cast<size_t>(a0.ldx) * sizeof(double),
                        d * sizeof(double), nchains, cudaMemcpyDeviceToDevice, stream);
  int st = e == cudaSuccess ? NAJA_OK : NAJA_ERR_CUDA;
  long long n_launch = 0;
  if (!st && own_states) {
    st = mrg_init_states(a0.seed, a0.chain_base, nchains, rs, stream);
    ++n_launch;
  }
  for (long long s = 0; s < nseg && !st; ++s) {
    const double* xin = xs[s % 2];
    st = precision == NAJA_PREC_FP64 ? slack_recompute(a0, xin, d, nchains, static_cast<double*>(sb), stream)
                                     : slack_recompute(a0, xin, d, nchains, static_cast<float*>(sb), stream);
    if (st) break;
    ChrArgs a = a0;
    a.X0 = xin;
    a.ldx = d;
    a.X_final = xs[(s + 1) % 2];
    a.t_first = s * K;
    a.steps = total - s * K < K ? total - s * K : K;
    a.slack_in = sb;
    a.resync = 0;  // this segment's recompute is the one just made
    a.slack_final = s + 1 == nseg ? a0.slack_final : nullptr;
    if (own_states) a.rng_state = rs;
    st = sp ? chr_sparse_launch(precision, a, *sp, nchains, cfg, stream)
            : chr_launch(precision, a, nchains, cfg, stream);
    n_launch += 2;
  }
  if (!st && a0.X_final) {
    e = cudaMemcpy2DAsync(a0.X_final, static_cast<size_t>(a0.ldx) * sizeof(double), xs[nseg % 2],
                          d * sizeof(double), d * sizeof(double), nchains, cudaMemcpyDeviceToDevice, stream);
    if (e != cudaSuccess) st = NAJA_ERR_CUDA;
  }
  release();
  if (launches) *launches = n_launch;
  return st;
}

int mrg_tape(unsigned long long seed, int chain_base, int nchains, long count, double* tape, cudaStream_t stream) {
  if (nchains <= 0 || count <= 0) return NAJA_OK;
  mrg_tape_kernel<<<(nchains + 63) / 64, 64, 0, stream>>>(seed, chain_base, nchains, count, tape);
  return cudaGetLastError() == cudaSuccess ? NAJA_OK : NAJA_ERR_CUDA;
}

int mrg_init_states(unsigned long long seed, int chain_base, int nchains, void* states, cudaStream_t stream) {
  if (nchains <= 0) return NAJA_OK;
  mrg_init_kernel<<<(nchains + 63) / 64, 64, 0, stream>>>(seed, chain_base, nchains,
                                                         static_cast<curandStateMRG32k3a*>(states));
  return cudaGetLastError() == cudaSuccess ? NAJA_OK : NAJA_ERR_CUDA;
}

int chr_batch_plan(int m_max, int d, int lda_max, BatchConfig* cfg) {
  if (cfg->sparse) return chr_sparse_batch_plan(m_max, d, cfg);
  const int nt = cfg->threads;
  if (nt != 128 && nt != 256 && nt != 512) return NAJA_ERR_INVALID_ARGUMENT;
  const int chunks = (m_max + 32 * kBatchV - 1) / (32 * kBatchV), warps = nt / 32;
  int rows = 0;
  for (const int* c = batch_chunk_capacities(nt, cfg->slack_smem != 0); *c; ++c) {
    if (*c * warps >= chunks) {
      rows = *c;
      break;
    }
  }
  if (rows == 0) return NAJA_ERR_UNSUPPORTED;
  if (cfg->slots != 0 && (cfg->slots < 2 || cfg->slots > kMaxSlots)) return NAJA_ERR_INVALID_ARGUMENT;
  cfg->rows = rows;
  cfg->lda_max = lda_max;
  const Layout L = make_layout(d, lda_max, 4, nt, cfg->slots, cfg->slack_smem ? lda_max : 0);
  // the kernel also holds one ChrArgs in static shared memory
  if (L.total + align_up(sizeof(ChrArgs), 128) > kSmemBudget) return NAJA_ERR_UNSUPPORTED;
  cfg->smem = L.total;
  return NAJA_OK;
}

static int batch_dispatch(const ChrArgs* base, const ModelDesc* models, const int* im, const int* ic, int nitems,
                          const BatchConfig& cfg, cudaStream_t stream, int* occ) {
  if (cfg.sparse) return chr_sparse_batch_dispatch(base, models, im, ic, nitems, cfg, stream, occ);
  switch (cfg.threads) {
    case 128: return chr_batch_dispatch_128(base, models, im, ic, nitems, cfg, stream, occ);
    case 256: return chr_batch_dispatch_256(base, models, im, ic, nitems, cfg, stream, occ);
    case 512: return chr_batch_dispatch_512(base, models, im, ic, nitems, cfg, stream, occ);
    default: return NAJA_ERR_UNSUPPORTED;
  }
}

int chr_batch_occupancy(const BatchConfig& cfg, int* ctas_per_sm) {
  return batch_dispatch(nullptr, nullptr, nullptr, nullptr, 0, cfg, nullptr, ctas_per_sm);
}

int chr_batch_launch(const ChrArgs& base, const ModelDesc* models, const int* item_model, const int* item_chain,
                     int nitems, const BatchConfig& cfg, cudaStream_t stream) {
  if (nitems <= 0) return NAJA_OK;
  return batch_dispatch(&base, models, item_model, item_chain, nitems, cfg, stream, nullptr);
}

size_t mrg_state_bytes() { return sizeof(curandStateMRG32k3a); }

}  // namespace naja
