// Sampling with the backmap and the delivery of its rows overlapped, as one
// call: naja_chr_run_backmapped (include/naja_chr.h).
//
// The reference's job (src/engine/job_sampling.cu:300-385 of
// quothbonney/naja) samples every chain to the end, then backmaps the whole
// sample matrix (CoordinateHitAndRunBackmap, src/gpu/chr.cu:72-99), then
// copies it to the host.  Here the chains run in chunks of whole
// lcm(resync, thinning) periods on one stream while the previous chunk's
// backmap (tensor cores, the SMs the chains leave idle) and its copy to the
// host run on a second stream:
//
//   stream chr : CHR(0)  CHR(1)  CHR(2) ...        (one CTA per chain)
//   stream bm  :         BM(0)+D2H(0)  BM(1)+D2H(1) ...
//
// Chunk k + 1 is queued before chunk k's backmap and copy, so a copy into
// pageable host memory (which returns only when it is done) never leaves
// the step kernel without queued work.  A chunk boundary falls where a
// single run recomputes the slack from x in FP64 anyway, and a launch starts
// from the previous chunk's final x (FP64) and the same Philox step counter:
// the samples are those of one naja_chr_run launch, bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <numeric>
#include <string>

#include "../../include/naja_chr.h"
#include "capi_internal.cuh"

namespace naja {
namespace {

constexpr long long kChunkTargetSteps = 1LL << 16;

// The two work streams and their events.  On destruction (every exit path)
// the caller's stream is made to wait for both, so the stream-ordered frees of
// the call's buffers on that stream come after every use of them.
struct WorkStreams {
  cudaStream_t caller = nullptr, chr = nullptr, bm = nullptr;
  cudaEvent_t start = nullptr, done[2] = {nullptr, nullptr}, freed[2] = {nullptr, nullptr}, end_chr = nullptr,
              end_bm = nullptr;
  bool freed_set[2] = {false, false};

  int create(cudaStream_t s) {
    caller = s;
    cudaError_t e = cudaStreamCreateWithFlags(&chr, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&bm, cudaStreamNonBlocking);
    cudaEvent_t* evs[] = {&start, &done[0], &done[1], &freed[0], &freed[1], &end_chr, &end_bm};
    for (cudaEvent_t* ev : evs)
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("naja_chr_run_backmapped: ") + cudaGetErrorString(e));
    return NAJA_OK;
  }
  // Both work streams start after everything queued on the caller's stream.
  int begin() {
    cudaError_t e = cudaEventRecord(start, caller);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(chr, start, 0);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(bm, start, 0);
    if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("naja_chr_run_backmapped: ") + cudaGetErrorString(e));
    return NAJA_OK;
  }
  void join() {
    if (chr && end_chr && cudaEventRecord(end_chr, chr) == cudaSuccess) cudaStreamWaitEvent(caller, end_chr, 0);
    if (bm && end_bm && cudaEventRecord(end_bm, bm) == cudaSuccess) cudaStreamWaitEvent(caller, end_bm, 0);
  }
  ~WorkStreams() {
    join();
    cudaEvent_t evs[] = {start, done[0], done[1], freed[0], freed[1], end_chr, end_bm};
    for (cudaEvent_t ev : evs)
      if (ev) cudaEventDestroy(ev);
    if (chr) cudaStreamDestroy(chr);
    if (bm) cudaStreamDestroy(bm);
  }
};

// Samples per chunk: whole periods of lcm(resync, thinning) steps, about
// kChunkTargetSteps steps long; all of nspc when the run cannot be split.
long long auto_chunk(const naja_chr_params* p) {
  if (p->rng != NAJA_RNG_PHILOX || p->resync_interval <= 0) return p->nspc;
  const long long period = std::lcm(static_cast<long long>(p->resync_interval), static_cast<long long>(p->thinning)) /
                           p->thinning;
  const long long k = std::max(1LL, kChunkTargetSteps / (period * p->thinning));
  return std::min<long long>(p->nspc, k * period);
}

int copy_rows(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s);
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("naja_chr_run_backmapped: copy: ") + cudaGetErrorString(e));
  return NAJA_OK;
}

}  // namespace
}  // namespace naja

using namespace naja;

extern "C" int naja_chr_run_backmapped(const naja_polytope* P, const naja_chr_params* params, const double* X0,
                                       int ldx, int n, const double* T, int ldt, const double* shift, int mode,
                                       void* V, int v_dtype, void* samples, double* X_final, int chunk_nspc,
                                       void* stream_ptr) {
  static const char* kFn = "naja_chr_run_backmapped";
  if (!P || !params || !X0 || !T || !shift || !V)
    return fail(NAJA_ERR_INVALID_ARGUMENT, std::string(kFn) + ": null argument");
  int m = 0, d = 0;
  naja_polytope_shape(P, &m, &d);
  const naja_chr_params& p = *params;
  if (p.nchains <= 0 || p.nspc <= 0 || p.thinning <= 0)
    return fail(NAJA_ERR_INVALID_ARGUMENT, std::string(kFn) + ": nchains, nspc and thinning must be positive");
  if (n <= 0 || ldt < n) return fail(NAJA_ERR_INVALID_ARGUMENT, "backmap_into: transformation shape mismatch with samples");
  if (ldx < d) return fail(NAJA_ERR_INVALID_ARGUMENT, std::string(kFn) + ": ldx < d");
  if (mode != NAJA_BACKMAP_FP64 && mode != NAJA_BACKMAP_BF16X3 && mode != NAJA_BACKMAP_TF32X3)
    return fail(NAJA_ERR_INVALID_ARGUMENT, std::string(kFn) + ": unknown backmap mode");
  if ((v_dtype != NAJA_DTYPE_F32 && v_dtype != NAJA_DTYPE_F64) ||
      (p.out_dtype != NAJA_DTYPE_F32 && p.out_dtype != NAJA_DTYPE_F64))
    return fail(NAJA_ERR_INVALID_ARGUMENT, std::string(kFn) + ": unknown dtype");
  if (p.chain_base != 0 || (p.out_nchains != 0 && p.out_nchains != p.nchains))
    return fail(NAJA_ERR_INVALID_ARGUMENT, std::string(kFn) + ": runs whole jobs (chain_base 0, out_nchains = nchains)");
  long long cs = chunk_nspc > 0 ? std::min<long long>(chunk_nspc, p.nspc) : auto_chunk(params);
  if (cs < p.nspc && (p.rng != NAJA_RNG_PHILOX || p.resync_interval <= 0 || p.rng_state ||
                      (cs * p.thinning) % p.resync_interval != 0))
    return fail(NAJA_ERR_INVALID_ARGUMENT,
                std::string(kFn) + ": a chunk must span whole resync intervals of a Philox run (resync_interval > 0)");
  const int device = polytope_device(P);
  DeviceGuard g(device);
  if (!g.ok()) return fail(NAJA_ERR_CUDA, std::string(kFn) + ": cannot select device");
  if (int st = require_local(kFn, {X0, T, shift, V, samples, X_final})) return st;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);

  // the kernel choice builds the compressed columns (synchronously) the first time
  naja_chr_params pk = p;
  pk.nspc = static_cast<int>(cs);
  pk.out_nchains = 0;
  int st = naja_chr_kernel_choice(P, &pk, nullptr, nullptr, nullptr, nullptr);
  if (st) return st;

  const int nch = p.nchains;
  const size_t selt = p.out_dtype == NAJA_DTYPE_F64 ? 8 : 4, velt = v_dtype == NAJA_DTYPE_F64 ? 8 : 4;
  const size_t chunk_rows = static_cast<size_t>(cs) * nch;
  const bool v_dev = is_device_ptr(V), s_dev = samples && is_device_ptr(samples);
  const bool tc = mode != NAJA_BACKMAP_FP64;

  DeviceBuffer bT, bsh, bx0, bx1, bs0, bs1, bv0, bv1, bTh, bTl, bYh, bYl, berr;
  const void *dT = nullptr, *dS = nullptr;
  if ((st = device_view(T, static_cast<size_t>(ldt) * (d - 1) * 8 + static_cast<size_t>(n) * 8, stream, bT, &dT)))
    return st;
  if ((st = device_view(shift, static_cast<size_t>(n) * 8, stream, bsh, &dS))) return st;
  const size_t xbytes = static_cast<size_t>(nch) * d * 8;
  if ((st = bx0.alloc(xbytes, stream)) || (st = bx1.alloc(xbytes, stream))) return st;
  if (!s_dev && ((st = bs0.alloc(chunk_rows * d * selt, stream)) || (st = bs1.alloc(chunk_rows * d * selt, stream))))
    return st;
  if (!v_dev && ((st = bv0.alloc(chunk_rows * n * velt, stream)) || (st = bv1.alloc(chunk_rows * n * velt, stream))))
    return st;
  if (tc) {
    const size_t yb = backmap_tc_operand_bytes(static_cast<long long>(chunk_rows), d, mode);
    const size_t tb = backmap_tc_operand_bytes(n, d, mode);
    if ((st = bTh.alloc(tb, stream)) || (st = bTl.alloc(tb, stream)) || (st = bYh.alloc(yb, stream)) ||
        (st = bYl.alloc(yb, stream)) || (st = berr.alloc(4 * sizeof(int), stream)))
      return st;
    const cudaError_t e = cudaMemsetAsync(berr.ptr, 0, 4 * sizeof(int), stream);
    if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string(kFn) + ": " + cudaGetErrorString(e));
  }
  double* xs[2] = {static_cast<double*>(bx0.ptr), static_cast<double*>(bx1.ptr)};
  cudaError_t e = cudaMemcpy2DAsync(xs[0], static_cast<size_t>(d) * 8, X0, static_cast<size_t>(ldx) * 8,
                                    static_cast<size_t>(d) * 8, nch, cudaMemcpyDefault, stream);
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string(kFn) + ": start points: " + cudaGetErrorString(e));

  WorkStreams ws;  // declared after the buffers: joins the caller's stream before they are freed
  if ((st = ws.create(stream)) || (st = ws.begin())) return st;
  if (tc && (st = backmap_tc_split_T(n, d, static_cast<const double*>(dT), ldt, bTh.ptr, bTl.ptr, mode, ws.bm)))
    return st;

  void* sbuf[2] = {bs0.ptr, bs1.ptr};
  void* vbuf[2] = {bv0.ptr, bv1.ptr};
  const long long nchunks = (p.nspc + cs - 1) / cs;
  auto rows_of = [&](long long k) { return static_cast<size_t>(std::min<long long>(cs, p.nspc - k * cs)) * nch; };
  auto sample_ptr = [&](long long k) -> void* {
    return s_dev ? static_cast<char*>(samples) + static_cast<size_t>(k * cs) * nch * d * selt : sbuf[k % 2];
  };
  // CHR of chunk k on the chr stream: from xs[k % 2] to xs[(k + 1) % 2]
  auto queue_chr = [&](long long k) -> int {
    const int b = static_cast<int>(k % 2);
    if (!s_dev && ws.freed_set[b] && (e = cudaStreamWaitEvent(ws.chr, ws.freed[b], 0)) != cudaSuccess)
      return fail(NAJA_ERR_CUDA, std::string(kFn) + ": " + cudaGetErrorString(e));
    naja_chr_params q = p;
    q.nspc = static_cast<int>(rows_of(k) / nch);
    q.out_nchains = 0;
    q.step_offset = p.step_offset + k * cs * p.thinning;
    int s2 = naja_chr_run(P, &q, xs[k % 2], d, sample_ptr(k), xs[(k + 1) % 2], ws.chr);
    if (s2) return s2;
    if ((e = cudaEventRecord(ws.done[b], ws.chr)) != cudaSuccess)
      return fail(NAJA_ERR_CUDA, std::string(kFn) + ": " + cudaGetErrorString(e));
    return NAJA_OK;
  };
  // backmap of chunk k and its copies on the bm stream
  auto queue_bm = [&](long long k) -> int {
    const int b = static_cast<int>(k % 2);
    if ((e = cudaStreamWaitEvent(ws.bm, ws.done[b], 0)) != cudaSuccess)
      return fail(NAJA_ERR_CUDA, std::string(kFn) + ": " + cudaGetErrorString(e));
    const size_t rows = rows_of(k);
    const size_t row0 = static_cast<size_t>(k * cs) * nch;
    void* vdst = v_dev ? static_cast<char*>(V) + row0 * n * velt : vbuf[b];
    const void* y = sample_ptr(k);
    int s2 = tc ? backmap_tc_enqueue(n, d, static_cast<long long>(rows), y, p.out_dtype, bTh.ptr, bTl.ptr, bYh.ptr,
                                     bYl.ptr, static_cast<const double*>(dS), vdst, v_dtype, mode,
                                     static_cast<int*>(berr.ptr), ws.bm)
                : backmap_fp64_enqueue(n, d, static_cast<long long>(rows), static_cast<const double*>(dT), ldt,
                                       static_cast<const double*>(dS), y, p.out_dtype, vdst, v_dtype, ws.bm);
    if (s2) return s2;
    if (!v_dev && (s2 = copy_rows(static_cast<char*>(V) + row0 * n * velt, vdst, rows * n * velt, ws.bm))) return s2;
    if (samples && !s_dev &&
        (s2 = copy_rows(static_cast<char*>(samples) + row0 * d * selt, y, rows * d * selt, ws.bm)))
      return s2;
    if ((e = cudaEventRecord(ws.freed[b], ws.bm)) != cudaSuccess)
      return fail(NAJA_ERR_CUDA, std::string(kFn) + ": " + cudaGetErrorString(e));
    ws.freed_set[b] = true;
    return NAJA_OK;
  };
  if ((st = queue_chr(0))) return st;
  for (long long k = 0; k < nchunks; ++k) {
    if (k + 1 < nchunks && (st = queue_chr(k + 1))) return st;
    if ((st = queue_bm(k))) return st;
  }
  if (X_final) {
    e = cudaMemcpy2DAsync(X_final, static_cast<size_t>(ldx) * 8, xs[nchunks % 2], static_cast<size_t>(d) * 8,
                          static_cast<size_t>(d) * 8, nch, cudaMemcpyDefault, ws.chr);
    if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string(kFn) + ": final state: " + cudaGetErrorString(e));
  }
  ws.join();
  e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string(kFn) + ": " + cudaGetErrorString(e));
  if ((st = naja_polytope_check(P))) return st;
  if (tc && (st = backmap_tc_read_error(static_cast<const int*>(berr.ptr), stream, "backmap"))) return st;
  return NAJA_OK;
}
