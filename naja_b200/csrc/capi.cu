// C ABI of libnaja_b200.so (declared in include/naja_chr.h).
//
// The host side of the reference's GPU API (src/gpu/chr.cu:13-99,
// src/gpu/dmatrix.cu, src/gpu/dvector.cu of quothbonney/naja) restated on
// plain pointers: argument checks raise the reference's error classes as
// status codes, CUDA failures are never swallowed (the reference's
// CUDA_CHECK only prints, src/gpu/helper.h:12-18), and every entry point
// records a thread-local message.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/naja_chr.h"
#include "capi_internal.cuh"
#include "chr.cuh"
#include "common.cuh"

namespace naja {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int ptr_location(const void* p) {
  if (!p) return 0;
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  if (attr.type == cudaMemoryTypeManaged) return 1;
  if (attr.type != cudaMemoryTypeDevice) return 0;
  int cur = -1;
  if (cudaGetDevice(&cur) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return attr.device == cur ? 1 : -1;
}

bool is_device_ptr(const void* p) { return ptr_location(p) != 0; }

int require_local(const char* fn, std::initializer_list<const void*> ptrs) {
  int k = 0;
  for (const void* p : ptrs) {
    if (ptr_location(p) < 0)
      return fail(NAJA_ERR_INVALID_ARGUMENT, std::string(fn) + ": pointer argument " + std::to_string(k) +
                                                 " is device memory of another GPU than the one the call runs on");
    ++k;
  }
  return NAJA_OK;
}

DeviceGuard::DeviceGuard(int device) {
  cudaGetDevice(&prev_);
  if (device >= 0 && device != prev_) {
    ok_ = cudaSetDevice(device) == cudaSuccess;
    switched_ = true;
  }
}
DeviceGuard::~DeviceGuard() {
  if (switched_) cudaSetDevice(prev_);
}

namespace {

__global__ void pad_convert_kernel(const double* __restrict__ src, long long lds, double* __restrict__ A64,
                                   float* __restrict__ A32, int m, int d, int lda) {
  const long long n = static_cast<long long>(lda) * d;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(i % lda);
    const long long c = i / lda;
    const double v = (r < m) ? src[c * lds + r] : 0.0;
    A64[i] = v;
    A32[i] = __double2float_rn(v);
  }
}

constexpr unsigned long long kWaitTimeoutNs = 5ull * 1000ull * 1000ull * 1000ull;

const char* dev_error_name(int code) {
  switch (code) {
    case kDevTimeoutFull: return "a consumer warp timed out waiting for a staged column";
    case kDevTimeoutEmpty: return "the producer timed out waiting for a free slot";
    case kDevTimeoutDrain: return "the exit path timed out draining its bulk copies";
    case kDevBadPair: return "pair schedule index outside [0, d)";
    case kDevTimeoutCluster: return "a CTA of a chain's cluster timed out waiting for its peers";
    default: return "unknown device error";
  }
}

// Reads (and clears) the error word of a finished launch.
int read_device_error(int* err) {
  int w[4] = {0, 0, 0, 0};
  cudaError_t e = cudaMemcpy(w, err, sizeof(w), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("reading the device error word: ") + cudaGetErrorString(e));
  if (w[0] == 0) return NAJA_OK;
  cudaMemset(err, 0, sizeof(w));
  return fail(NAJA_ERR_DEVICE, std::string("device error: ") + dev_error_name(w[0]) + " (" + std::to_string(w[1]) +
                                   ", " + std::to_string(w[2]) + ", " + std::to_string(w[3]) + ")");
}

}  // namespace

// Scoped stream-ordered device buffer; staged copies of host arguments.
DeviceBuffer::~DeviceBuffer() {
  if (ptr) cudaFreeAsync(ptr, stream);
}
int DeviceBuffer::alloc(size_t nbytes, cudaStream_t s) {
  stream = s;
  bytes = nbytes;
  if (nbytes == 0) return NAJA_OK;
  cudaError_t e = cudaMallocAsync(&ptr, nbytes, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    ptr = nullptr;
    return fail(NAJA_ERR_NO_MEMORY, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
  }
  return NAJA_OK;
}

// Returns a device view of `p` (n bytes): itself if already on the device,
// else a staged copy in `buf`.
int device_view(const void* p, size_t n, cudaStream_t s, DeviceBuffer& buf, const void** out) {
  if (!p || is_device_ptr(p)) {
    *out = p;
    return NAJA_OK;
  }
  int st = buf.alloc(n, s);
  if (st) return st;
  cudaError_t e = cudaMemcpyAsync(buf.ptr, p, n, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("cudaMemcpyAsync H2D: ") + cudaGetErrorString(e));
  *out = buf.ptr;
  return NAJA_OK;
}

}  // namespace naja

using namespace naja;

// Compressed copies of A for the sparse-column kernel, built on the first
// run that may use them.
struct SparseStore {
  bool built = false;
  long long nnz = 0;        // nonzeros of the FP64 A
  long long tot32 = 0, tot64 = 0;  // column entries stored, padding included
  void* cols32 = nullptr;   // (float, int) entries of A32 by columns
  int* cs32 = nullptr;
  int max32 = 0;
  void* cols64 = nullptr;   // (double, int, pad) entries of A64 by columns
  int* cs64 = nullptr;
  int max64 = 0;
  int* row_start = nullptr; // A64 by rows, (value, column) entries in groups of kSpRowGroup
  void* row_ent = nullptr;
};

struct naja_polytope {
  int device = 0;
  int m = 0, d = 0, lda = 0;
  double* A64 = nullptr;
  float* A32 = nullptr;
  double* b = nullptr;
  int* err = nullptr;
  std::mutex sparse_mu;
  SparseStore sp;
};

namespace naja {
int polytope_device(const naja_polytope* P) { return P ? P->device : 0; }
}  // namespace naja

namespace sparse_build {

void free_sparse(SparseStore& s) {
  cudaFree(s.cols32);
  cudaFree(s.cs32);
  cudaFree(s.cols64);
  cudaFree(s.cs64);
  cudaFree(s.row_start);
  cudaFree(s.row_ent);
  s = SparseStore();
}

struct SpE32 {
  float v;
  int r;
};
struct __align__(16) SpE64 {
  double v;
  int r;
  int pad;
};
static_assert(sizeof(SpE32) == kSpEntryBytes32 && sizeof(SpE64) == kSpEntryBytes64, "entry layout");

// Entries a compressed column of n nonzeros stores: FP32 entries come in
// pairs (16 bytes), every column holds at least one 16-byte group.
inline int padded32(int n) { return n < 2 ? 2 : n + (n & 1); }
inline int padded64(int n) { return n < 1 ? 1 : n; }

// One warp per column: nonzeros of the FP32 and FP64 column, and per row
// the FP64 nonzeros (for the row offsets).
__global__ void sp_count_kernel(const double* A64, const float* A32, int m, int d, int lda, int* cnt32, int* cnt64,
                                int* rowcnt) {
  const int j = static_cast<int>((blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (j >= d) return;
  const double* c64 = A64 + static_cast<size_t>(j) * lda;
  const float* c32 = A32 + static_cast<size_t>(j) * lda;
  int n32 = 0, n64 = 0;
  for (int r0 = 0; r0 < m; r0 += 32) {
    const int r = r0 + lane;
    const bool nz64 = r < m && c64[r] != 0.0;
    const bool nz32 = r < m && c32[r] != 0.0f;
    n64 += __popc(__ballot_sync(0xffffffffu, nz64));
    n32 += __popc(__ballot_sync(0xffffffffu, nz32));
    if (nz64) atomicAdd(&rowcnt[r], 1);
  }
  if (lane == 0) {
    cnt32[j] = n32;
    cnt64[j] = n64;
  }
}

// One warp per column: the nonzeros in row order (ballot compaction), then
// the (0, m) padding.
__global__ void sp_fill_cols_kernel(const double* A64, const float* A32, int m, int d, int lda, const int* cs32,
                                    const int* cs64, SpE32* cols32, SpE64* cols64) {
  const int j = static_cast<int>((blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (j >= d) return;
  const double* c64 = A64 + static_cast<size_t>(j) * lda;
  const float* c32 = A32 + static_cast<size_t>(j) * lda;
  const unsigned lt = (1u << lane) - 1u;
  int p32 = cs32[j], p64 = cs64[j];
  for (int r0 = 0; r0 < m; r0 += 32) {
    const int r = r0 + lane;
    const double v64 = r < m ? c64[r] : 0.0;
    const float v32 = r < m ? c32[r] : 0.0f;
    const unsigned b64 = __ballot_sync(0xffffffffu, v64 != 0.0);
    const unsigned b32 = __ballot_sync(0xffffffffu, v32 != 0.0f);
    if (v64 != 0.0) cols64[p64 + __popc(b64 & lt)] = SpE64{v64, r, 0};
    if (v32 != 0.0f) cols32[p32 + __popc(b32 & lt)] = SpE32{v32, r};
    p64 += __popc(b64);
    p32 += __popc(b32);
  }
  for (int q = p32 + lane; q < cs32[j + 1]; q += 32) cols32[q] = SpE32{0.0f, m};
  for (int q = p64 + lane; q < cs64[j + 1]; q += 32) cols64[q] = SpE64{0.0, m, 0};
}

// One warp per row: the FP64 nonzeros in column order, then (0, 0)
// padding to the row's group boundary.
__global__ void sp_fill_rows_kernel(const double* A64, int m, int d, int lda, const int* row_start, SpE64* row_ent) {
  const int r = static_cast<int>((blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (r >= m) return;
  const unsigned lt = (1u << lane) - 1u;
  int p = row_start[r];
  for (int j0 = 0; j0 < d; j0 += 32) {
    const int j = j0 + lane;
    const double v = j < d ? A64[r + static_cast<size_t>(j) * lda] : 0.0;
    const unsigned bm = __ballot_sync(0xffffffffu, v != 0.0);
    if (v != 0.0) row_ent[p + __popc(bm & lt)] = SpE64{v, j, 0};
    p += __popc(bm);
  }
  for (int q = p + lane; q < row_start[r + 1]; q += 32) row_ent[q] = SpE64{0.0, 0, 0};
}

// Builds the compressed columns of both tiers (entries where the tier's A
// is nonzero, rows ascending, padded with (0, m) entries to 16 bytes) and
// the FP64 rows (columns ascending) from the device copies of A: counts on
// the device, offsets on the host, entries filled by ballot compaction.
int build_sparse(naja_polytope* P) {
  SparseStore& S = P->sp;
  const int m = P->m, d = P->d, lda = P->lda;
  int* cnt = nullptr;  // cnt32[d], cnt64[d], rowcnt[m]
  cudaError_t e = cudaMalloc(&cnt, (2 * static_cast<size_t>(d) + m) * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(cnt, 0, (2 * static_cast<size_t>(d) + m) * sizeof(int));
  const int col_blocks = (d + 7) / 8, row_blocks = (m + 7) / 8;
  if (e == cudaSuccess) {
    sp_count_kernel<<<col_blocks, 256>>>(P->A64, P->A32, m, d, lda, cnt, cnt + d, cnt + 2 * d);
    e = cudaGetLastError();
  }
  std::vector<int> h(2 * static_cast<size_t>(d) + m);
  if (e == cudaSuccess) e = cudaMemcpy(h.data(), cnt, h.size() * sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(cnt);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(NAJA_ERR_CUDA, std::string("building compressed columns: ") + cudaGetErrorString(e));
  }
  std::vector<int> cs32(d + 1), cs64(d + 1), rs(m + 1);
  long long t32 = 0, t64 = 0, nnz = 0;
  int max32 = 0, max64 = 0;
  for (int j = 0; j < d; ++j) {
    cs32[j] = static_cast<int>(t32);
    cs64[j] = static_cast<int>(t64);
    const int p32 = padded32(h[j]), p64 = padded64(h[d + j]);
    t32 += p32;
    t64 += p64;
    max32 = std::max(max32, p32);
    max64 = std::max(max64, p64);
    if (t32 > (1LL << 30) || t64 > (1LL << 30))
      return fail(NAJA_ERR_UNSUPPORTED, "building compressed columns: too many nonzeros");
  }
  cs32[d] = static_cast<int>(t32);
  cs64[d] = static_cast<int>(t64);
  long long nrow = 0;  // row entries, padding included
  for (int r = 0; r < m; ++r) {
    rs[r] = static_cast<int>(nrow);
    nnz += h[2 * d + r];
    nrow += (h[2 * d + r] + kSpRowGroup - 1) / kSpRowGroup * kSpRowGroup;
    if (nrow > (1LL << 30)) return fail(NAJA_ERR_UNSUPPORTED, "building compressed rows: too many nonzeros");
  }
  rs[m] = static_cast<int>(nrow);
  e = cudaMalloc(&S.cols32, static_cast<size_t>(t32) * sizeof(SpE32));
  if (e == cudaSuccess) e = cudaMalloc(&S.cols64, static_cast<size_t>(t64) * sizeof(SpE64));
  if (e == cudaSuccess) e = cudaMalloc(&S.cs32, (d + 1) * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&S.cs64, (d + 1) * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&S.row_start, (m + 1) * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&S.row_ent, std::max<long long>(nrow, 1) * sizeof(SpE64));
  if (e == cudaSuccess) e = cudaMemcpy(S.cs32, cs32.data(), (d + 1) * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(S.cs64, cs64.data(), (d + 1) * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(S.row_start, rs.data(), (m + 1) * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    sp_fill_cols_kernel<<<col_blocks, 256>>>(P->A64, P->A32, m, d, lda, S.cs32, S.cs64,
                                             static_cast<SpE32*>(S.cols32), static_cast<SpE64*>(S.cols64));
    sp_fill_rows_kernel<<<row_blocks, 256>>>(P->A64, m, d, lda, S.row_start, static_cast<SpE64*>(S.row_ent));
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    cudaGetLastError();
    free_sparse(S);
    return fail(NAJA_ERR_NO_MEMORY, std::string("building compressed columns: ") + cudaGetErrorString(e));
  }
  S.max32 = max32;
  S.max64 = max64;
  S.tot32 = t32;
  S.tot64 = t64;
  S.nnz = nnz;
  S.built = true;
  return NAJA_OK;
}

}  // namespace sparse_build

namespace {
// Picks the step kernel and its launch configuration for a run (the same
// choice for naja_chr_run and naja_chr_kernel_choice).  Compressed columns:
// forced, or automatic when the columns are at most a quarter full on
// average and the chain's state fits on chip.  Results are the same either
// way.
int choose_kernel(const naja_polytope* P, const naja_chr_params* p, ChrLaunchConfig* cfg, SpArgs* spa,
                  bool* use_sparse) {
  if (p->cluster < 0 || p->cluster > 8)
    return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_chr_run: cluster must be 0 (automatic) or 1..8");
  if (p->sparse < NAJA_SPARSE_AUTO || p->sparse > NAJA_SPARSE_COLUMNS)
    return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_chr_run: unknown sparse mode");
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, P->device);
  // carried MRG states are read and written by one CTA per chain
  const int cluster_req = p->rng_state ? 1 : p->cluster;
  std::memset(spa, 0, sizeof(*spa));
  *use_sparse = false;
  int st = NAJA_OK;
  // automatic: only when the thread count is automatic too
  const bool tpb_ok = p->tpb <= 0 || (p->sparse == NAJA_SPARSE_COLUMNS &&
                                      (p->tpb == 32 || p->tpb == 64 || p->tpb == 128 || p->tpb == 256 ||
                                       p->tpb == 512));
  const bool sparse_shape = p->ksparse_prob <= 0.0 && cluster_req <= 1 && tpb_ok;
  if (p->sparse == NAJA_SPARSE_COLUMNS && !sparse_shape)
    return fail(NAJA_ERR_UNSUPPORTED, "naja_chr_run: compressed columns need ksparse_prob = 0, one CTA per chain "
                                      "and tpb 0, 32, 64, 128, 256 or 512");
  if (p->sparse != NAJA_SPARSE_DENSE && sparse_shape) {
    naja_polytope* Pm = const_cast<naja_polytope*>(P);
    std::lock_guard<std::mutex> lock(Pm->sparse_mu);
    if (!Pm->sp.built && (st = sparse_build::build_sparse(Pm))) return st;
    const SparseStore& S = Pm->sp;
    const bool f64 = p->precision == NAJA_PREC_FP64;
    const int max_col = f64 ? S.max64 : S.max32;
    const long long tot = f64 ? S.tot64 : S.tot32;
    if (p->sparse == NAJA_SPARSE_COLUMNS || 4 * tot <= static_cast<long long>(P->m) * P->d) {
      st = chr_sparse_plan(p->precision, P->m, P->d, max_col, static_cast<double>(tot) / P->d, p->tpb,
                           p->max_slots, cfg);
      if (st == NAJA_OK) {
        *use_sparse = true;
        spa->cols = f64 ? S.cols64 : S.cols32;
        spa->col_start = f64 ? S.cs64 : S.cs32;
        spa->row_start = S.row_start;
        spa->row_ent = S.row_ent;
        return NAJA_OK;
      }
      if (p->sparse == NAJA_SPARSE_COLUMNS)
        return fail(st, "naja_chr_run: the compressed columns' state (m=" + std::to_string(P->m) + ", d=" +
                            std::to_string(P->d) + ") does not fit in shared memory");
    }
  }
  st = chr_plan(p->precision, P->m, P->d, P->lda, p->tpb, p->max_slots, p->nchains, cluster_req, sms, cfg);
  if (st == NAJA_ERR_INVALID_ARGUMENT) return fail(st, "Invalid threads per block");
  if (st) return fail(st, "CoordinateHitAndRun: shape (m=" + std::to_string(P->m) + ", d=" + std::to_string(P->d) +
                              ") exceeds the step kernel's capacity for this thread count");
  return NAJA_OK;
}
}  // namespace

extern "C" {

const char* naja_last_error(void) { return g_last_error.c_str(); }

const char* naja_version(void) { return "naja_b200 0.1 (sm_100a)"; }

size_t naja_mrg_state_bytes(void) { return mrg_state_bytes(); }

void naja_chr_params_default(naja_chr_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->thinning = 1;
  p->tpb = 0;
  p->ksparse_k = 8;
  p->pair_mode = 1;
  p->precision = NAJA_PREC_FP32;
  p->rng = NAJA_RNG_PHILOX;
  p->out_dtype = NAJA_DTYPE_F32;
}

int naja_polytope_create(int device, int m, int d, const double* A, int lda, const double* b,
                         naja_polytope** out) {
  if (!out) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_polytope_create: out is null");
  *out = nullptr;
  if (m <= 0 || d <= 0) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_polytope_create: empty polytope");
  if (!A || !b) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_polytope_create: A or b is null");
  if (lda < m) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_polytope_create: lda < m");
  DeviceGuard g(device);
  if (!g.ok()) return fail(NAJA_ERR_CUDA, "naja_polytope_create: cannot select device");
  if (int st = require_local("naja_polytope_create", {A, b})) return st;
  naja_polytope* P = new naja_polytope();
  P->device = device;
  P->m = m;
  P->d = d;
  P->lda = (m + 31) / 32 * 32;
  const size_t n = static_cast<size_t>(P->lda) * d;
  cudaError_t e = cudaMalloc(&P->A64, n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&P->A32, n * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&P->b, m * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&P->err, 4 * sizeof(int));
  if (e != cudaSuccess) {
    cudaGetLastError();
    naja_polytope_destroy(P);
    return fail(NAJA_ERR_NO_MEMORY, std::string("naja_polytope_create: ") + cudaGetErrorString(e));
  }
  const double* src = A;
  double* staged = nullptr;
  if (!is_device_ptr(A)) {
    e = cudaMalloc(&staged, static_cast<size_t>(lda) * d * sizeof(double));
    if (e == cudaSuccess)
      e = cudaMemcpy(staged, A, static_cast<size_t>(lda) * d * sizeof(double), cudaMemcpyHostToDevice);
    src = staged;
  }
  if (e == cudaSuccess) {
    const long long total = static_cast<long long>(P->lda) * d;
    const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 148LL * 16));
    pad_convert_kernel<<<blocks, 256>>>(src, lda, P->A64, P->A32, m, d, P->lda);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpy(P->b, b, m * sizeof(double), is_device_ptr(b) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(P->err, 0, 4 * sizeof(int));
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (staged) cudaFree(staged);
  if (e != cudaSuccess) {
    naja_polytope_destroy(P);
    return fail(NAJA_ERR_CUDA, std::string("naja_polytope_create: ") + cudaGetErrorString(e));
  }
  *out = P;
  return NAJA_OK;
}

int naja_polytope_destroy(naja_polytope* P) {
  if (!P) return NAJA_OK;
  DeviceGuard g(P->device);
  cudaFree(P->A64);
  cudaFree(P->A32);
  cudaFree(P->b);
  cudaFree(P->err);
  sparse_build::free_sparse(P->sp);
  delete P;
  return NAJA_OK;
}

int naja_polytope_shape(const naja_polytope* P, int* m, int* d) {
  if (!P) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_polytope_shape: null polytope");
  if (m) *m = P->m;
  if (d) *d = P->d;
  return NAJA_OK;
}

int naja_polytope_check(const naja_polytope* P) {
  if (!P) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_polytope_check: null polytope");
  DeviceGuard g(P->device);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("naja_polytope_check: ") + cudaGetErrorString(e));
  return read_device_error(P->err);
}

int naja_chr_kernel_choice(const naja_polytope* P, const naja_chr_params* p, int* sparse_kernel, int* threads,
                           int* slots, size_t* smem) {
  if (!P || !p) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_chr_kernel_choice: null polytope or params");
  DeviceGuard g(P->device);
  if (!g.ok()) return fail(NAJA_ERR_CUDA, "naja_chr_kernel_choice: cannot select device");
  ChrLaunchConfig cfg;
  SpArgs spa;
  bool use_sparse = false;
  const int st = choose_kernel(P, p, &cfg, &spa, &use_sparse);
  if (st) return st;
  if (sparse_kernel) *sparse_kernel = use_sparse ? 1 : 0;
  if (threads) *threads = cfg.threads;
  if (slots) *slots = cfg.slots;
  if (smem) *smem = cfg.smem;
  return NAJA_OK;
}

int naja_chr_run(const naja_polytope* P, const naja_chr_params* p, const double* X0, int ldx, void* samples,
                 double* X_final, void* stream_ptr) {
  if (!P || !p) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_chr_run: null polytope or params");
  if (p->nchains <= 0) return fail(NAJA_ERR_INVALID_ARGUMENT, "CoordinateHitAndRun: nchains must be positive");
  if (p->nspc <= 0) return fail(NAJA_ERR_INVALID_ARGUMENT, "CoordinateHitAndRun: nspc must be positive");
  if (p->thinning <= 0) return fail(NAJA_ERR_INVALID_ARGUMENT, "CoordinateHitAndRun: thinning must be positive");
  if (!X0 || !samples) return fail(NAJA_ERR_INVALID_ARGUMENT, "CoordinateHitAndRun: X0 or samples is null");
  if (ldx < P->d) return fail(NAJA_ERR_INVALID_ARGUMENT, "CoordinateHitAndRun: ldx < d");
  if (p->precision != NAJA_PREC_FP32 && p->precision != NAJA_PREC_FP64)
    return fail(NAJA_ERR_INVALID_ARGUMENT, "CoordinateHitAndRun: unknown precision");
  if (p->rng != NAJA_RNG_PHILOX && p->rng != NAJA_RNG_REF_MRG)
    return fail(NAJA_ERR_INVALID_ARGUMENT, "CoordinateHitAndRun: unknown rng");
  if (p->out_dtype != NAJA_DTYPE_F32 && p->out_dtype != NAJA_DTYPE_F64)
    return fail(NAJA_ERR_INVALID_ARGUMENT, "CoordinateHitAndRun: unknown output dtype");
  if (p->resync_interval < 0) return fail(NAJA_ERR_INVALID_ARGUMENT, "CoordinateHitAndRun: resync_interval < 0");
  if (p->chain_base < 0) return fail(NAJA_ERR_INVALID_ARGUMENT, "CoordinateHitAndRun: chain_base < 0");
  const int out_nchains = p->out_nchains > 0 ? p->out_nchains : p->nchains;
  if (out_nchains < p->chain_base + p->nchains)
    return fail(NAJA_ERR_INVALID_ARGUMENT, "CoordinateHitAndRun: out_nchains < chain_base + nchains");
  if (p->pair_mode == 2 && p->pair_prob > 0.0 && p->n_pairs > 0 &&
      (!p->pair_i || !p->pair_j || !p->pair_c || !p->pair_s))
    return fail(NAJA_ERR_INVALID_ARGUMENT, "CoordinateHitAndRun: pair schedule arrays missing");
  if (static_cast<long long>(p->nspc) * p->thinning > (1LL << 62))
    return fail(NAJA_ERR_INVALID_ARGUMENT, "CoordinateHitAndRun: too many steps");

  DeviceGuard g(P->device);
  if (!g.ok()) return fail(NAJA_ERR_CUDA, "naja_chr_run: cannot select device");
  if (int st = require_local("CoordinateHitAndRun", {X0, samples, X_final, p->pair_i, p->pair_j, p->pair_c,
                                                      p->pair_s, p->rng_state, p->wait_cycles, p->slack_final}))
    return st;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);

  ChrLaunchConfig cfg;
  SpArgs spa;
  bool use_sparse = false;
  int st = choose_kernel(P, p, &cfg, &spa, &use_sparse);
  if (st) return st;

  const int d = P->d;
  const size_t out_elt = p->out_dtype == NAJA_DTYPE_F64 ? 8 : 4;
  const size_t out_bytes = static_cast<size_t>(p->nspc) * out_nchains * d * out_elt;
  const size_t x_bytes = static_cast<size_t>(ldx) * (p->nchains - 1) * sizeof(double) + d * sizeof(double);

  DeviceBuffer bx0, bout, bxf, bpi, bpj, bpc, bps, bsf;
  const void* dX0 = nullptr;
  if ((st = device_view(X0, x_bytes, stream, bx0, &dX0))) return st;
  void* dout = samples;
  const bool host_out = !is_device_ptr(samples);
  if (host_out) {
    if ((st = bout.alloc(out_bytes, stream))) return st;
    dout = bout.ptr;
    if (out_nchains != p->nchains) {
      // rows of other chains are left as the caller had them
      cudaError_t e = cudaMemcpyAsync(dout, samples, out_bytes, cudaMemcpyHostToDevice, stream);
      if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("cudaMemcpyAsync: ") + cudaGetErrorString(e));
    }
  }
  double* dxf = X_final;
  const bool host_xf = X_final && !is_device_ptr(X_final);
  if (host_xf) {
    if ((st = bxf.alloc(x_bytes, stream))) return st;
    dxf = static_cast<double*>(bxf.ptr);
  }
  if (p->slack_final && cfg.cluster > 1)
    return fail(NAJA_ERR_UNSUPPORTED, "CoordinateHitAndRun: slack_final needs one CTA per chain (cluster <= 1)");
  const size_t sf_bytes = static_cast<size_t>(p->nchains) * P->m * (p->precision == NAJA_PREC_FP64 ? 8 : 4);
  void* dsf = p->slack_final;
  const bool host_sf = p->slack_final && !is_device_ptr(p->slack_final);
  if (host_sf) {
    if ((st = bsf.alloc(sf_bytes, stream))) return st;
    dsf = bsf.ptr;
  }
  const void *dpi = nullptr, *dpj = nullptr, *dpc = nullptr, *dps = nullptr;
  if (p->n_pairs > 0) {
    const size_t ni = static_cast<size_t>(p->n_pairs) * sizeof(int), nd = static_cast<size_t>(p->n_pairs) * 8;
    if ((st = device_view(p->pair_i, ni, stream, bpi, &dpi))) return st;
    if ((st = device_view(p->pair_j, ni, stream, bpj, &dpj))) return st;
    if ((st = device_view(p->pair_c, nd, stream, bpc, &dpc))) return st;
    if ((st = device_view(p->pair_s, nd, stream, bps, &dps))) return st;
  }

  ChrArgs a;
  std::memset(&a, 0, sizeof(a));
  a.A32 = P->A32;
  a.A64 = P->A64;
  a.lda = P->lda;
  a.b = P->b;
  a.m = P->m;
  a.d = d;
  a.X0 = static_cast<const double*>(dX0);
  a.ldx = ldx;
  a.X_final = dxf;
  a.samples = dout;
  a.out_f64 = p->out_dtype == NAJA_DTYPE_F64;
  a.out_nchains = out_nchains;
  a.chain_base = p->chain_base;
  a.nspc = p->nspc;
  a.thinning = p->thinning;
  a.step_offset = p->step_offset;
  a.seed = p->seed;
  a.pair_prob = p->pair_prob;
  a.ksparse_prob = p->ksparse_prob;
  a.ksparse_k = p->ksparse_k;
  a.pair_mode = p->pair_mode;
  a.pair_i = static_cast<const int*>(dpi);
  a.pair_j = static_cast<const int*>(dpj);
  a.pair_c = static_cast<const double*>(dpc);
  a.pair_s = static_cast<const double*>(dps);
  a.n_pairs = p->n_pairs;
  a.resync = p->resync_interval;
  a.rng = p->rng;
  a.rng_state = p->rng_state;
  a.err = P->err;
  a.timeout_ns = kWaitTimeoutNs;
  a.wait_cycles = p->wait_cycles;
  a.slack_final = dsf;

  const long long total_steps = static_cast<long long>(p->nspc) * p->thinning;
  const bool segments =
      chr_use_segments(P->m, d, p->resync_interval, total_steps, cfg.cluster, p->wait_cycles != nullptr);
  if (segments)
    st = chr_run_segmented(p->precision, a, p->nchains, cfg, stream, nullptr, use_sparse ? &spa : nullptr);
  else if (use_sparse)
    st = chr_sparse_launch(p->precision, a, spa, p->nchains, cfg, stream);
  else
    st = chr_launch(p->precision, a, p->nchains, cfg, stream);
  if (st) {
    cudaError_t e = cudaGetLastError();
    return fail(st, std::string("CoordinateHitAndRun: launch failed: ") + cudaGetErrorString(e));
  }
  if (host_out || host_xf || host_sf) {
    cudaError_t e = cudaSuccess;
    if (host_out) e = cudaMemcpyAsync(samples, dout, out_bytes, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && host_xf) e = cudaMemcpyAsync(X_final, dxf, x_bytes, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && host_sf) e = cudaMemcpyAsync(p->slack_final, dsf, sf_bytes, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("CoordinateHitAndRun: ") + cudaGetErrorString(e));
    if ((st = read_device_error(P->err))) return st;
  }
  return NAJA_OK;
}

int naja_mrg_init_states(int device, unsigned long long seed, int chain_base, int nchains, void* states) {
  if (nchains <= 0 || !states) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_mrg_init_states: bad arguments");
  DeviceGuard g(device);
  if (!is_device_ptr(states)) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_mrg_init_states: states must be device memory");
  if (int st = require_local("naja_mrg_init_states", {states})) return st;
  int st = mrg_init_states(seed, chain_base, nchains, states, 0);
  if (st) return fail(st, "naja_mrg_init_states: launch failed");
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("naja_mrg_init_states: ") + cudaGetErrorString(e));
  return NAJA_OK;
}

int naja_mrg_tape(int device, unsigned long long seed, int chain_base, int nchains, long long count, double* tape) {
  if (nchains <= 0 || count <= 0 || !tape) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_mrg_tape: bad arguments");
  DeviceGuard g(device);
  if (int st = require_local("naja_mrg_tape", {tape})) return st;
  DeviceBuffer buf;
  void* dt = tape;
  const size_t bytes = static_cast<size_t>(nchains) * count * sizeof(double);
  const bool host = !is_device_ptr(tape);
  int st;
  if (host) {
    if ((st = buf.alloc(bytes, 0))) return st;
    dt = buf.ptr;
  }
  st = mrg_tape(seed, chain_base, nchains, static_cast<long>(count), static_cast<double*>(dt), 0);
  if (st) return fail(st, "naja_mrg_tape: launch failed");
  cudaError_t e = cudaSuccess;
  if (host) e = cudaMemcpy(tape, dt, bytes, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("naja_mrg_tape: ") + cudaGetErrorString(e));
  return NAJA_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ batches
namespace {

struct BatchPrep {
  ChrArgs base;
  BatchConfig cfg;
  std::vector<ModelDesc> descs;
  std::vector<int> item_model, item_chain;
  int device = 0;
};

// Builds every model's compressed columns (once per polytope) and records
// the longest FP32 column for a compressed-column batch.
int batch_sparse_prepare(int nmodels, const naja_polytope* const* models, BatchConfig* cfg) {
  int max_col = 0;
  for (int k = 0; k < nmodels; ++k) {
    naja_polytope* Pm = const_cast<naja_polytope*>(models[k]);
    if (!Pm) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_chr_run_batched: null model");
    std::lock_guard<std::mutex> lock(Pm->sparse_mu);
    DeviceGuard g(Pm->device);
    int st = NAJA_OK;
    if (!Pm->sp.built && (st = sparse_build::build_sparse(Pm))) return st;
    max_col = std::max(max_col, Pm->sp.max32);
  }
  cfg->sparse = 1;
  cfg->max_col = max_col;
  return NAJA_OK;
}

int prep_batch(int nmodels, const naja_polytope* const* models, const naja_chr_params* p, const double* const* X0s,
               int ldx, void* const* samples, double* const* X_finals, unsigned long long seed_stride,
               const naja_batch_config* c, BatchPrep* out) {
  if (nmodels <= 0 || !models || !p || !X0s || !samples || !c)
    return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_chr_run_batched: null or empty argument");
  if (p->nchains <= 0 || p->nspc <= 0 || p->thinning <= 0)
    return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_chr_run_batched: nchains, nspc and thinning must be positive");
  if (p->precision != NAJA_PREC_FP32)
    return fail(NAJA_ERR_UNSUPPORTED, "naja_chr_run_batched: the batched kernel runs the FP32 tier");
  if (p->rng != NAJA_RNG_PHILOX && p->rng != NAJA_RNG_REF_MRG)
    return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_chr_run_batched: unknown rng");
  if (p->rng_state) return fail(NAJA_ERR_UNSUPPORTED, "naja_chr_run_batched: carried MRG states are not supported");
  if (p->out_dtype != NAJA_DTYPE_F32 && p->out_dtype != NAJA_DTYPE_F64)
    return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_chr_run_batched: unknown output dtype");
  if (p->n_pairs > 0 && (!is_device_ptr(p->pair_i) || !is_device_ptr(p->pair_j) || !is_device_ptr(p->pair_c) ||
                         !is_device_ptr(p->pair_s)))
    return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_chr_run_batched: the pair schedule must be device memory");
  const int d = models[0] ? models[0]->d : 0;
  int lda_max = 0, m_max = 0;
  for (int k = 0; k < nmodels; ++k) {
    const naja_polytope* P = models[k];
    if (!P) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_chr_run_batched: null model");
    if (P->d != d) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_chr_run_batched: models differ in d");
    if (P->device != models[0]->device) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_chr_run_batched: models on different devices");
    if (!X0s[k] || !samples[k] || !is_device_ptr(X0s[k]) || !is_device_ptr(samples[k]))
      return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_chr_run_batched: X0s and samples must be device pointers");
    if (X_finals && X_finals[k] && !is_device_ptr(X_finals[k]))
      return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_chr_run_batched: X_finals must be device pointers");
    lda_max = std::max(lda_max, P->lda);
    m_max = std::max(m_max, P->m);
  }
  if (ldx < d) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_chr_run_batched: ldx < d");
  {
    DeviceGuard g(models[0]->device);
    if (int st = require_local("naja_chr_run_batched", {p->pair_i, p->pair_j, p->pair_c, p->pair_s})) return st;
    for (int k = 0; k < nmodels; ++k)
      if (int st = require_local("naja_chr_run_batched (X0s[k], samples[k], X_finals[k])",
                                 {X0s[k], samples[k], X_finals ? X_finals[k] : nullptr}))
        return st;
  }
  BatchConfig cfg;
  std::memset(&cfg, 0, sizeof(cfg));
  cfg.threads = c->threads;
  cfg.slots = c->slots;
  cfg.slack_smem = c->slack_smem;
  cfg.ctas_per_sm = c->ctas_per_sm;
  int st = NAJA_OK;
  if (c->sparse) {
    if (p->ksparse_prob > 0.0)
      return fail(NAJA_ERR_UNSUPPORTED, "naja_chr_run_batched: compressed columns need ksparse_prob = 0");
    if ((st = batch_sparse_prepare(nmodels, models, &cfg))) return st;
  }
  st = chr_batch_plan(m_max, d, lda_max, &cfg);
  if (st == NAJA_ERR_INVALID_ARGUMENT) return fail(st, "naja_chr_run_batched: bad batch configuration");
  if (st) return fail(st, "naja_chr_run_batched: configuration cannot hold models of " + std::to_string(m_max) + " rows");
  ChrArgs& a = out->base;
  std::memset(&a, 0, sizeof(a));
  a.d = d;
  a.lda = lda_max;
  a.out_f64 = p->out_dtype == NAJA_DTYPE_F64;
  a.out_nchains = p->nchains;
  a.nspc = p->nspc;
  a.thinning = p->thinning;
  a.step_offset = p->step_offset;
  a.pair_prob = p->pair_prob;
  a.ksparse_prob = p->ksparse_prob;
  a.ksparse_k = p->ksparse_k;
  a.pair_mode = p->pair_mode;
  a.pair_i = p->pair_i;
  a.pair_j = p->pair_j;
  a.pair_c = p->pair_c;
  a.pair_s = p->pair_s;
  a.n_pairs = p->n_pairs;
  a.resync = p->resync_interval;
  a.rng = p->rng;
  a.err = models[0]->err;
  a.timeout_ns = kWaitTimeoutNs;
  out->cfg = cfg;
  out->device = models[0]->device;
  out->descs.resize(nmodels);
  for (int k = 0; k < nmodels; ++k) {
    const naja_polytope* P = models[k];
    ModelDesc& m = out->descs[k];
    m.A32 = P->A32;
    m.A64 = P->A64;
    m.lda = P->lda;
    m.m = P->m;
    m.b = P->b;
    m.X0 = X0s[k];
    m.ldx = ldx;
    m.samples = samples[k];
    m.X_final = X_finals ? X_finals[k] : nullptr;
    m.seed = p->seed + static_cast<unsigned long long>(k) * seed_stride;
    std::memset(&m.sp, 0, sizeof(m.sp));
    if (cfg.sparse) {
      m.sp.cols = P->sp.cols32;
      m.sp.col_start = P->sp.cs32;
      m.sp.row_start = P->sp.row_start;
      m.sp.row_ent = P->sp.row_ent;
    }
  }
  // chains of different models interleave, so resident CTAs spread over models
  for (int ch = 0; ch < p->nchains; ++ch)
    for (int k = 0; k < nmodels; ++k) {
      out->item_model.push_back(k);
      out->item_chain.push_back(ch);
    }
  return NAJA_OK;
}

size_t batch_bytes(const BatchPrep& b) {
  return b.descs.size() * sizeof(ModelDesc) + 2 * b.item_model.size() * sizeof(int) + 64;
}

void batch_pack(const BatchPrep& b, std::vector<unsigned char>& host, void* dev, const ModelDesc** dm, const int** im,
                const int** ic) {
  host.assign(batch_bytes(b), 0);
  size_t off = 0;
  std::memcpy(host.data(), b.descs.data(), b.descs.size() * sizeof(ModelDesc));
  *dm = reinterpret_cast<const ModelDesc*>(static_cast<char*>(dev) + off);
  off += (b.descs.size() * sizeof(ModelDesc) + 15) / 16 * 16;
  std::memcpy(host.data() + off, b.item_model.data(), b.item_model.size() * sizeof(int));
  *im = reinterpret_cast<const int*>(static_cast<char*>(dev) + off);
  off += b.item_model.size() * sizeof(int);
  std::memcpy(host.data() + off, b.item_chain.data(), b.item_chain.size() * sizeof(int));
  *ic = reinterpret_cast<const int*>(static_cast<char*>(dev) + off);
}

struct GraphHandle {
  int device = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  void* dev = nullptr;
  int* err = nullptr;
};

}  // namespace

extern "C" int naja_chr_run_batched(int nmodels, const naja_polytope* const* models, const naja_chr_params* p,
                                    const double* const* X0s, int ldx, void* const* samples, double* const* X_finals,
                                    unsigned long long seed_stride, const naja_batch_config* c, void* stream_ptr) {
  BatchPrep b;
  int st = prep_batch(nmodels, models, p, X0s, ldx, samples, X_finals, seed_stride, c, &b);
  if (st) return st;
  DeviceGuard g(b.device);
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  DeviceBuffer buf;
  if ((st = buf.alloc(batch_bytes(b), stream))) return st;
  std::vector<unsigned char> host;
  const ModelDesc* dm;
  const int *im, *ic;
  batch_pack(b, host, buf.ptr, &dm, &im, &ic);
  cudaError_t e = cudaMemcpyAsync(buf.ptr, host.data(), host.size(), cudaMemcpyHostToDevice, stream);
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("naja_chr_run_batched: ") + cudaGetErrorString(e));
  st = chr_batch_launch(b.base, dm, im, ic, static_cast<int>(b.item_model.size()), b.cfg, stream);
  if (st) return fail(st, std::string("naja_chr_run_batched: launch failed: ") + cudaGetErrorString(cudaGetLastError()));
  // the staging copy above is from pageable memory: it has completed when cudaMemcpyAsync returned
  return NAJA_OK;
}

extern "C" int naja_batch_occupancy(int nmodels, const naja_polytope* const* models, const naja_batch_config* c,
                                    int* ctas_per_sm) {
  if (!ctas_per_sm || !c || nmodels <= 0 || !models || !models[0])
    return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_batch_occupancy: bad arguments");
  int lda_max = 0, m_max = 0;
  for (int k = 0; k < nmodels; ++k) {
    lda_max = std::max(lda_max, models[k]->lda);
    m_max = std::max(m_max, models[k]->m);
  }
  BatchConfig cfg;
  std::memset(&cfg, 0, sizeof(cfg));
  cfg.threads = c->threads;
  cfg.slots = c->slots;
  cfg.slack_smem = c->slack_smem;
  cfg.ctas_per_sm = c->ctas_per_sm;
  *ctas_per_sm = 0;
  if (c->sparse) {
    const int st = batch_sparse_prepare(nmodels, models, &cfg);
    if (st) return st;
  }
  if (chr_batch_plan(m_max, models[0]->d, lda_max, &cfg) != NAJA_OK) return NAJA_OK;
  DeviceGuard g(models[0]->device);
  int st = chr_batch_occupancy(cfg, ctas_per_sm);
  if (st) *ctas_per_sm = 0;
  return NAJA_OK;
}

extern "C" int naja_chr_capture_batched(int nmodels, const naja_polytope* const* models, const naja_chr_params* p,
                                        const double* const* X0s, int ldx, void* const* samples,
                                        double* const* X_finals, unsigned long long seed_stride,
                                        const naja_batch_config* c, void** graph) {
  if (!graph) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_chr_capture_batched: graph is null");
  *graph = nullptr;
  BatchPrep b;
  int st = prep_batch(nmodels, models, p, X0s, ldx, samples, X_finals, seed_stride, c, &b);
  if (st) return st;
  DeviceGuard g(b.device);
  GraphHandle* h = new GraphHandle();
  h->device = b.device;
  cudaError_t e = cudaMalloc(&h->dev, batch_bytes(b));
  if (e == cudaSuccess) e = cudaMalloc(&h->err, 4 * sizeof(int));
  if (e != cudaSuccess) {
    naja_graph_destroy(h);
    return fail(NAJA_ERR_NO_MEMORY, std::string("naja_chr_capture_batched: ") + cudaGetErrorString(e));
  }
  std::vector<unsigned char> host;
  const ModelDesc* dm;
  const int *im, *ic;
  batch_pack(b, host, h->dev, &dm, &im, &ic);
  e = cudaMemcpy(h->dev, host.data(), host.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(h->err, 0, 4 * sizeof(int));
  b.base.err = h->err;
  int occ = 0;
  if (e == cudaSuccess) chr_batch_occupancy(b.cfg, &occ);  // sets the kernel's smem attribute outside the capture
  cudaStream_t s = nullptr;
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed);
  if (e == cudaSuccess) {
    st = chr_batch_launch(b.base, dm, im, ic, static_cast<int>(b.item_model.size()), b.cfg, s);
    cudaError_t e2 = cudaStreamEndCapture(s, &h->graph);
    if (st == NAJA_OK) e = e2;
  }
  if (e == cudaSuccess && st == NAJA_OK) e = cudaGraphInstantiate(&h->exec, h->graph, 0);
  if (s) cudaStreamDestroy(s);
  if (e != cudaSuccess || st != NAJA_OK) {
    naja_graph_destroy(h);
    return fail(st ? st : NAJA_ERR_CUDA, std::string("naja_chr_capture_batched: ") + cudaGetErrorString(e));
  }
  *graph = h;
  return NAJA_OK;
}

extern "C" int naja_graph_launch(void* graph, void* stream) {
  GraphHandle* h = static_cast<GraphHandle*>(graph);
  if (!h || !h->exec) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_graph_launch: null graph");
  DeviceGuard g(h->device);
  cudaError_t e = cudaGraphLaunch(h->exec, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("naja_graph_launch: ") + cudaGetErrorString(e));
  return NAJA_OK;
}

extern "C" int naja_graph_check(void* graph) {
  GraphHandle* h = static_cast<GraphHandle*>(graph);
  if (!h) return fail(NAJA_ERR_INVALID_ARGUMENT, "naja_graph_check: null graph");
  DeviceGuard g(h->device);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("naja_graph_check: ") + cudaGetErrorString(e));
  return read_device_error(h->err);
}

extern "C" int naja_graph_destroy(void* graph) {
  GraphHandle* h = static_cast<GraphHandle*>(graph);
  if (!h) return NAJA_OK;
  DeviceGuard g(h->device);
  if (h->exec) cudaGraphExecDestroy(h->exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  cudaFree(h->dev);
  cudaFree(h->err);
  delete h;
  return NAJA_OK;
}
