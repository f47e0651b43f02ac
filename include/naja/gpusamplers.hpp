// naja/gpusamplers.hpp -- header-only C++ adapter over the C ABI
// (naja_chr.h) that reproduces the reference's GPU sampler API
// (src/gpu/gpusamplers.h:30-86, src/gpu/dmatrix.h:23-74,
// src/gpu/dvector.h:22-62 of quothbonney/naja) so its callers compile
// unchanged:
//
//   naja::gpu::DMatrix<double>  column-major, int dims, members dmat/rows/cols/ownsData
//   naja::gpu::DVector<T>       members dvec/len
//   naja::gpu::CoordinateHitAndRun(...)         -> DMatrix<double> d x (nchains*nspc)
//   naja::gpu::CoordinateHitAndRunBackmap(...)  -> DMatrix<double> n x (nchains*nspc)
//   naja::gpu::CoordinateHitAndRunStreamed(...) -> chunks to a host sink
//
// Errors follow the reference: std::invalid_argument for argument errors,
// std::runtime_error for everything else (the reference's CUDA_CHECK only
// printed; here a CUDA failure throws).
//
// Arithmetic tier: by default the adapter runs the reference's arithmetic
// (FP64 throughout) and its random stream (cuRAND MRG32k3a seeded
// curand_init(seed, chain, 0)), which reproduces the reference's samples bit
// for bit whenever A x0 is exact.  Pass a `Tier` as the trailing argument
// for the FP32 / Philox fast tier.
//
// Host matrices: any type with data(), rows(), cols() (Eigen::MatrixXd
// included) constructs a DMatrix; toHost() returns Eigen types when
// <Eigen/Dense> is available, else naja::gpu::HostMatrix.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../naja_chr.h"

#if __has_include(<Eigen/Dense>)
#include <Eigen/Dense>
#define NAJA_ADAPTER_HAS_EIGEN 1
#endif

namespace naja {
namespace gpu {

#ifdef NAJA_ADAPTER_HAS_EIGEN
template <typename Real>
using HMatrix = Eigen::Matrix<Real, Eigen::Dynamic, Eigen::Dynamic>;
template <typename Real>
using HVector = Eigen::Matrix<Real, Eigen::Dynamic, 1>;
#else
// Column-major host matrix with the members the API uses.
template <typename Real>
struct HostMatrix {
  HostMatrix() = default;
  explicit HostMatrix(long n) : r(n), c(1), v(static_cast<size_t>(n)) {}
  HostMatrix(long rows_, long cols_) : r(rows_), c(cols_), v(static_cast<size_t>(rows_ * cols_)) {}
  Real* data() { return v.data(); }
  const Real* data() const { return v.data(); }
  long rows() const { return r; }
  long cols() const { return c; }
  long size() const { return r * c; }
  Real& operator()(long i, long j) { return v[static_cast<size_t>(j * r + i)]; }
  const Real& operator()(long i, long j) const { return v[static_cast<size_t>(j * r + i)]; }
  Real& operator[](long i) { return v[static_cast<size_t>(i)]; }
  const Real& operator[](long i) const { return v[static_cast<size_t>(i)]; }
  long r = 0, c = 0;
  std::vector<Real> v;
};
template <typename Real>
using HMatrix = HostMatrix<Real>;
template <typename Real>
using HVector = HostMatrix<Real>;
#endif

namespace detail {
inline void throw_status(int st, const char* where) {
  if (st == NAJA_OK) return;
  std::string msg = std::string(where) + ": " + naja_last_error();
  if (st == NAJA_ERR_INVALID_ARGUMENT) throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}
inline void cuda_check(cudaError_t e, const char* where) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(where) + ": " + cudaGetErrorString(e));
}
template <class T, class = void>
struct is_host_matrix : std::false_type {};
template <class T>
struct is_host_matrix<T, std::void_t<decltype(std::declval<const T&>().data()), decltype(std::declval<const T&>().rows()),
                                     decltype(std::declval<const T&>().cols())>> : std::true_type {};
}  // namespace detail

template <typename Real>
struct DVector {
  Real* dvec = nullptr;
  int len = 0;

  template <class V, class = std::enable_if_t<detail::is_host_matrix<V>::value>>
  DVector(const V& v) : len(static_cast<int>(v.size())) {
    detail::cuda_check(cudaMalloc(&dvec, sizeof(Real) * std::max(len, 1)), "DVector");
    detail::cuda_check(cudaMemcpy(dvec, v.data(), sizeof(Real) * len, cudaMemcpyHostToDevice), "DVector");
  }
  explicit DVector(int len_) : len(len_) { detail::cuda_check(cudaMalloc(&dvec, sizeof(Real) * std::max(len, 1)), "DVector"); }
  DVector(int len_, Real value) : DVector(len_) { fill(value); }
  DVector(const DVector& o) : DVector(o.len) {
    detail::cuda_check(cudaMemcpy(dvec, o.dvec, sizeof(Real) * len, cudaMemcpyDeviceToDevice), "DVector");
  }
  DVector(DVector&& o) noexcept : dvec(o.dvec), len(o.len) {
    o.dvec = nullptr;
    o.len = 0;
  }
  DVector& operator=(const DVector& o) {
    if (this != &o) {
      DVector t(o);
      std::swap(dvec, t.dvec);
      std::swap(len, t.len);
    }
    return *this;
  }
  DVector& operator=(DVector&& o) noexcept {
    std::swap(dvec, o.dvec);
    std::swap(len, o.len);
    return *this;
  }
  ~DVector() {
    if (dvec) cudaFree(dvec);
  }
  void fill(Real value) {
    std::vector<Real> h(static_cast<size_t>(len), value);
    detail::cuda_check(cudaMemcpy(dvec, h.data(), sizeof(Real) * len, cudaMemcpyHostToDevice), "DVector::fill");
  }
  HVector<Real> toHost() const {
    HVector<Real> v(len);
    detail::cuda_check(cudaMemcpy(v.data(), dvec, sizeof(Real) * len, cudaMemcpyDeviceToHost), "DVector::toHost");
    return v;
  }
};

template <typename Real>
struct DMatrix {
  Real* dmat = nullptr;
  int rows = 0;
  int cols = 0;
  bool ownsData = false;

  template <class M, class = std::enable_if_t<detail::is_host_matrix<M>::value>>
  DMatrix(const M& m) : rows(static_cast<int>(m.rows())), cols(static_cast<int>(m.cols())), ownsData(true) {
    alloc();
    detail::cuda_check(cudaMemcpy(dmat, m.data(), bytes(), cudaMemcpyHostToDevice), "DMatrix");
  }
  DMatrix(int rows_, int cols_) : rows(rows_), cols(cols_), ownsData(true) { alloc(); }
  // Broadcast a device vector into `cols_` columns (dmatrix.cu:61-68).
  DMatrix(const DVector<Real>& v, int cols_) : rows(v.len), cols(cols_), ownsData(true) {
    alloc();
    for (int c = 0; c < cols; ++c)
      detail::cuda_check(cudaMemcpy(dmat + static_cast<size_t>(c) * rows, v.dvec, sizeof(Real) * rows,
                                    cudaMemcpyDeviceToDevice),
                         "DMatrix");
  }
  // Non-owning view (dmatrix.h:52).
  DMatrix(Real* p, int rows_, int cols_) : dmat(p), rows(rows_), cols(cols_), ownsData(false) {}
  DMatrix(const DMatrix& o) : rows(o.rows), cols(o.cols), ownsData(true) {
    alloc();
    detail::cuda_check(cudaMemcpy(dmat, o.dmat, bytes(), cudaMemcpyDeviceToDevice), "DMatrix");
  }
  DMatrix(DMatrix&& o) noexcept : dmat(o.dmat), rows(o.rows), cols(o.cols), ownsData(o.ownsData) {
    o.dmat = nullptr;
    o.ownsData = false;
  }
  DMatrix& operator=(const DMatrix&) = delete;
  DMatrix& operator=(DMatrix&&) = delete;
  ~DMatrix() {
    if (ownsData && dmat) cudaFree(dmat);
  }
  HMatrix<Real> toHost() const {
    HMatrix<Real> m(rows, cols);
    detail::cuda_check(cudaMemcpy(m.data(), dmat, bytes(), cudaMemcpyDeviceToHost), "DMatrix::toHost");
    return m;
  }
  DMatrix subMatrix(int r0, int c0, int r1, int c1) const {
    return DMatrix(dmat + static_cast<size_t>(c0) * rows + r0, r1 - r0, c1 - c0);
  }

 private:
  size_t bytes() const { return sizeof(Real) * static_cast<size_t>(rows) * cols; }
  void alloc() { detail::cuda_check(cudaMalloc(&dmat, std::max<size_t>(bytes(), 1)), "DMatrix"); }
};

// Arithmetic / RNG tier of a call (see the header comment).
struct Tier {
  int precision = NAJA_PREC_FP64;
  int rng = NAJA_RNG_REF_MRG;
  static Tier reference() { return Tier{}; }
  static Tier fast() { return Tier{NAJA_PREC_FP32, NAJA_RNG_PHILOX}; }
};

namespace detail {
struct PolytopeHandle {
  naja_polytope* p = nullptr;
  PolytopeHandle(const DMatrix<double>& A, const DVector<double>& b) {
    int dev = 0;
    cudaGetDevice(&dev);
    throw_status(naja_polytope_create(dev, A.rows, A.cols, A.dmat, A.rows, b.dvec, &p), "CoordinateHitAndRun");
  }
  ~PolytopeHandle() { naja_polytope_destroy(p); }
};

inline naja_chr_params make_params(int nspc, int thinning, int nchains, int tpb_ss, int seed, double pair_prob,
                                   int resync_interval, double ksparse_prob, int ksparse_k, int pair_mode,
                                   const DVector<int>* pair_i, const DVector<int>* pair_j,
                                   const DVector<double>* pair_c, const DVector<double>* pair_s, const Tier& tier) {
  naja_chr_params p;
  naja_chr_params_default(&p);
  p.nspc = nspc;
  p.thinning = thinning;
  p.nchains = nchains;
  p.tpb = tpb_ss > 0 ? tpb_ss : 0;
  // The reference passes an int seed to curand_init(unsigned long long, ...).
  p.seed = static_cast<unsigned long long>(static_cast<long long>(seed));
  p.pair_prob = pair_prob;
  p.resync_interval = resync_interval;
  p.ksparse_prob = ksparse_prob;
  p.ksparse_k = ksparse_k;
  p.pair_mode = pair_mode;
  if (pair_i && pair_j && pair_c && pair_s) {
    p.pair_i = pair_i->dvec;
    p.pair_j = pair_j->dvec;
    p.pair_c = pair_c->dvec;
    p.pair_s = pair_s->dvec;
    p.n_pairs = pair_i->len;
  }
  p.precision = tier.precision;
  p.rng = tier.rng;
  p.out_dtype = NAJA_DTYPE_F64;
  return p;
}
}  // namespace detail

inline DMatrix<double> CoordinateHitAndRun(DMatrix<double>& A_d, DVector<double>& b_d, DMatrix<double>& X_d, int nspc,
                                           int thinning, int nchains, int tpb_ss = -1, int seed = 0,
                                           double pair_prob = 0.0, int resync_interval = 0, double ksparse_prob = 0.0,
                                           int ksparse_k = 8, int pair_mode = 1,
                                           const DVector<int>* pair_i = nullptr, const DVector<int>* pair_j = nullptr,
                                           const DVector<double>* pair_c = nullptr,
                                           const DVector<double>* pair_s = nullptr, Tier tier = Tier::reference()) {
  detail::PolytopeHandle P(A_d, b_d);
  DMatrix<double> out(A_d.cols, nchains * nspc);
  naja_chr_params p = detail::make_params(nspc, thinning, nchains, tpb_ss, seed, pair_prob, resync_interval,
                                          ksparse_prob, ksparse_k, pair_mode, pair_i, pair_j, pair_c, pair_s, tier);
  detail::throw_status(naja_chr_run(P.p, &p, X_d.dmat, X_d.rows, out.dmat, nullptr, nullptr), "CoordinateHitAndRun");
  detail::throw_status(naja_polytope_check(P.p), "CoordinateHitAndRun");
  return out;
}

inline DMatrix<double> CoordinateHitAndRunBackmap(
    DMatrix<double>& A_d, DVector<double>& b_d, DMatrix<double>& X_d, const DMatrix<double>& transformation_d,
    const DVector<double>& shift_d, int nspc, int thinning, int nchains, int tpb_ss = -1, int seed = 0,
    double pair_prob = 0.0, int resync_interval = 0, double ksparse_prob = 0.0, int ksparse_k = 8, int pair_mode = 1,
    const DVector<int>* pair_i = nullptr, const DVector<int>* pair_j = nullptr,
    const DVector<double>* pair_c = nullptr, const DVector<double>* pair_s = nullptr, Tier tier = Tier::reference(),
    int backmap_mode = NAJA_BACKMAP_FP64) {
  if (transformation_d.cols != A_d.cols)
    throw std::invalid_argument("backmap_into: transformation shape mismatch with samples");
  if (shift_d.len != transformation_d.rows)
    throw std::invalid_argument("backmap_into: shift length mismatch with transformation rows");
  // One library call: sampling, then the backmap of each chunk of samples
  // while the next chunk samples (a single chunk for the MRG32k3a streams or
  // without a resync interval); the samples are those of CoordinateHitAndRun.
  detail::PolytopeHandle P(A_d, b_d);
  naja_chr_params p = detail::make_params(nspc, thinning, nchains, tpb_ss, seed, pair_prob, resync_interval,
                                          ksparse_prob, ksparse_k, pair_mode, pair_i, pair_j, pair_c, pair_s, tier);
  DMatrix<double> V(transformation_d.rows, nchains * nspc);
  detail::throw_status(naja_chr_run_backmapped(P.p, &p, X_d.dmat, X_d.rows, transformation_d.rows,
                                               transformation_d.dmat, transformation_d.rows, shift_d.dvec,
                                               backmap_mode, V.dmat, NAJA_DTYPE_F64, nullptr, nullptr, 0, nullptr),
                       "CoordinateHitAndRunBackmap");
  return V;
}

// Chunked sampling with the final state carried between chunks
// (src/gpu/chr.cu:101-230).  Philox chains continue by step offset; MRG
// chains carry their cuRAND states.  Each chunk (d x nchains*chunk columns)
// is handed to `host_sink` once it is on the host.
inline void CoordinateHitAndRunStreamed(DMatrix<double>& A_d, DVector<double>& b_d, DMatrix<double>& X_d, int nspc_total,
                                        int chunk_nspc, int thinning, int nchains, int tpb_ss, int seed,
                                        double pair_prob, int resync_interval, double ksparse_prob, int ksparse_k,
                                        int pair_mode, const DVector<int>* pair_i, const DVector<int>* pair_j,
                                        const DVector<double>* pair_c, const DVector<double>* pair_s,
                                        const std::function<void(const double*, int, int)>& host_sink,
                                        Tier tier = Tier::reference()) {
  if (nchains <= 0) throw std::invalid_argument("CoordinateHitAndRunStreamed: nchains must be positive");
  if (chunk_nspc <= 0) throw std::invalid_argument("CoordinateHitAndRunStreamed: chunk_nspc must be positive");
  if (nspc_total <= 0) return;
  if (!host_sink) throw std::invalid_argument("CoordinateHitAndRunStreamed: host_sink must be callable");
  const int N = A_d.cols;
  if (N <= 0) return;
  detail::PolytopeHandle P(A_d, b_d);
  void* states = nullptr;
  if (tier.rng == NAJA_RNG_REF_MRG) {
    // per-chain cuRAND states seeded as the reference seeds them, carried across chunks
    detail::cuda_check(cudaMalloc(&states, naja_mrg_state_bytes() * nchains), "CoordinateHitAndRunStreamed");
    int dev = 0;
    cudaGetDevice(&dev);
    detail::throw_status(naja_mrg_init_states(dev, static_cast<unsigned long long>(static_cast<long long>(seed)), 0,
                                              nchains, states),
                         "CoordinateHitAndRunStreamed");
  }
  DMatrix<double> chunk(N, nchains * chunk_nspc);
  std::vector<double> host(static_cast<size_t>(N) * nchains * chunk_nspc);
  long long step = 0;
  for (int done = 0; done < nspc_total; done += chunk_nspc) {
    const int n_this = std::min(chunk_nspc, nspc_total - done);
    naja_chr_params p = detail::make_params(n_this, thinning, nchains, tpb_ss, seed, pair_prob, resync_interval,
                                            ksparse_prob, ksparse_k, pair_mode, pair_i, pair_j, pair_c, pair_s, tier);
    p.step_offset = step;
    p.rng_state = states;
    // X_d is the chain state: read at the start of the chunk, written at its end (chr.cu:485-489)
    int st = naja_chr_run(P.p, &p, X_d.dmat, X_d.rows, chunk.dmat, X_d.dmat, nullptr);
    detail::throw_status(st, "CoordinateHitAndRunStreamed");
    detail::throw_status(naja_polytope_check(P.p), "CoordinateHitAndRunStreamed");
    const size_t cols = static_cast<size_t>(nchains) * n_this;
    detail::cuda_check(cudaMemcpy(host.data(), chunk.dmat, sizeof(double) * N * cols, cudaMemcpyDeviceToHost),
                       "CoordinateHitAndRunStreamed");
    host_sink(host.data(), N, static_cast<int>(cols));
    step += static_cast<long long>(n_this) * thinning;
  }
  if (states) cudaFree(states);
}

}  // namespace gpu
}  // namespace naja
