// TEST INFRASTRUCTURE ONLY -- C entry points over the reference's own GPU
// sampler API (naja::gpu::CoordinateHitAndRun / backmap_into from
// src/gpu/{chr,backmap}.cu of quothbonney/naja, compiled unmodified from the
// reference tree by oracle/refharness/Makefile).  The parity tests call these
// to compare against the reference's kernel; bench.py's reference arm times
// them.  Nothing in the product links this.
#include <cuda_runtime.h>

#include <chrono>
#include <cstring>
#include <exception>
#include <string>

#include "backmap.cuh"
#include "cublaswrapper.h"
#include "dmatrix.h"
#include "dvector.h"
#include "gpusamplers.h"

using naja::gpu::DMatrix;
using naja::gpu::DVector;

namespace {
thread_local std::string g_err;

Eigen::MatrixXd host_matrix(const double* p, int rows, int cols) {
  Eigen::MatrixXd M(rows, cols);
  std::memcpy(M.data(), p, sizeof(double) * static_cast<size_t>(rows) * cols);
  return M;
}
Eigen::VectorXd host_vector(const double* p, int n) {
  Eigen::VectorXd v(n);
  std::memcpy(v.data(), p, sizeof(double) * n);
  return v;
}
}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

// Runs the reference's CoordinateHitAndRun.  A is m x d column-major, X0 is
// d x nchains column-major; samples receives d x (nchains*nspc) column-major
// (nullable).  If T (n x d column-major) and shift are given, the reference's
// backmap_into is applied to the device samples as CoordinateHitAndRunBackmap
// does (chr.cu:92-96) and V (nullable) receives n x (nchains*nspc).
// *sampling_ms is the wall time of the sampling (+ backmap) call followed by
// cudaDeviceSynchronize, as src/engine/job_sampling.cu times it.
int ref_chr_run(const double* A, int m, int d, const double* b, const double* X0, int nspc, int thinning,
                int nchains, int tpb, int seed, double pair_prob, int resync_interval, double ksparse_prob,
                int ksparse_k, int pair_mode, const int* pi, const int* pj, const double* pc, const double* ps,
                int n_pairs, const double* T, int n, const double* shift, double* samples, double* V,
                double* sampling_ms) {
  try {
    DMatrix<double> A_d(host_matrix(A, m, d));
    DVector<double> b_d(host_vector(b, m));
    DMatrix<double> X_d(host_matrix(X0, d, nchains));
    DVector<int>* pi_d = nullptr;
    DVector<int>* pj_d = nullptr;
    DVector<double>* pc_d = nullptr;
    DVector<double>* ps_d = nullptr;
    if (n_pairs > 0) {
      Eigen::Matrix<int, Eigen::Dynamic, 1> vi(n_pairs), vj(n_pairs);
      std::memcpy(vi.data(), pi, sizeof(int) * n_pairs);
      std::memcpy(vj.data(), pj, sizeof(int) * n_pairs);
      pi_d = new DVector<int>(vi);
      pj_d = new DVector<int>(vj);
      pc_d = new DVector<double>(host_vector(pc, n_pairs));
      ps_d = new DVector<double>(host_vector(ps, n_pairs));
    }
    DMatrix<double>* T_d = nullptr;
    DVector<double>* s_d = nullptr;
    if (T) {
      T_d = new DMatrix<double>(host_matrix(T, n, d));
      s_d = new DVector<double>(host_vector(shift, n));
    }
    cudaDeviceSynchronize();
    auto t0 = std::chrono::steady_clock::now();
    DMatrix<double> S = naja::gpu::CoordinateHitAndRun(A_d, b_d, X_d, nspc, thinning, nchains, tpb, seed, pair_prob,
                                                       resync_interval, ksparse_prob, ksparse_k, pair_mode, pi_d,
                                                       pj_d, pc_d, ps_d);
    DMatrix<double>* Vd = nullptr;
    if (T_d) {
      naja::gpu::CUBLASHandle handle;
      Vd = new DMatrix<double>(T_d->rows, S.cols);
      naja::gpu::backmap_into<double>(*T_d, *s_d, S, *Vd, handle, 0);
    }
    cudaError_t e = cudaDeviceSynchronize();
    auto t1 = std::chrono::steady_clock::now();
    if (sampling_ms) *sampling_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess && samples)
      e = cudaMemcpy(samples, S.dmat, sizeof(double) * static_cast<size_t>(d) * S.cols, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && V && Vd)
      e = cudaMemcpy(V, Vd->dmat, sizeof(double) * static_cast<size_t>(n) * S.cols, cudaMemcpyDeviceToHost);
    delete Vd;
    delete T_d;
    delete s_d;
    delete pi_d;
    delete pj_d;
    delete pc_d;
    delete ps_d;
    if (e != cudaSuccess) {
      g_err = cudaGetErrorString(e);
      return 3;
    }
    return 0;
  } catch (const std::exception& ex) {
    g_err = ex.what();
    return 2;
  }
}

}  // extern "C"
