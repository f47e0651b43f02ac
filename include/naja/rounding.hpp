// naja/rounding.hpp -- header-only producers of the sampler's rounding inputs
// over the C ABI (naja_chr.h), restating quothbonney/naja's
//
//   src/rounding/jacobi.cpp:8-22           jacobi_rotation_cs
//   src/rounding/schedule_io.cpp:12-88     pair schedule CSV "i,j,c,s"
//   src/rounding/runtime_warmup.cpp:16-108 estimate_runtime_pair_schedule
//   src/rounding/plan.cpp:12-62            build_rounding_plan (file or warm-up)
//   src/engine/job_sampling.cu:196-235     affine-hull reduction of a polytope
//
// The pair schedule feeds pair_mode 2 of naja_chr_run (Jacobi-rotated pair
// directions).  Errors throw std::invalid_argument / std::runtime_error as
// the reference does.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <fstream>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../naja_chr.h"

namespace naja {
namespace rounding {

// (c, s) = (cos theta, sin theta), theta = atan2(2 cov, var_i - var_j) / 2:
// the rotation of coordinates (i, j) that diagonalises the 2 x 2 covariance
// [[var_i, cov], [cov, var_j]]; (1, 0) when cov is 0.
inline std::pair<double, double> jacobi_rotation_cs(double var_i, double var_j, double cov_ij) {
  if (!(var_i >= 0.0) || !(var_j >= 0.0))
    throw std::invalid_argument("jacobi_rotation_cs: variances must be nonnegative");
  if (!std::isfinite(var_i) || !std::isfinite(var_j) || !std::isfinite(cov_ij))
    throw std::invalid_argument("jacobi_rotation_cs: inputs must be finite");
  if (cov_ij == 0.0) return {1.0, 0.0};
  const double theta = 0.5 * std::atan2(2.0 * cov_ij, var_i - var_j);
  return {std::cos(theta), std::sin(theta)};
}

struct PairSchedule {
  std::vector<int> i, j;
  std::vector<double> c, s;
  int size() const { return static_cast<int>(i.size()); }
};

// CSV rows "i,j,c,s"; blank lines and lines starting with '#' (after leading
// blanks) are skipped.  Indices must be >= 0, c and s finite and not both 0.
inline PairSchedule load_pair_schedule_csv(const std::string& path) {
  std::ifstream f(path);
  if (!f.is_open()) throw std::runtime_error("cannot open pair schedule: " + path);
  PairSchedule out;
  std::string line;
  int lineno = 0;
  while (std::getline(f, line)) {
    ++lineno;
    const size_t first = line.find_first_not_of(" \t");
    if (first == std::string::npos || line[first] == '#') continue;
    std::vector<std::string> cells;
    std::stringstream ss(line.substr(first));
    for (std::string cell; std::getline(ss, cell, ',');) cells.push_back(cell);
    const std::string where = "pair schedule parse error at line " + std::to_string(lineno);
    if (cells.size() != 4) throw std::runtime_error(where + ": expected 4 columns");
    const int a = std::stoi(cells[0]), b = std::stoi(cells[1]);
    const double c = std::stod(cells[2]), s = std::stod(cells[3]);
    if (a < 0 || b < 0) throw std::runtime_error(where + ": negative index");
    if (!std::isfinite(c) || !std::isfinite(s)) throw std::runtime_error(where + ": non-finite c/s");
    if (!(c * c + s * s > 0.0)) throw std::runtime_error(where + ": zero norm");
    out.i.push_back(a);
    out.j.push_back(b);
    out.c.push_back(c);
    out.s.push_back(s);
  }
  if (out.i.empty()) throw std::runtime_error("pair schedule is empty: " + path);
  return out;
}

inline void write_pair_schedule_csv(const std::string& path, const PairSchedule& p) {
  if (p.j.size() != p.i.size() || p.c.size() != p.i.size() || p.s.size() != p.i.size())
    throw std::invalid_argument("write_pair_schedule_csv: schedule arrays must have same length");
  std::ofstream f(path);
  if (!f.is_open()) throw std::runtime_error("cannot write pair schedule: " + path);
  for (int k = 0; k < p.size(); ++k) f << p.i[k] << "," << p.j[k] << "," << p.c[k] << "," << p.s[k] << "\n";
}

// Disjoint pairs (perm[2k], perm[2k+1]) of a seeded shuffle of 0..d-1,
// angle 0: std::shuffle with std::mt19937_64 seeded by `engine_seed`.
inline PairSchedule random_pairing(int d, uint64_t engine_seed) {
  std::vector<int> perm(d);
  for (int k = 0; k < d; ++k) perm[k] = k;
  std::mt19937_64 rng(engine_seed);
  std::shuffle(perm.begin(), perm.end(), rng);
  PairSchedule p;
  for (int k = 0; k < d / 2; ++k) {
    p.i.push_back(perm[2 * k]);
    p.j.push_back(perm[2 * k + 1]);
    p.c.push_back(1.0);
    p.s.push_back(0.0);
  }
  return p;
}

// Population moments of coordinates (i, j) over the samples (rows of d
// values): the pair's Jacobi rotation.
inline std::pair<double, double> pair_rotation(const std::vector<double>& W, long n, int d, int ii, int jj) {
  double mi = 0.0, mj = 0.0;
  for (long t = 0; t < n; ++t) {
    mi += W[static_cast<size_t>(t) * d + ii];
    mj += W[static_cast<size_t>(t) * d + jj];
  }
  mi /= static_cast<double>(n);
  mj /= static_cast<double>(n);
  double vi = 0.0, vj = 0.0, cij = 0.0;
  for (long t = 0; t < n; ++t) {
    const double di = W[static_cast<size_t>(t) * d + ii] - mi, dj = W[static_cast<size_t>(t) * d + jj] - mj;
    vi += di * di;
    vj += dj * dj;
    cij += di * dj;
  }
  return jacobi_rotation_cs(vi / n, vj / n, cij / n);
}

// Warm-up estimate of the pair schedule (the reference's iterative
// rounding-lite): pairs from a shuffle seeded with seed ^ 0x9e3779b97f4a7c15,
// then `passes` warm-up runs of one chain (`warmup` samples, thinning 1, pair
// probability clamped to [0.05, 0.5], seed ^ (pass + 1); pass 0 with the
// fixed (e_i - e_j)/sqrt 2 pairs, later passes with the schedule so far), each
// followed by the Jacobi rotation of every pair's sample moments.  `tier`
// supplies precision / rng / tpb of the warm-up runs (the reference's are
// FP64 with cuRAND MRG32k3a).
inline PairSchedule estimate_runtime_pair_schedule(naja_polytope* P, const std::vector<double>& x0, int seed,
                                                   int passes, int warmup, double pair_prob,
                                                   const naja_chr_params& tier) {
  int m = 0, d = 0;
  naja_polytope_shape(P, &m, &d);
  if (d < 2) throw std::invalid_argument("estimate_runtime_pair_schedule: reduced_dim must be >= 2");
  if (passes <= 0) throw std::invalid_argument("estimate_runtime_pair_schedule: passes must be > 0");
  if (warmup <= 0) throw std::invalid_argument("estimate_runtime_pair_schedule: warmup must be > 0");
  if (static_cast<int>(x0.size()) != d) throw std::invalid_argument("estimate_runtime_pair_schedule: x0 size != d");
  PairSchedule sched = random_pairing(d, static_cast<uint64_t>(seed) ^ 0x9e3779b97f4a7c15ULL);
  std::vector<double> W(static_cast<size_t>(warmup) * d);
  for (int pass = 0; pass < passes; ++pass) {
    naja_chr_params p = tier;
    p.nspc = warmup;
    p.thinning = 1;
    p.nchains = 1;
    p.seed = static_cast<unsigned long long>(static_cast<long long>(seed ^ (pass + 1)));
    p.pair_prob = std::min(std::max(pair_prob, 0.05), 0.5);
    p.resync_interval = 0;
    p.ksparse_prob = 0.0;
    p.pair_mode = pass == 0 ? 1 : 2;
    p.pair_i = pass == 0 ? nullptr : sched.i.data();
    p.pair_j = pass == 0 ? nullptr : sched.j.data();
    p.pair_c = pass == 0 ? nullptr : sched.c.data();
    p.pair_s = pass == 0 ? nullptr : sched.s.data();
    p.n_pairs = pass == 0 ? 0 : sched.size();
    p.out_dtype = NAJA_DTYPE_F64;
    p.chain_base = 0;
    p.out_nchains = 0;
    p.step_offset = 0;
    p.rng_state = nullptr;
    int st = naja_chr_run(P, &p, x0.data(), d, W.data(), nullptr, nullptr);
    if (st == NAJA_OK) st = naja_polytope_check(P);
    if (st != NAJA_OK) throw std::runtime_error(std::string("estimate_runtime_pair_schedule: ") + naja_last_error());
    for (int k = 0; k < sched.size(); ++k) {
      const auto cs = pair_rotation(W, warmup, d, sched.i[k], sched.j[k]);
      sched.c[k] = cs.first;
      sched.s[k] = cs.second;
    }
  }
  return sched;
}

// Null-space basis of the rows of A (m x n, row-major) tight at x0 (slack
// b - A x0 <= tol): the affine hull {x0 + B z} the chains can move in.
// Householder QR with column pivoting of the tight rows' transpose (n x k):
// rank r = pivots above 1e-10 * the largest; B = the last n - r columns of Q
// (orthonormal, n x (n - r), row-major).  Returns false (B empty) when no row
// is tight or the rank is 0 or n.  The reference takes Eigen's FullPivLU
// kernel of the same rows (threshold 1e-10); both bases span the same null
// space, so the chains sample the same affine hull, in other coordinates.
inline bool affine_hull_basis(const std::vector<double>& A, const std::vector<double>& b, const std::vector<double>& x0,
                              int m, int n, double tol, std::vector<double>& B, int* dim, int* n_tight) {
  std::vector<int> rows;
  for (int i = 0; i < m; ++i) {
    double s = b[i];
    for (int k = 0; k < n; ++k) s -= A[static_cast<size_t>(i) * n + k] * x0[k];
    if (s <= tol) rows.push_back(i);
  }
  *n_tight = static_cast<int>(rows.size());
  B.clear();
  *dim = n;
  const int kk = static_cast<int>(rows.size());
  if (kk == 0) return false;
  // M = Aeq^T, n x kk, column-major
  std::vector<double> M(static_cast<size_t>(n) * kk);
  for (int c = 0; c < kk; ++c)
    for (int r = 0; r < n; ++r) M[static_cast<size_t>(c) * n + r] = A[static_cast<size_t>(rows[c]) * n + r];
  std::vector<double> norms(kk);
  for (int c = 0; c < kk; ++c) {
    double s = 0.0;
    for (int r = 0; r < n; ++r) s += M[static_cast<size_t>(c) * n + r] * M[static_cast<size_t>(c) * n + r];
    norms[c] = s;
  }
  std::vector<std::vector<double>> V;  // Householder vectors
  const int steps = std::min(n, kk);
  double first = -1.0;
  int rank = 0;
  for (int t = 0; t < steps; ++t) {
    int piv = t;
    for (int c = t + 1; c < kk; ++c)
      if (norms[c] > norms[piv]) piv = c;
    if (piv != t) {
      for (int r = 0; r < n; ++r) std::swap(M[static_cast<size_t>(t) * n + r], M[static_cast<size_t>(piv) * n + r]);
      std::swap(norms[t], norms[piv]);
    }
    double* col = &M[static_cast<size_t>(t) * n];
    double alpha = 0.0;
    for (int r = t; r < n; ++r) alpha += col[r] * col[r];
    alpha = std::sqrt(alpha);
    if (first < 0.0) first = alpha;
    if (!(alpha > 1e-10 * first) || alpha == 0.0) break;
    ++rank;
    std::vector<double> v(n, 0.0);
    for (int r = t; r < n; ++r) v[r] = col[r];
    v[t] += col[t] >= 0.0 ? alpha : -alpha;
    double vv = 0.0;
    for (int r = t; r < n; ++r) vv += v[r] * v[r];
    for (int c = t; c < kk; ++c) {
      double* mc = &M[static_cast<size_t>(c) * n];
      double dot = 0.0;
      for (int r = t; r < n; ++r) dot += v[r] * mc[r];
      const double f = 2.0 * dot / vv;
      for (int r = t; r < n; ++r) mc[r] -= f * v[r];
    }
    for (int c = t + 1; c < kk; ++c) norms[c] -= M[static_cast<size_t>(c) * n + t] * M[static_cast<size_t>(c) * n + t];
    for (double& x : v) x /= std::sqrt(vv);
    V.push_back(std::move(v));
  }
  const int dd = n - rank;
  if (rank == 0 || dd <= 0) return false;
  // columns rank..n-1 of Q = H_0 H_1 ... H_{r-1} e_c
  B.assign(static_cast<size_t>(n) * dd, 0.0);
  std::vector<double> e(n);
  for (int q = 0; q < dd; ++q) {
    std::fill(e.begin(), e.end(), 0.0);
    e[rank + q] = 1.0;
    for (int h = rank - 1; h >= 0; --h) {
      double dot = 0.0;
      for (int r = 0; r < n; ++r) dot += V[h][r] * e[r];
      for (int r = 0; r < n; ++r) e[r] -= 2.0 * dot * V[h][r];
    }
    for (int r = 0; r < n; ++r) B[static_cast<size_t>(r) * dd + q] = e[r];
  }
  *dim = dd;
  return true;
}

}  // namespace rounding
}  // namespace naja
