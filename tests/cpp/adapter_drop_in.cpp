// Exercises include/naja/gpusamplers.hpp the way the reference's callers use
// naja::gpu (src/engine/job_sampling.cu:258-405): host matrices uploaded into
// DMatrix / DVector, CoordinateHitAndRun[Backmap|Streamed], toHost().
// Exit status 0 = all checks passed.
#include <naja/gpusamplers.hpp>

#include <cmath>
#include <cstdio>
#include <vector>

using naja::gpu::DMatrix;
using naja::gpu::DVector;
using naja::gpu::HMatrix;
using naja::gpu::HVector;

static int fails = 0;
#define CHECK(c)                                              \
  do {                                                        \
    if (!(c)) {                                               \
      std::fprintf(stderr, "check failed: %s (line %d)\n", #c, __LINE__); \
      ++fails;                                                \
    }                                                         \
  } while (0)

int main() {
  const int d = 6, m = 2 * d, k = 4, nspc = 4000, thin = 10;
  HMatrix<double> A(m, d);
  HVector<double> b(m);
  for (int i = 0; i < m; ++i) {
    b[i] = 1.0;
    for (int j = 0; j < d; ++j) A(i, j) = 0.0;
  }
  for (int i = 0; i < d; ++i) {
    A(2 * i, i) = 1.0;
    A(2 * i + 1, i) = -1.0;
  }
  HMatrix<double> X0(d, k);
  for (int c = 0; c < k; ++c)
    for (int j = 0; j < d; ++j) X0(j, c) = 0.0;

  DMatrix<double> A_d(A);
  DVector<double> b_d(b);
  DMatrix<double> X_d(X0);

  // 1. one-shot sampling, reference tier: shape, feasibility, moments
  DMatrix<double> S_d = naja::gpu::CoordinateHitAndRun(A_d, b_d, X_d, nspc, thin, k, 128, 42);
  CHECK(S_d.rows == d && S_d.cols == k * nspc);
  HMatrix<double> S = S_d.toHost();
  double worst = -1e300, var = 0.0;
  for (long c = 0; c < S.cols(); ++c)
    for (int j = 0; j < d; ++j) {
      worst = std::fmax(worst, std::fabs(S(j, c)) - 1.0);
      var += S(j, c) * S(j, c);
    }
  var /= static_cast<double>(S.cols()) * d;
  CHECK(worst <= 1e-12);
  CHECK(std::fabs(var - 1.0 / 3.0) < 0.05);

  // 2. argument errors throw the reference's exception classes
  bool threw = false;
  try {
    naja::gpu::CoordinateHitAndRun(A_d, b_d, X_d, nspc, thin, k, 100, 42);
  } catch (const std::invalid_argument&) {
    threw = true;
  }
  CHECK(threw);

  // 3. backmap: V = T y + shift, column by column
  const int n = 9;
  HMatrix<double> T(n, d);
  HVector<double> shift(n);
  for (int i = 0; i < n; ++i) {
    shift[i] = 0.1 * i;
    for (int j = 0; j < d; ++j) T(i, j) = std::sin(1.0 + i * d + j);
  }
  DMatrix<double> T_d(T);
  DVector<double> s_d(shift);
  DMatrix<double> V_d = naja::gpu::CoordinateHitAndRunBackmap(A_d, b_d, X_d, T_d, s_d, 500, thin, k, 128, 42);
  CHECK(V_d.rows == n && V_d.cols == k * 500);
  HMatrix<double> V = V_d.toHost();
  double err = 0.0;
  for (long c = 0; c < V.cols(); ++c)
    for (int i = 0; i < n; ++i) {
      double v = shift[i];
      for (int j = 0; j < d; ++j) v += T(i, j) * S(j, c);
      err = std::fmax(err, std::fabs(v - V(i, c)));
    }
  CHECK(err < 1e-9);  // same seed, same first 500 samples per chain

  // 4. streamed chunks reproduce the one-shot run
  DMatrix<double> X2(X0);
  std::vector<double> streamed;
  naja::gpu::CoordinateHitAndRunStreamed(A_d, b_d, X2, nspc, 700, thin, k, 128, 42, 0.0, 0, 0.0, 8, 1, nullptr,
                                         nullptr, nullptr, nullptr,
                                         [&](const double* p, int rows, int cols) {
                                           streamed.insert(streamed.end(), p, p + static_cast<size_t>(rows) * cols);
                                         });
  CHECK(streamed.size() == static_cast<size_t>(d) * k * nspc);
  double sdiff = 0.0;
  for (size_t i = 0; i < streamed.size() && i < static_cast<size_t>(S.size()); ++i)
    sdiff = std::fmax(sdiff, std::fabs(streamed[i] - S.data()[i]));
  CHECK(sdiff < 1e-12);

  // 5. fast tier runs and stays feasible
  DMatrix<double> F_d = naja::gpu::CoordinateHitAndRun(A_d, b_d, X_d, 1000, thin, k, -1, 7, 0.3, 64, 0.0, 8, 1,
                                                       nullptr, nullptr, nullptr, nullptr, naja::gpu::Tier::fast());
  HMatrix<double> F = F_d.toHost();
  double fw = -1e300;
  for (long i = 0; i < F.size(); ++i) fw = std::fmax(fw, std::fabs(F.data()[i]) - 1.0);
  CHECK(fw <= 1e-6);

  if (fails == 0) std::printf("adapter ok\n");
  return fails == 0 ? 0 : 1;
}
