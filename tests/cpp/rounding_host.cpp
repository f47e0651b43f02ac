// Host-side checks of include/naja/rounding.hpp (no GPU work is run):
// jacobi_rotation_cs on the reference's cases
// (tests/test_iterative_rounding_jacobi.cpp:7-31 of quothbonney/naja), the
// pair-schedule CSV round trip (tests/test_pair_schedule_io.cpp) and its
// errors, the seeded pairing, and the affine-hull basis of a known system.
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#include "naja/rounding.hpp"

using naja::rounding::PairSchedule;

static int fails = 0;
#define CHECK(cond)                                                   \
  do {                                                                \
    if (!(cond)) {                                                    \
      std::cerr << "check failed line " << __LINE__ << ": " #cond "\n"; \
      ++fails;                                                        \
    }                                                                 \
  } while (0)

static bool diagonalises(double a, double b, double c) {
  const auto cs = naja::rounding::jacobi_rotation_cs(a, b, c);
  // off-diagonal of R^T S R, S = [a c; c b], R = [cs -sn; sn cs]
  const double d01 = (b - a) * cs.first * cs.second + c * (cs.first * cs.first - cs.second * cs.second);
  return std::abs(d01) < 1e-10 && std::abs(cs.first * cs.first + cs.second * cs.second - 1.0) < 1e-14;
}

template <class F>
static bool throws(F f) {
  try {
    f();
  } catch (const std::exception&) {
    return true;
  }
  return false;
}

int main(int argc, char** argv) {
  const std::string dir = argc > 1 ? argv[1] : "/tmp";
  CHECK(diagonalises(4.0, 1.0, 1.2));
  CHECK(diagonalises(0.5, 3.0, -0.7));
  CHECK(diagonalises(2.0, 5.0, 0.0));
  CHECK(naja::rounding::jacobi_rotation_cs(2.0, 5.0, 0.0) == std::make_pair(1.0, 0.0));
  CHECK(throws([] { naja::rounding::jacobi_rotation_cs(-1.0, 1.0, 0.1); }));
  CHECK(throws([] { naja::rounding::jacobi_rotation_cs(1.0, NAN, 0.1); }));

  const std::string path = dir + "/naja_pair_schedule.csv";
  {
    std::ofstream f(path);
    f << "# pairs\n0,1,1,0\n\n  2,3,0.6,0.8\n";
  }
  PairSchedule s = naja::rounding::load_pair_schedule_csv(path);
  CHECK(s.size() == 2 && s.i[0] == 0 && s.j[0] == 1 && s.i[1] == 2 && s.j[1] == 3);
  CHECK(std::abs(s.c[1] * s.c[1] + s.s[1] * s.s[1] - 1.0) < 1e-12);
  naja::rounding::write_pair_schedule_csv(path, s);
  PairSchedule s2 = naja::rounding::load_pair_schedule_csv(path);
  CHECK(s2.i == s.i && s2.j == s.j && s2.c == s.c && s2.s == s.s);
  const char* bad[] = {"0,1,1\n", "-1,2,1,0\n", "0,1,0,0\n", "0,1,nan,0\n", "# only a comment\n"};
  for (const char* text : bad) {
    {
      std::ofstream f(path);
      f << text;
    }
    CHECK(throws([&] { naja::rounding::load_pair_schedule_csv(path); }));
  }
  CHECK(throws([&] { naja::rounding::load_pair_schedule_csv(dir + "/does_not_exist.csv"); }));
  std::remove(path.c_str());

  PairSchedule p = naja::rounding::random_pairing(9, 7);
  std::set<int> seen;
  for (int k = 0; k < p.size(); ++k) {
    seen.insert(p.i[k]);
    seen.insert(p.j[k]);
  }
  CHECK(p.size() == 4 && seen.size() == 8 && *seen.rbegin() <= 8);
  PairSchedule q = naja::rounding::random_pairing(9, 7);
  CHECK(q.i == p.i && q.j == p.j);

  // y1 + y2 + y3 <= 1 and -(y1 + y2 + y3) <= -1 are tight at x0 = (1/3, 1/3, 1/3):
  // the hull is the plane y1 + y2 + y3 = 1 (dimension 2); a loose box row is ignored.
  const int m = 3, n = 3;
  std::vector<double> A = {1, 1, 1, -1, -1, -1, 1, 0, 0}, b = {1, -1, 5}, x0 = {1.0 / 3, 1.0 / 3, 1.0 / 3};
  std::vector<double> B;
  int dim = 0, tight = 0;
  CHECK(naja::rounding::affine_hull_basis(A, b, x0, m, n, 1e-9, B, &dim, &tight));
  CHECK(dim == 2 && tight == 2 && B.size() == 6);
  for (int q2 = 0; q2 < 2; ++q2) {
    CHECK(std::abs(B[0 * 2 + q2] + B[1 * 2 + q2] + B[2 * 2 + q2]) < 1e-12);  // in the null space
    double nn = 0.0;
    for (int r = 0; r < 3; ++r) nn += B[r * 2 + q2] * B[r * 2 + q2];
    CHECK(std::abs(nn - 1.0) < 1e-12);
  }
  CHECK(std::abs(B[0] * B[1] + B[2] * B[3] + B[4] * B[5]) < 1e-12);  // orthonormal columns
  std::vector<double> b_loose = {2, 0, 5};
  CHECK(!naja::rounding::affine_hull_basis(A, b_loose, x0, m, n, 1e-9, B, &dim, &tight) && tight == 0);
  if (fails) return 1;
  std::cout << "rounding host ok\n";
  return 0;
}
