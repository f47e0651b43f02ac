// TEST INFRASTRUCTURE ONLY -- C entry points over the reference's own CPU
// validate path (naja::validate::compute_ess / compute_split_rhat from
// src/validate/mcmc.cpp of quothbonney/naja, with the kissfft it vendors in
// extern/kissfft), compiled unmodified from the reference tree by
// oracle/refharness/Makefile.  tests/golden/make_golden.py calls these to
// record golden vectors; nothing in the product links this.
#include <cstring>
#include <exception>
#include <string>

#include "validate/mcmc.h"

namespace {
thread_local std::string g_err;
}

extern "C" {

const char* ref_validate_last_error() { return g_err.c_str(); }

// samples: (dim, n_total) column-major float32, chains concatenated
// [c0 | c1 | ...] -- the reference's layout (mcmc.h).  ess_out: dim values;
// summary_out: min, p10, median, max.
int ref_compute_ess(const float* samples, int dim, int n_total, int n_chains, float* ess_out, float* summary_out) {
  try {
    Eigen::MatrixXf M(dim, n_total);
    std::memcpy(M.data(), samples, sizeof(float) * static_cast<size_t>(dim) * n_total);
    const naja::validate::EssResult r = naja::validate::compute_ess(M, n_chains);
    std::memcpy(ess_out, r.ess.data(), sizeof(float) * static_cast<size_t>(dim));
    summary_out[0] = r.min;
    summary_out[1] = r.p10;
    summary_out[2] = r.median;
    summary_out[3] = r.max;
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

// rhat_out: dim values; summary_out: median, max, above_1_1, above_1_2.
int ref_compute_split_rhat(const float* samples, int dim, int n_total, int n_chains, float* rhat_out,
                           float* summary_out) {
  try {
    Eigen::MatrixXf M(dim, n_total);
    std::memcpy(M.data(), samples, sizeof(float) * static_cast<size_t>(dim) * n_total);
    const naja::validate::RhatResult r = naja::validate::compute_split_rhat(M, n_chains);
    std::memcpy(rhat_out, r.rhat.data(), sizeof(float) * static_cast<size_t>(dim));
    summary_out[0] = r.median;
    summary_out[1] = r.max;
    summary_out[2] = static_cast<float>(r.above_1_1);
    summary_out[3] = static_cast<float>(r.above_1_2);
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}
}
