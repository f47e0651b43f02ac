/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle for the `naja validate` metric path.
 * Only tests/ and bench.py's cpu_baseline leg may load it.
 *
 * Restates src/validate/mcmc.cpp of quothbonney/naja:
 *   - per-series autocovariance acov[k] = (1/n) sum_{t<n-k} (x_t-mean)(x_{t+k}-mean)
 *     (mcmc.cpp:15-57; the reference computes it with a float kissfft of size 2n,
 *     here it is an exact FP64 direct sum, evaluated only for the lags Geyer's
 *     rule reaches)
 *   - Geyer's initial positive sequence: tau = 1 + 2 sum_{k>=1}(rho_{2k-1}+rho_{2k})
 *     stopping at the first negative pair, k < n/2, tau floored at 1,
 *     ESS = n/tau; n < 4 -> n; acov[0] < 1e-30 -> 1 (mcmc.cpp:59-76)
 *   - split-R-hat with Bessel-corrected half-chain variances,
 *     var_hat = (h-1)/h W + B/h, R = sqrt(var_hat/W), W <= 1e-30 -> 1
 *     (mcmc.cpp:126-194), sums in FP64 as in the reference.
 *
 * Layouts of the (N, dim) row-major float32 sample matrix:
 *   layout 0  reference semantics: chain c = rows [c*spc, (c+1)*spc)
 *             (mcmc.cpp:103-109, 148)
 *   layout 1  chain-correct: chain c = rows c, c+nchains, c+2*nchains, ...
 *             (the order the sampler writes, chr.cu:284)
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

static double series_value(const float* s, long N, int dim, int nchains, int layout,
                           int d, int c, long i, long spc) {
    (void)N;
    long row = layout == 0 ? (long)c * spc + i : i * nchains + c;
    return (double)s[row * dim + d];
}

/* Geyer ESS of one series of length n (FP64). */
double oracle_ess_series(const double* x, long n) {
    if (n < 4) return (double)n;
    double mean = 0.0;
    for (long i = 0; i < n; ++i) mean += x[i];
    mean /= (double)n;
    double* y = (double*)malloc(sizeof(double) * n);
    if (!y) return -1.0;
    for (long i = 0; i < n; ++i) y[i] = x[i] - mean;
#define ACOV(k) ({ double _a = 0.0; for (long _t = 0; _t + (k) < n; ++_t) _a += y[_t] * y[_t + (k)]; _a / (double)n; })
    const double var = ACOV(0);
    if (var < 1e-30) { free(y); return 1.0; }
    double tau = 1.0;
    for (long k = 1; k < n / 2; ++k) {
        double pair = ACOV(2 * k - 1) / var + ACOV(2 * k) / var;
        if (pair < 0.0) break;
        tau += 2.0 * pair;
    }
#undef ACOV
    free(y);
    if (tau < 1.0) tau = 1.0;
    return (double)n / tau;
}

/* ESS per (dim, chain): out[d*nchains + c]. */
int oracle_ess(const float* samples, long N, int dim, int nchains, int layout, double* out) {
    if (nchains < 1 || N % nchains != 0) return 1;
    const long spc = N / nchains;
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 1) collapse(2)
    for (int d = 0; d < dim; ++d) {
        for (int c = 0; c < nchains; ++c) {
            double* x = (double*)malloc(sizeof(double) * spc);
            if (!x) { bad = 1; continue; }
            for (long i = 0; i < spc; ++i) x[i] = series_value(samples, N, dim, nchains, layout, d, c, i, spc);
            out[(long)d * nchains + c] = oracle_ess_series(x, spc);
            free(x);
        }
    }
    return bad;
}

/* Split-R-hat per dim. */
int oracle_split_rhat(const float* samples, long N, int dim, int nchains, int layout, double* out) {
    if (nchains < 1 || N % nchains != 0) return 1;
    const long spc = N / nchains;
    const long half = spc / 2;
    if (half < 2) return 2;
    const int m = 2 * nchains;
#pragma omp parallel for schedule(static)
    for (int d = 0; d < dim; ++d) {
        double grand = 0.0, W = 0.0;
        double* means = (double*)malloc(sizeof(double) * m);
        for (int c = 0; c < nchains; ++c) {
            for (int h = 0; h < 2; ++h) {
                double s = 0.0, s2 = 0.0;
                for (long i = 0; i < half; ++i) {
                    double v = series_value(samples, N, dim, nchains, layout, d, c, h * half + i, spc);
                    s += v;
                    s2 += v * v;
                }
                double mean = s / half;
                double var = (s2 / half) - mean * mean;
                var = var * half / (half - 1);
                means[2 * c + h] = mean;
                W += var;
                grand += mean;
            }
        }
        grand /= m;
        double B = 0.0;
        for (int j = 0; j < m; ++j) B += (means[j] - grand) * (means[j] - grand);
        B *= (double)half / (m - 1);
        W /= m;
        double var_hat = ((half - 1.0) / half) * W + B / half;
        out[d] = (W > 1e-30) ? sqrt(var_hat / W) : 1.0;
        free(means);
    }
    return 0;
}
