/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle for the coordinate hit-and-run
 * (CHR) sampler.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg (and its `--impl reference` fallback) may load this file's
 * library; the product path (naja_b200) never links or calls it.
 *
 * It restates, in plain C on the host, the per-step semantics of the
 * reference kernel `chrKernel` (src/gpu/chr.cu:232-490 of quothbonney/naja):
 *
 *   - draw order per step (chr.cu:285-374, 436-437):
 *       ucoord -> ei -> [k-sparse: (idx, sign) x k | pair mode 1: r |
 *       pair mode 2: k, which, sign] -> usample
 *   - clamps of every index draw (chr.cu:294-295, 310-311, 327-329, 338-339)
 *   - inverse-distance rule with the s==0 and NaN cases (chr.cu:420-429)
 *   - alpha = 1/min + u*(1/max - 1/min) (chr.cu:438)
 *   - x update (chr.cu:439-451), save after the update when t%thin==0 into
 *     column chain + (t/thin)*nchains (chr.cu:283-284, 457-461)
 *   - slack update slack -= alpha*ae (chr.cu:463-482)
 *   - optional resync slack = b - A*x every resync_interval steps, t=0
 *     included (chr.cu:386-395)
 *   - persist final x (chr.cu:485-489)
 *
 * Two arithmetic tiers are restated:
 *   precision=1  FP64 throughout (the reference's tier).  Multiply-adds are
 *                written as explicit fma() at the points nvcc contracts in
 *                the reference build (-fmad defaults to true there).
 *   precision=0  the FP32 tier of the new sampler: FP32 A copy, FP32 slack
 *                with negative slack treated as 0 in the ratio, a zero
 *                numerator giving the ratio +0 for any slack, FP32 ratios
 *                and alpha, FP64 position x, FP64 slack recompute
 *                (b - A64*x64, sequential fma over columns) every
 *                resync_interval steps.
 *
 * Uniform sources:
 *   rng=0  Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
 *          numbers: as easy as 1, 2, 3", SC'11), counter
 *          {step_lo, step_hi, chain, draw/4}, key {seed_lo, seed_hi};
 *          draw j of a step is word j%4; u = (word + 1) * 2^-32 in (0, 1].
 *   rng=1  an injected tape of uniforms per chain, consumed in draw order.
 *          The tape is recorded on the GPU by calling cuRAND's
 *          curand_uniform_double on curand_init(seed, chain, 0) states,
 *          which is how the reference seeds its chains (chr.cu:555-560).
 *
 * Slack at t=0 is b - A*x0 with a sequential FP64 fma over columns.  The
 * reference computes it with cublasDgemm (chr.cu:40), whose summation order
 * is not specified; the two agree exactly whenever A*x0 is exact (x0 = 0).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_OK 0
#define ORACLE_EINVAL 1
#define ORACLE_ETAPE 2
#define ORACLE_ENOMEM 3

/* ---------------------------------------------------------------- Philox */

static void philox4x32_10(uint32_t ctr[4], uint32_t k0, uint32_t k1) {
    for (int round = 0; round < 10; ++round) {
        uint64_t p0 = (uint64_t)0xD2511F53u * ctr[0];
        uint64_t p1 = (uint64_t)0xCD9E8D57u * ctr[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ ctr[1] ^ k0;
        uint32_t n2 = hi0 ^ ctr[3] ^ k1;
        ctr[0] = n0; ctr[1] = lo1; ctr[2] = n2; ctr[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

void oracle_philox4x32_10(const uint32_t ctr_in[4], uint32_t k0, uint32_t k1, uint32_t out[4]) {
    uint32_t c[4] = {ctr_in[0], ctr_in[1], ctr_in[2], ctr_in[3]};
    philox4x32_10(c, k0, k1);
    memcpy(out, c, sizeof(c));
}

typedef struct {
    int rng;
    uint64_t seed;
    uint32_t chain;
    uint64_t step;
    int j;
    int blk_id;
    uint32_t blk[4];
    const double* tape;
    long tape_len;
    long pos;
    int overrun;
} draw_src;

static void src_begin_step(draw_src* s, uint64_t step) {
    s->step = step;
    s->j = 0;
    s->blk_id = -1;
}

static double next_u(draw_src* s) {
    if (s->rng == 1) {
        if (s->pos >= s->tape_len) { s->overrun = 1; return 0.5; }
        return s->tape[s->pos++];
    }
    int b = s->j >> 2;
    if (b != s->blk_id) {
        uint32_t c[4] = {(uint32_t)s->step, (uint32_t)(s->step >> 32), s->chain, (uint32_t)b};
        philox4x32_10(c, (uint32_t)s->seed, (uint32_t)(s->seed >> 32));
        memcpy(s->blk, c, sizeof(c));
        s->blk_id = b;
    }
    uint32_t w = s->blk[s->j & 3];
    s->j++;
    return ((double)w + 1.0) * 0x1p-32;
}

/* ------------------------------------------------------------- direction */

enum { KIND_COORD = 0, KIND_PAIR = 1, KIND_KSPARSE = 2 };

typedef struct {
    int kind;
    int ei, ej;
    double ci, cj;
    int k;
    int ks_idx[32];
    double ks_coef[32];
    double u;
} step_dir;

typedef struct {
    int d;
    double pair_prob, ksparse_prob;
    int ksparse_k, pair_mode;
    const int* pi; const int* pj; const double* pc; const double* ps; int n_pairs;
} dir_cfg;

/* chr.cu:285-364 and 436-437, in draw order. */
static void draw_direction(draw_src* s, const dir_cfg* g, step_dir* o) {
    const int cols = g->d;
    double ucoord = next_u(s);
    int want_ks = (g->ksparse_prob > 0.0 && ucoord < g->ksparse_prob) ? 1 : 0;
    int want_pair = (!want_ks && g->pair_prob > 0.0 && ucoord < (g->ksparse_prob + g->pair_prob)) ? 1 : 0;
    int use_pair = want_pair, use_ks = want_ks;
    int ei = (int)(next_u(s) * (double)cols);
    if (ei >= cols) ei = cols - 1;
    int ej = -1;
    double ci = 1.0, cj = 0.0;
    int k = g->ksparse_k;
    if (k < 1) k = 1;
    if (k > 32) k = 32;
    if (k > cols) k = cols;
    if (use_ks) {
        const double inv_sqrt_k = 1.0 / sqrt((double)k);
        for (int t = 0; t < k; ++t) {
            int idx = (int)(next_u(s) * (double)cols);
            if (idx >= cols) idx = cols - 1;
            const double sign = (next_u(s) < 0.5) ? 1.0 : -1.0;
            o->ks_idx[t] = idx;
            o->ks_coef[t] = sign * inv_sqrt_k;
        }
    }
    if (use_pair) {
        if (cols < 2) {
            use_pair = 0;
        } else if (g->pair_mode == 1) {
            int r = (int)(next_u(s) * (double)(cols - 1));
            if (r >= cols - 1) r = cols - 2;
            ej = (r >= ei) ? (r + 1) : r;
            ci = 0.70710678118654752440;
            cj = -0.70710678118654752440;
        } else if (g->pair_mode == 2) {
            if (g->n_pairs <= 0 || !g->pi || !g->pj || !g->pc || !g->ps) {
                use_pair = 0;
            } else {
                int kk = (int)(next_u(s) * (double)g->n_pairs);
                if (kk >= g->n_pairs) kk = g->n_pairs - 1;
                ei = g->pi[kk];
                ej = g->pj[kk];
                double c = g->pc[kk], sn = g->ps[kk];
                int which = (next_u(s) < 0.5) ? 0 : 1;
                if (which == 0) { ci = c; cj = sn; } else { ci = -sn; cj = c; }
                double sign = (next_u(s) < 0.5) ? 1.0 : -1.0;
                ci *= sign;
                cj *= sign;
            }
        } else {
            use_pair = 0;
        }
    }
    o->kind = use_ks ? KIND_KSPARSE : (use_pair ? KIND_PAIR : KIND_COORD);
    o->ei = ei; o->ej = ej; o->ci = ci; o->cj = cj; o->k = k;
    o->u = next_u(s);
}

/* -------------------------------------------------------- ordered compare */
/* Maximum / minimum under the total order of IEEE values in which
 * -0 < +0 (values here are never NaN).  Bit-equivalent to an exact
 * max/min reduction in any order. */

static inline uint64_t key64(double v) {
    uint64_t u; memcpy(&u, &v, 8);
    return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
static inline uint32_t key32(float v) {
    uint32_t u; memcpy(&u, &v, 4);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

/* ------------------------------------------------------------- one chain */

typedef struct {
    int m, d, lda;
    const double* A;
    const float* A32;
    const double* b;
    int nspc, thinning, nchains, resync;
    int precision;
    int pair_variant; /* 0: fma(ai,ci,aj*cj) 1: fma(aj,cj,ai*ci) 2: ai*ci+aj*cj */
    dir_cfg g;
} run_cfg;

static inline double ae64(const run_cfg* c, const step_dir* dir, int r) {
    const double* A = c->A;
    const long lda = c->lda;
    if (dir->kind == KIND_KSPARSE) {
        double acc = 0.0;
        for (int t = 0; t < dir->k; ++t) acc = fma(A[r + dir->ks_idx[t] * lda], dir->ks_coef[t], acc);
        return acc;
    }
    if (dir->kind == KIND_COORD) return A[r + dir->ei * lda];
    const double ai = A[r + dir->ei * lda], aj = A[r + dir->ej * lda];
    if (c->pair_variant == 0) return fma(ai, dir->ci, aj * dir->cj);
    if (c->pair_variant == 1) return fma(aj, dir->cj, ai * dir->ci);
    return ai * dir->ci + aj * dir->cj;
}

static inline float ae32(const run_cfg* c, const step_dir* dir, int r) {
    const float* A = c->A32;
    const long lda = c->lda;
    if (dir->kind == KIND_KSPARSE) {
        float acc = 0.0f;
        for (int t = 0; t < dir->k; ++t) acc = fmaf(A[r + dir->ks_idx[t] * lda], (float)dir->ks_coef[t], acc);
        return acc;
    }
    if (dir->kind == KIND_COORD) return A[r + dir->ei * lda];
    const float ai = A[r + dir->ei * lda], aj = A[r + dir->ej * lda];
    return fmaf(ai, (float)dir->ci, aj * (float)dir->cj);
}

static void recompute_slack64(const run_cfg* c, const double* x, double* slack) {
    for (int r = 0; r < c->m; ++r) {
        double acc = 0.0;
        for (int j = 0; j < c->d; ++j) acc = fma(c->A[r + (long)j * c->lda], x[j], acc);
        slack[r] = c->b[r] - acc;
    }
}

static int run_chain(const run_cfg* c, int chain, draw_src* src, uint64_t step_offset,
                     double* x, double* samples, int* trace) {
    const int m = c->m, d = c->d;
    const long total = (long)c->nspc * c->thinning;
    double* s64 = NULL;
    float* s32 = NULL;
    double* aes64 = NULL;
    float* aes32 = NULL;
    if (c->precision == 1) {
        s64 = (double*)malloc(sizeof(double) * m);
        aes64 = (double*)malloc(sizeof(double) * m);
        if (!s64 || !aes64) { free(s64); free(aes64); return ORACLE_ENOMEM; }
        recompute_slack64(c, x, s64);
    } else {
        s64 = (double*)malloc(sizeof(double) * m);
        s32 = (float*)malloc(sizeof(float) * m);
        aes32 = (float*)malloc(sizeof(float) * m);
        if (!s64 || !s32 || !aes32) { free(s64); free(s32); free(aes32); return ORACLE_ENOMEM; }
        recompute_slack64(c, x, s64);
        for (int r = 0; r < m; ++r) s32[r] = (float)s64[r];
    }
    step_dir dir;
    for (long t = 0; t < total; ++t) {
        src_begin_step(src, step_offset + (uint64_t)t);
        draw_direction(src, &c->g, &dir);
        if (trace) {
            trace[2 * t + 0] = dir.ei;
            trace[2 * t + 1] = (dir.kind == KIND_PAIR) ? dir.ej : (dir.kind == KIND_KSPARSE ? -2 : -1);
        }
        if (c->resync > 0 && (t % c->resync) == 0) {
            recompute_slack64(c, x, s64);
            if (c->precision == 0)
                for (int r = 0; r < m; ++r) s32[r] = (float)s64[r];
        }
        if (c->precision == 1) {
            uint64_t kmax = key64(-DBL_MAX), kmin = key64(DBL_MAX);
            for (int r = 0; r < m; ++r) {
                const double s = s64[r];
                const double ae = ae64(c, &dir, r);
                aes64[r] = ae;
                double inv;
                if (s == 0.0) {
                    inv = (ae > 0.0) ? INFINITY : ((ae < 0.0) ? -INFINITY : 0.0);
                } else {
                    inv = ae / s;
                    if (isnan(inv)) inv = 0.0;
                }
                uint64_t kv = key64(inv);
                if (kv > kmax) kmax = kv;
                if (kv < kmin) kmin = kv;
            }
            double mx, mn;
            {
                uint64_t u = (kmax & 0x8000000000000000ull) ? (kmax & 0x7fffffffffffffffull) : ~kmax;
                memcpy(&mx, &u, 8);
                u = (kmin & 0x8000000000000000ull) ? (kmin & 0x7fffffffffffffffull) : ~kmin;
                memcpy(&mn, &u, 8);
            }
            const double lo = 1.0 / mn, hi = 1.0 / mx;
            const double alpha = fma(dir.u, hi - lo, lo);
            if (dir.kind == KIND_KSPARSE) {
                for (int q = 0; q < dir.k; ++q) x[dir.ks_idx[q]] = fma(alpha, dir.ks_coef[q], x[dir.ks_idx[q]]);
            } else if (dir.kind == KIND_COORD) {
                x[dir.ei] = x[dir.ei] + alpha;
            } else {
                x[dir.ei] = fma(alpha, dir.ci, x[dir.ei]);
                x[dir.ej] = fma(alpha, dir.cj, x[dir.ej]);
            }
            if (t % c->thinning == 0) {
                double* out = samples + ((long)(t / c->thinning) * c->nchains + chain) * (long)d;
                memcpy(out, x, sizeof(double) * d);
            }
            for (int r = 0; r < m; ++r) s64[r] = fma(-alpha, aes64[r], s64[r]);
        } else {
            uint32_t kmax = key32(-FLT_MAX), kmin = key32(FLT_MAX);
            for (int r = 0; r < m; ++r) {
                float s = s32[r];
                if (s < 0.0f) s = 0.0f;
                const float ae = ae32(c, &dir, r);
                aes32[r] = ae;
                float inv;
                if (ae == 0.0f) {
                    inv = 0.0f; /* the FP32 tier's zero numerator: +0 */
                } else if (s == 0.0f) {
                    inv = (ae > 0.0f) ? INFINITY : -INFINITY;
                } else {
                    inv = ae / s;
                }
                uint32_t kv = key32(inv);
                if (kv > kmax) kmax = kv;
                if (kv < kmin) kmin = kv;
            }
            float mx, mn;
            {
                uint32_t u = (kmax & 0x80000000u) ? (kmax & 0x7fffffffu) : ~kmax;
                memcpy(&mx, &u, 4);
                u = (kmin & 0x80000000u) ? (kmin & 0x7fffffffu) : ~kmin;
                memcpy(&mn, &u, 4);
            }
            const float lo = 1.0f / mn, hi = 1.0f / mx;
            const float alpha = fmaf((float)dir.u, hi - lo, lo);
            const double a64 = (double)alpha;
            if (dir.kind == KIND_KSPARSE) {
                for (int q = 0; q < dir.k; ++q)
                    x[dir.ks_idx[q]] = fma(a64, (double)(float)dir.ks_coef[q], x[dir.ks_idx[q]]);
            } else if (dir.kind == KIND_COORD) {
                x[dir.ei] = x[dir.ei] + a64;
            } else {
                x[dir.ei] = fma(a64, (double)(float)dir.ci, x[dir.ei]);
                x[dir.ej] = fma(a64, (double)(float)dir.cj, x[dir.ej]);
            }
            if (t % c->thinning == 0) {
                double* out = samples + ((long)(t / c->thinning) * c->nchains + chain) * (long)d;
                memcpy(out, x, sizeof(double) * d);
            }
            for (int r = 0; r < m; ++r) s32[r] = fmaf(-alpha, aes32[r], s32[r]);
        }
        if (src->overrun) break;
    }
    free(s64); free(s32); free(aes64); free(aes32);
    return src->overrun ? ORACLE_ETAPE : ORACLE_OK;
}

/* ------------------------------------------------------------------ API */

/*
 * Runs nchains chains of CHR.  A is m x d column-major with leading
 * dimension lda; X0 is d x nchains column-major with leading dimension ldx.
 * samples (nspc*nchains rows of d, row-major) receives the saved states,
 * row = sample*nchains + chain, which is the reference's column order
 * (chr.cu:284, 460).  X_final (nullable) receives the final state of each
 * chain (d x nchains, leading dimension ldx).  trace (nullable) receives
 * (ei, ej) per chain per step, ej = -1 for a coordinate step and -2 for a
 * k-sparse step.  Returns 0 on success.
 */
int oracle_chr_run(int m, int d, const double* A, int lda, const double* b,
                   const double* X0, int ldx,
                   int nspc, int thinning, int nchains,
                   uint64_t seed, double pair_prob, int resync_interval,
                   double ksparse_prob, int ksparse_k, int pair_mode,
                   const int* pair_i, const int* pair_j,
                   const double* pair_c, const double* pair_s, int n_pairs,
                   int precision, int rng,
                   const double* tape, long tape_stride,
                   uint64_t step_offset, int pair_variant,
                   double* samples, double* X_final, int* trace, int nthreads) {
    if (m <= 0 || d <= 0 || lda < m || ldx < d || nspc <= 0 || thinning <= 0 || nchains <= 0)
        return ORACLE_EINVAL;
    if (rng == 1 && (!tape || tape_stride <= 0)) return ORACLE_EINVAL;
    run_cfg c;
    memset(&c, 0, sizeof(c));
    c.m = m; c.d = d; c.lda = lda; c.A = A; c.b = b;
    c.nspc = nspc; c.thinning = thinning; c.nchains = nchains;
    c.resync = resync_interval; c.precision = precision; c.pair_variant = pair_variant;
    c.g.d = d; c.g.pair_prob = pair_prob; c.g.ksparse_prob = ksparse_prob;
    c.g.ksparse_k = ksparse_k; c.g.pair_mode = pair_mode;
    c.g.pi = pair_i; c.g.pj = pair_j; c.g.pc = pair_c; c.g.ps = pair_s; c.g.n_pairs = n_pairs;
    float* A32 = NULL;
    if (precision == 0) {
        A32 = (float*)malloc(sizeof(float) * (size_t)lda * d);
        if (!A32) return ORACLE_ENOMEM;
        for (size_t i = 0; i < (size_t)lda * d; ++i) A32[i] = (float)A[i];
        c.A32 = A32;
    }
    const long total = (long)nspc * thinning;
    int status = ORACLE_OK;
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1) reduction(max : status)
    for (int ch = 0; ch < nchains; ++ch) {
        double* x = (double*)malloc(sizeof(double) * d);
        if (!x) { status = ORACLE_ENOMEM; continue; }
        memcpy(x, X0 + (long)ch * ldx, sizeof(double) * d);
        draw_src src;
        memset(&src, 0, sizeof(src));
        src.rng = rng; src.seed = seed; src.chain = (uint32_t)ch;
        if (rng == 1) { src.tape = tape + (long)ch * tape_stride; src.tape_len = tape_stride; }
        int st = run_chain(&c, ch, &src, step_offset, x, samples, trace ? trace + (long)ch * total * 2 : NULL);
        if (st > status) status = st;
        if (X_final) memcpy(X_final + (long)ch * ldx, x, sizeof(double) * d);
        free(x);
    }
    free(A32);
    return status;
}

/* Number of uniforms a chain consumes over `steps` steps given the same
 * configuration (used to size a recorded tape). */
long oracle_draws_needed(int d, long steps, uint64_t seed, int chain, double pair_prob,
                         double ksparse_prob, int ksparse_k, int pair_mode, int n_pairs) {
    (void)seed; (void)chain;
    /* Upper bound: every step a k-sparse or mode-2 pair draw. */
    int k = ksparse_k < 1 ? 1 : (ksparse_k > 32 ? 32 : ksparse_k);
    if (k > d) k = d;
    long per = 3;
    if (ksparse_prob > 0.0) per += 2 * k;
    if (pair_prob > 0.0) per += (pair_mode == 2 && n_pairs > 0) ? 3 : 1;
    return per * steps;
}
