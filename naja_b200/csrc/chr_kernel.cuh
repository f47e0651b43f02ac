// Multi-chain coordinate hit-and-run step kernel for sm_100a.
//
// Semantics follow the reference kernel chrKernel (src/gpu/chr.cu:232-490 of
// quothbonney/naja): per step a direction (coordinate e_i, pair
// (e_i - e_j)/sqrt 2 or a Jacobi pair, or a k-sparse direction) is drawn in
// the reference's order, the chord through x is bounded by max/min over
// rows of ae/s (s = slack, ae = A u) with the s == 0 and NaN rules of
// chr.cu:420-429, alpha = 1/min + u (1/max - 1/min), x += alpha u, the state
// is saved every `thinning` steps after the update, and slack -= alpha ae.
//
// The B200 organisation differs from the reference:
//   * One CTA per chain = NT consumer threads + 1 producer warp.
//   * The direction of a step never depends on the chain's state, so the
//     producer thread draws the RNG up to `slots` steps ahead and streams the
//     A columns those steps need into a ring of shared-memory slots with
//     1-D bulk copies (cp.async.bulk) that complete on per-slot mbarriers.
//     The consumers find the column already on chip.
//   * The slack vector lives in the consumers' registers (warp w owns the
//     32 V-row chunks w, w + NW, ..., lane l the V consecutive rows at
//     l V of each), so the only memory traffic per step is one column of A
//     (two for a pair step) plus the amortised sample write, read with
//     vector accesses.
//   * max/min run on the integer reduction unit (redux.sync) over
//     order-preserving keys, then across warps through a double-buffered
//     shared array and one named barrier per step: exact in any order.
//   * x is kept in FP64 in shared memory; entry j is only ever touched by
//     consumer thread j % NT, so updates and saves need no barrier.
//   * FP32 tier: FP32 A copy, FP32 slack (a negative slack counts as 0 in
//     the ratio), FP32 ratios and alpha, FP64 x, and an FP64 recompute
//     slack = b - A64 x every `resync` steps (the reference's
//     resync_interval hook, chr.cu:384-395).  FP64 tier: the reference's
//     arithmetic, with fma at the points nvcc contracts in the reference.
//   * Every spin-wait is bounded by the global timer; on expiry the kernel
//     records an error code, drains its own copies and returns.
#pragma once
#include <curand_kernel.h>

#include <algorithm>

#include "chr.cuh"
#include "common.cuh"
#include "../../include/naja_chr.h"

namespace naja {
namespace chr_detail {
namespace {

// One step's record in the ring.  The first 32 bytes are what the FP32 tier
// reads every step (two 16-byte loads): the direction, and its coefficients
// and alpha uniform rounded to float once by the producer.
struct __align__(16) StepMeta {
  int kind;
  int ei;
  int ej;
  int slot_b;
  int k;
  float cif;
  float cjf;
  float uf;
  double ci;
  double cj;
  double u;
  int na;  // sparse-column kernel: entries staged in slot_a / slot_b
  int nb;
  int ks_idx[32];
  double ks_coef[32];
};

// One step's direction as the producer draws it (register-resident; the
// k-sparse index/coefficient lists live in small local arrays).
struct StepDir {
  int kind;
  int ei;
  int ej;
  int k;
  double ci;
  double cj;
  double u;
};

struct RedEntry {
  unsigned long long kmax;
  unsigned long long kmin;
  unsigned long long kmin2;
  int abort;
  int pad;
};

constexpr size_t kSmemBudget = 227 * 1024;
constexpr int kMaxSlots = 8;

__host__ __device__ inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

struct Layout {
  size_t x_off, slot_off, slot_bytes, meta_off, full_off, empty_off, red_off, flag_off, tail_off, slack_off, total;
  int slots;
  bool direct;
  // sparse-column kernel only: column offsets and the pair-step scratch column
  size_t cs_off, ajd_off;
};

// slack_rows > 0 reserves a shared-memory slack store (slack_rows values of
// `elt` bytes) for kernels that keep slack on chip outside the registers.
__host__ __device__ inline Layout make_layout(int d, int lda, int elt, int nthreads, int slots_req,
                                              int slack_rows = 0) {
  Layout L;
  const int nw = nthreads / 32;
  const bool direct = slots_req <= 0;
  const int S = direct ? kMaxSlots : slots_req;
  size_t off = 0;
  L.x_off = off;
  off = align_up(off + static_cast<size_t>(d) * 8, 128);
  L.slot_off = off;
  L.slot_bytes = direct ? 0 : align_up(static_cast<size_t>(lda) * elt, 128);
  off += L.slot_bytes * S;
  L.meta_off = off;
  off = align_up(off + sizeof(StepMeta) * S, 16);
  L.full_off = off;
  off += 8 * S;
  L.empty_off = off;
  off += 8 * S;
  L.red_off = off;
  off = align_up(off + sizeof(RedEntry) * 2 * nw, 16);
  L.flag_off = off;
  off += 16;
  // slack of the rows of the partial chunk at the end of the rows (at most
  // one chunk of 32 * 4 values) when the full chunks keep theirs in registers
  L.tail_off = align_up(off, 16);
  off = L.tail_off + 128 * static_cast<size_t>(elt);
  L.slack_off = align_up(off, 128);
  if (slack_rows > 0) off = L.slack_off + static_cast<size_t>(slack_rows) * elt;
  L.total = align_up(off, 128);
  L.slots = S;
  L.direct = direct;
  L.cs_off = L.ajd_off = 0;
  return L;
}

// -------------------------------------------------------------- RNG sources
struct PhiloxSource {
  uint32_t k0, k1, chain;
  uint64_t step;
  int j, blk_id;
  Philox4 blk;
  __device__ void begin_step(uint64_t s) {
    step = s;
    j = 0;
    blk_id = -1;
  }
  __device__ double next() {
    const int b = j >> 2;
    if (b != blk_id) {
      blk = philox4x32_10(static_cast<uint32_t>(step), static_cast<uint32_t>(step >> 32), chain,
                          static_cast<uint32_t>(b), k0, k1);
      blk_id = b;
    }
    const uint32_t w = blk.v[j & 3];
    ++j;
    return u01_from_word(w);
  }
};

struct MrgSource {
  curandStateMRG32k3a st;
  __device__ void begin_step(uint64_t) {}
  __device__ double next() { return curand_uniform_double(&st); }
};

// Draws one step's direction in the reference's order (chr.cu:285-364),
// then the alpha uniform (chr.cu:437).  Returns false on a bad pair index.
template <class Src>
__device__ bool draw_direction(Src& src, const ChrArgs& a, StepDir& o, int* ks_idx, double* ks_coef) {
  const int cols = a.d;
  const double ucoord = src.next();
  const int want_ks = (a.ksparse_prob > 0.0 && ucoord < a.ksparse_prob) ? 1 : 0;
  const int want_pair = (!want_ks && a.pair_prob > 0.0 && ucoord < (a.ksparse_prob + a.pair_prob)) ? 1 : 0;
  int use_pair = want_pair;
  const int use_ks = want_ks;
  int ei = static_cast<int>(src.next() * static_cast<double>(cols));
  if (ei >= cols) ei = cols - 1;
  int ej = -1;
  double ci = 1.0, cj = 0.0;
  int k = a.ksparse_k;
  if (k < 1) k = 1;
  if (k > 32) k = 32;
  if (k > cols) k = cols;
  if (use_ks) {
    const double inv_sqrt_k = 1.0 / sqrt(static_cast<double>(k));
    for (int t = 0; t < k; ++t) {
      int idx = static_cast<int>(src.next() * static_cast<double>(cols));
      if (idx >= cols) idx = cols - 1;
      const double sign = (src.next() < 0.5) ? 1.0 : -1.0;
      ks_idx[t] = idx;
      ks_coef[t] = __dmul_rn(sign, inv_sqrt_k);
    }
  }
  bool ok = true;
  if (use_pair) {
    if (cols < 2) {
      use_pair = 0;
    } else if (a.pair_mode == 1) {
      int r = static_cast<int>(src.next() * static_cast<double>(cols - 1));
      if (r >= cols - 1) r = cols - 2;
      ej = (r >= ei) ? (r + 1) : r;
      ci = 0.70710678118654752440;
      cj = -0.70710678118654752440;
    } else if (a.pair_mode == 2) {
      if (a.n_pairs <= 0 || !a.pair_i || !a.pair_j || !a.pair_c || !a.pair_s) {
        use_pair = 0;
      } else {
        int kk = static_cast<int>(src.next() * static_cast<double>(a.n_pairs));
        if (kk >= a.n_pairs) kk = a.n_pairs - 1;
        ei = a.pair_i[kk];
        ej = a.pair_j[kk];
        const double c = a.pair_c[kk], s = a.pair_s[kk];
        const int which = (src.next() < 0.5) ? 0 : 1;
        if (which == 0) {
          ci = c;
          cj = s;
        } else {
          ci = -s;
          cj = c;
        }
        const double sign = (src.next() < 0.5) ? 1.0 : -1.0;
        ci = __dmul_rn(ci, sign);
        cj = __dmul_rn(cj, sign);
        ok = (ei >= 0 && ei < cols && ej >= 0 && ej < cols);
      }
    } else {
      use_pair = 0;
    }
  }
  o.kind = use_ks ? kKSparse : (use_pair ? kPair : kCoord);
  o.ei = ok ? ei : 0;
  o.ej = ok ? ej : 0;
  o.ci = ci;
  o.cj = cj;
  o.k = k;
  o.u = src.next();
  return ok;
}

template <class Real>
struct Tier;

template <>
struct Tier<float> {
  using Key = uint32_t;
  __device__ static Key key(float v) { return fkey(v); }
  __device__ static float unkey(Key k) { return fkey_inv(k); }
  __device__ static Key wmax(Key k) { return __reduce_max_sync(0xffffffffu, k); }
  __device__ static Key wmin(Key k) { return __reduce_min_sync(0xffffffffu, k); }
  __device__ static float lowest() { return -3.402823466e+38f; }
  __device__ static float highest() { return 3.402823466e+38f; }
  __device__ static const float* A(const ChrArgs& a) { return a.A32; }
  __device__ static float pair_ae_r(float ai, float aj, float ci, float cj) {
    return __fmaf_rn(ai, ci, __fmul_rn(aj, cj));
  }
  __device__ static float ks_acc(float acc, float av, double coef) {
    return __fmaf_rn(av, static_cast<float>(coef), acc);
  }
  // Ratio ae/s of the FP32 tier: a negative slack counts as 0 (it can only
  // come from FP32 rounding), so a nonzero ae over zero slack is +-inf (the
  // reference's s == 0 rule, chr.cu:420-429), and a zero ae gives +0 whatever
  // the slack.  A nonzero ae over a finite slack >= +0 is never NaN.  The
  // zero numerator is replaced by 1 before dividing: most rows of a sparse A
  // are zero and a division of zero leaves the division's fast path.
  // The clamp is one signed-integer max on the bit pattern: every value with
  // the sign bit set, -0 included, becomes +0.
  __device__ static float ratio(float ae, float s) {
    s = __int_as_float(max(__float_as_int(s), 0));
    const bool z = (ae == 0.0f);
    const float q = __fdiv_rn(z ? 1.0f : ae, s);
    return z ? 0.0f : q;
  }
  // Running extremes on the raw bit patterns (ratios are never NaN), exact
  // in the key order -0 < +0 without transforming each value:
  //   hi  = signed-integer max: the largest ratio whenever some ratio has a
  //         clear sign bit (integer order is float order there, and every
  //         such value is above every value with the sign bit set);
  //   lo  = unsigned max: the most negative ratio whenever some ratio has its
  //         sign bit set (the magnitude grows with the unsigned value);
  //   lo2 = unsigned min: the largest ratio when all have the sign bit set
  //         (smallest magnitude), the smallest when none has.
  using Acc = uint32_t;
  __device__ static Acc acc_hi0() { return 0x80000000u; }
  __device__ static Acc acc_lo0() { return 0u; }
  __device__ static Acc acc_lo20() { return 0xffffffffu; }
  __device__ static void acc(Acc& hi, Acc& lo, Acc& lo2, float v) {
    const uint32_t b = __float_as_uint(v);
    hi = static_cast<uint32_t>(max(static_cast<int>(hi), static_cast<int>(b)));
    lo = max(lo, b);
    lo2 = min(lo2, b);
  }
  __device__ static Acc red_hi(Acc v) {
    return static_cast<uint32_t>(__reduce_max_sync(0xffffffffu, static_cast<int>(v)));
  }
  __device__ static Acc red_lo(Acc v) { return __reduce_max_sync(0xffffffffu, v); }
  __device__ static Acc red_lo2(Acc v) { return __reduce_min_sync(0xffffffffu, v); }
  __device__ static void decode(Acc hi, Acc lo, Acc lo2, float& mx, float& mn) {
    mx = __uint_as_float(static_cast<int>(hi) >= 0 ? hi : lo2);
    mn = __uint_as_float(lo >= 0x80000000u ? lo : lo2);
  }
  using UType = float;
  __device__ static float alpha(float mx, float mn, float u) {
    const float lo = __fdiv_rn(1.0f, mn), hi = __fdiv_rn(1.0f, mx);
    return __fmaf_rn(u, __fsub_rn(hi, lo), lo);
  }
  __device__ static double coef(double c) { return static_cast<double>(static_cast<float>(c)); }
  __device__ static float slack_update(float s, float alpha, float ae) { return __fmaf_rn(-alpha, ae, s); }
  __device__ static float from64(double v) { return __double2float_rn(v); }
};

template <>
struct Tier<double> {
  using Key = unsigned long long;
  __device__ static Key key(double v) { return dkey(v); }
  __device__ static double unkey(Key k) { return dkey_inv(k); }
  __device__ static Key wmax(Key k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const Key q = __shfl_xor_sync(0xffffffffu, k, o);
      k = q > k ? q : k;
    }
    return k;
  }
  __device__ static Key wmin(Key k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const Key q = __shfl_xor_sync(0xffffffffu, k, o);
      k = q < k ? q : k;
    }
    return k;
  }
  __device__ static double lowest() { return -1.7976931348623157e+308; }
  __device__ static double highest() { return 1.7976931348623157e+308; }
  __device__ static const double* A(const ChrArgs& a) { return a.A64; }
  __device__ static double pair_ae_r(double ai, double aj, double ci, double cj) {
    return __fma_rn(ai, ci, __dmul_rn(aj, cj));
  }
  __device__ static double ks_acc(double acc, double av, double coef) { return __fma_rn(av, coef, acc); }
  // s == 0 of either sign becomes +0: ae/+0 = +-inf, 0/0 = NaN -> 0, the
  // reference's rule (chr.cu:420-429); negative slack divides as it is.
  // A nonzero ae over a finite slack is never NaN, so the NaN -> 0 rule only
  // concerns 0/0, answered by the zero-numerator branch.
  __device__ static double ratio(double ae, double s) {
    s = (s == 0.0) ? 0.0 : s;
    const bool z = (ae == 0.0);
    const double q = __ddiv_rn(z ? 1.0 : ae, z ? 1.0 : s);
    return z ? ((s > 0.0) ? ae : ((s < 0.0) ? -ae : 0.0)) : q;
  }
  // Extremes over order-preserving keys (exact in any order); lo2 unused.
  using Acc = unsigned long long;
  __device__ static Acc acc_hi0() { return dkey(lowest()); }
  __device__ static Acc acc_lo0() { return dkey(highest()); }
  __device__ static Acc acc_lo20() { return 0ull; }
  __device__ static void acc(Acc& hi, Acc& lo, Acc&, double v) {
    const Acc kv = dkey(v);
    hi = kv > hi ? kv : hi;
    lo = kv < lo ? kv : lo;
  }
  __device__ static Acc red_hi(Acc v) { return wmax(v); }
  __device__ static Acc red_lo(Acc v) { return wmin(v); }
  __device__ static Acc red_lo2(Acc v) { return v; }
  __device__ static void decode(Acc hi, Acc lo, Acc, double& mx, double& mn) {
    mx = dkey_inv(hi);
    mn = dkey_inv(lo);
  }
  using UType = double;
  __device__ static double alpha(double mx, double mn, double u) {
    const double lo = __ddiv_rn(1.0, mn), hi = __ddiv_rn(1.0, mx);
    return __fma_rn(u, __dsub_rn(hi, lo), lo);
  }
  __device__ static double coef(double c) { return c; }
  __device__ static double slack_update(double s, double alpha, double ae) { return __fma_rn(-alpha, ae, s); }
  __device__ static double from64(double v) { return v; }
};


// Steps of one launch (ChrArgs::t_first, ChrArgs::steps).
__device__ __forceinline__ long long launch_steps(const ChrArgs& a) {
  return a.steps > 0 ? a.steps : static_cast<long long>(a.nspc) * a.thinning;
}

// ------------------------------------------------------------------ producer
// One thread: draws each step's direction ahead of the consumers, claims one
// ring slot per staged column (two for a pair step, one metadata-only slot
// for a k-sparse step), writes the step record and starts the bulk copy.
// SPARSE: the slot receives the column's compressed entries (offsets from
// the shared copy `cs` of col_start, entry size `eb`) and the record their
// count.
template <class Real, class Src, bool SPARSE = false>
__device__ __noinline__ void run_producer(const ChrArgs& a, Src& src, const Layout& L, unsigned char* smem,
                                          const SpArgs* sp = nullptr, const int* cs = nullptr, int eb = 0) {
  StepMeta* meta = reinterpret_cast<StepMeta*>(smem + L.meta_off);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.full_off);
  uint64_t* empty = reinterpret_cast<uint64_t*>(smem + L.empty_off);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + L.flag_off);
  const Real* A = Tier<Real>::A(a);
  const uint32_t col_bytes = static_cast<uint32_t>(align_up(static_cast<size_t>(a.m) * sizeof(Real), 16));
  const int S = L.slots;
  const long long total = launch_steps(a);
  // Slots are claimed round-robin.  `slot` is the next one, `round` how many
  // times the ring has wrapped: a slot's use number is the round it is
  // claimed in, its fill waits for the empty-barrier phase of round - 1.
  int slot = 0;
  uint32_t round = 0;
  uint32_t used_mask = 0, last_parity = 0;  // per slot: used at all / parity of its last use
  StepDir dir;
  int ks_idx[32];
  double ks_coef[32];
  unsigned long long w_empty = 0;
  const unsigned long long p_start = clock64();
  for (long long t = 0; t < total; ++t) {
    if (*abort_flag) break;
    src.begin_step(static_cast<uint64_t>(a.step_offset + a.t_first + t));
    if (!draw_direction(src, a, dir, ks_idx, ks_coef)) {
      set_error(a.err, kDevBadPair, dir.ei, dir.ej, static_cast<int>(t));
      *abort_flag = 1;
      break;
    }
    const int sa = slot;
    const uint32_t ra = round;
    if (++slot == S) {
      slot = 0;
      ++round;
    }
    const unsigned long long w0 = a.wait_cycles ? clock64() : 0ull;
    if (ra >= 1 && !mbar_wait_bounded_sleep(&empty[sa], (ra - 1) & 1u, a.timeout_ns, 64)) {
      set_error(a.err, kDevTimeoutEmpty, sa, static_cast<int>(ra), static_cast<int>(t));
      *abort_flag = 1;
      break;
    }
    if (a.wait_cycles) w_empty += clock64() - w0;
    int sb = -1;
    uint32_t rb = 0;
    if (dir.kind == kPair) {
      sb = slot;
      rb = round;
      if (++slot == S) {
        slot = 0;
        ++round;
      }
      if (rb >= 1 && !mbar_wait_bounded_sleep(&empty[sb], (rb - 1) & 1u, a.timeout_ns, 64)) {
        set_error(a.err, kDevTimeoutEmpty, sb, static_cast<int>(rb), static_cast<int>(t));
        *abort_flag = 1;
        break;
      }
    }
    StepMeta& M = meta[sa];
    M.kind = dir.kind;
    M.ei = dir.ei;
    M.ej = dir.ej;
    M.slot_b = sb;
    M.ci = dir.ci;
    M.cj = dir.cj;
    M.u = dir.u;
    M.k = dir.k;
    M.cif = static_cast<float>(dir.ci);
    M.cjf = static_cast<float>(dir.cj);
    M.uf = static_cast<float>(dir.u);
    if (dir.kind == kKSparse) {
      for (int q = 0; q < dir.k; ++q) {
        M.ks_idx[q] = ks_idx[q];
        M.ks_coef[q] = ks_coef[q];
      }
    }
    // The drain below waits for the full-barrier phase of each slot's most
    // recent use, whatever its kind, so every use is recorded here.
    used_mask |= 1u << sa;
    last_parity = (last_parity & ~(1u << sa)) | ((ra & 1u) << sa);
    if (sb >= 0) {
      used_mask |= 1u << sb;
      last_parity = (last_parity & ~(1u << sb)) | ((rb & 1u) << sb);
    }
    if constexpr (SPARSE) {
      // every column holds at least one 16-byte group of entries
      const unsigned char* cols = static_cast<const unsigned char*>(sp->cols);
      const int s0 = cs[dir.ei], n0 = cs[dir.ei + 1] - s0;
      M.na = n0;
      M.nb = 0;
      if (sb >= 0) M.nb = cs[dir.ej + 1] - cs[dir.ej];
      mbar_arrive_expect_tx(&full[sa], static_cast<uint32_t>(n0 * eb));
      bulk_g2s(smem + L.slot_off + static_cast<size_t>(sa) * L.slot_bytes, cols + static_cast<size_t>(s0) * eb,
               static_cast<uint32_t>(n0 * eb), &full[sa]);
      if (sb >= 0) {
        const int s1 = cs[dir.ej];
        mbar_arrive_expect_tx(&full[sb], static_cast<uint32_t>(M.nb * eb));
        bulk_g2s(smem + L.slot_off + static_cast<size_t>(sb) * L.slot_bytes, cols + static_cast<size_t>(s1) * eb,
                 static_cast<uint32_t>(M.nb * eb), &full[sb]);
      }
    } else if (!L.direct && dir.kind != kKSparse) {
      mbar_arrive_expect_tx(&full[sa], col_bytes);
      bulk_g2s(smem + L.slot_off + static_cast<size_t>(sa) * L.slot_bytes, A + static_cast<size_t>(dir.ei) * a.lda,
               col_bytes, &full[sa]);
      if (sb >= 0) {
        mbar_arrive_expect_tx(&full[sb], col_bytes);
        bulk_g2s(smem + L.slot_off + static_cast<size_t>(sb) * L.slot_bytes,
                 A + static_cast<size_t>(dir.ej) * a.lda, col_bytes, &full[sb]);
      }
    } else {
      mbar_arrive(&full[sa]);
      if (sb >= 0) mbar_arrive(&full[sb]);
    }
  }
  if (a.wait_cycles) {
    a.wait_cycles[4 * (blockIdx.x) + 1] = w_empty;
    a.wait_cycles[4 * (blockIdx.x) + 3] = clock64() - p_start;
  }
  // Drain: never leave the CTA with a bulk copy still writing into it.
  for (int q = 0; q < S; ++q) {
    if (((used_mask >> q) & 1u) && !mbar_wait_bounded(&full[q], (last_parity >> q) & 1u, a.timeout_ns)) {
      set_error(a.err, kDevTimeoutDrain, q, static_cast<int>((last_parity >> q) & 1u), static_cast<int>(round));
    }
  }
}

template <class Real, bool SPARSE = false>
__device__ __noinline__ void producer_entry(const ChrArgs& a, const Layout& L, unsigned char* smem, int chain_local,
                                            const SpArgs* sp = nullptr, const int* cs = nullptr, int eb = 0) {
  const int gchain = a.chain_base + chain_local;
  if (a.rng == 0) {
    PhiloxSource src;
    src.k0 = static_cast<uint32_t>(a.seed);
    src.k1 = static_cast<uint32_t>(a.seed >> 32);
    src.chain = static_cast<uint32_t>(gchain);
    run_producer<Real, PhiloxSource, SPARSE>(a, src, L, smem, sp, cs, eb);
  } else {
    MrgSource src;
    curandStateMRG32k3a* states = reinterpret_cast<curandStateMRG32k3a*>(a.rng_state);
    if (states) {
      src.st = states[chain_local];
    } else {
      curand_init(a.seed, static_cast<unsigned long long>(gchain), 0ull, &src.st);
    }
    run_producer<Real, MrgSource, SPARSE>(a, src, L, smem, sp, cs, eb);
    if (states) states[chain_local] = src.st;
  }
}

// V consecutive values through 16-byte (or narrower) vector accesses; the
// address is a multiple of V elements.
template <class Real, int V>
__device__ __forceinline__ void vload(const Real* p, Real (&o)[V]) {
  if constexpr (sizeof(Real) == 4 && V % 4 == 0) {
#pragma unroll
    for (int i = 0; i < V; i += 4) {
      const float4 q = *reinterpret_cast<const float4*>(p + i);
      o[i] = q.x;
      o[i + 1] = q.y;
      o[i + 2] = q.z;
      o[i + 3] = q.w;
    }
  } else if constexpr (sizeof(Real) == 4 && V == 2) {
    const float2 q = *reinterpret_cast<const float2*>(p);
    o[0] = q.x;
    o[1] = q.y;
  } else if constexpr (sizeof(Real) == 8 && V % 2 == 0) {
#pragma unroll
    for (int i = 0; i < V; i += 2) {
      const double2 q = *reinterpret_cast<const double2*>(p + i);
      o[i] = q.x;
      o[i + 1] = q.y;
    }
  } else {
#pragma unroll
    for (int i = 0; i < V; ++i) o[i] = p[i];
  }
}

template <class Real, int V>
__device__ __forceinline__ void vstore(Real* p, const Real (&v)[V]) {
  if constexpr (sizeof(Real) == 4 && V % 4 == 0) {
#pragma unroll
    for (int i = 0; i < V; i += 4) *reinterpret_cast<float4*>(p + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
  } else if constexpr (sizeof(Real) == 4 && V == 2) {
    *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
  } else if constexpr (sizeof(Real) == 8 && V % 2 == 0) {
#pragma unroll
    for (int i = 0; i < V; i += 2) *reinterpret_cast<double2*>(p + i) = make_double2(v[i], v[i + 1]);
  } else {
#pragma unroll
    for (int i = 0; i < V; ++i) p[i] = v[i];
  }
}

// Cross-CTA exchange of a chain split over a thread-block cluster: entry
// [buffer][rank] holds rank's (hi, lo, lo2, abort) of one step, written by
// the owner into every peer's copy; `bar[buffer]` completes when all CTAs
// of the cluster have written.  Buffers alternate between steps.
struct ClusterXEntry {
  unsigned long long hi, lo, lo2, abort;
};
struct ClusterCtx {
  ClusterXEntry* xbuf;  // [2][size]
  uint64_t* bar;        // [2], expected count = size
  int* flag;            // [2], outcome of the local wait
  uint32_t rank, size;
};

// Consumer side of one chain.
//
// Rows are handed out in chunks of C = 32 V rows: chunk c covers rows
// [c C, c C + C), lane l of the owning warp holds rows c C + l V + [0, V)
// and reads them with one vector access.  Warp w owns chunks w, w + NW, ...
// (at most R of them).  Every chunk test is uniform across the warp, so
// rows past m cost nothing; only the one partial chunk at the end of the
// rows tests each row.
//
// SS: slack in shared memory (row r of this chain at slack[r]) instead of
// the consumer threads' registers; used by the batched kernel so that several
// chains share an SM without register pressure.
// FUSED: the slack update of step t-1 runs inside the ratio pass of step t,
// with step t-1's column values kept in registers (R V per lane), so each
// step makes one pass over its rows and releases its column slot right
// after that pass.  The values are exactly those of the two-pass order.
// UNI: every warp runs exactly R chunks with no test on the chunk count, so
// a step's row pass is one straight-line block (its loads, divisions and
// extremes can overlap across all R V rows of a lane).  Chunk k of a lane
// covers rows min(base0 + k NW C, m - V) + v: past the last row the lanes
// repeat the last V rows (m % V == 0 keeps that group aligned and whole),
// whose ratios, slack and updates are bit for bit those of the rows they
// repeat, so the extremes are unchanged; only the owner of a row writes it.
// (Skipping a last chunk that would only repeat rows, by a warp-uniform
// test, was measured 1.4 % slower at the headline shape.)
template <class Real, int NT, int R, int V, bool SS = false, bool TIMING = true, bool MAYBE_DIRECT = true,
          bool CL = false, bool FUSED = false, bool UNI = false>
__device__ void run_consumers(const ChrArgs& a, const Layout& L, unsigned char* smem, int chain_local,
                              const ClusterCtx* cx = nullptr) {
  static_assert(!UNI || (!SS && !CL), "uniform chunks keep the slack in registers, one CTA per chain");
  using T = Tier<Real>;
  using Acc = typename T::Acc;
  using UT = typename T::UType;
  constexpr int NW = NT / 32;
  constexpr int C = 32 * V;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  double* xs = reinterpret_cast<double*>(smem + L.x_off);
  const StepMeta* meta = reinterpret_cast<const StepMeta*>(smem + L.meta_off);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.full_off);
  uint64_t* empty = reinterpret_cast<uint64_t*>(smem + L.empty_off);
  RedEntry* red = reinterpret_cast<RedEntry*>(smem + L.red_off);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + L.flag_off);
  const Real* A = T::A(a);
  const int m = a.m, d = a.d, lda = a.lda, S = L.slots;
  const int gchain = a.chain_base + chain_local;
  const bool direct = MAYBE_DIRECT && L.direct;
  // This warp's chunks: full ones at k < my_full, then (for one warp) the
  // partial chunk at k == my_full.
  const int n_full = m / C;
  const int my_full = n_full > warp ? (n_full - warp + NW - 1) / NW : 0;
  const bool my_tail = !UNI && (m % C) != 0 && (n_full % NW) == warp;
  const int base0 = warp * C + lane * V;

  for (int j = tid; j < d; j += NT) xs[j] = a.X0[static_cast<size_t>(chain_local) * a.ldx + j];
  named_bar_sync(1, NT);

  // Calls full(k, base) for each full chunk of this warp (k, the chunk's
  // index in the warp, is a constant once the loop is unrolled; base is the
  // lane's first row), then tail(base) for the partial chunk if this warp
  // owns it.
  const int tail_base = base0 + my_full * NW * C;
  auto for_chunks = [&](auto&& full_fn, auto&& tail_fn) {
    if constexpr (UNI) {
#pragma unroll
      for (int k = 0; k < R; ++k) full_fn(k, min(base0 + k * NW * C, m - V));
    } else {
#pragma unroll
      for (int k = 0; k < R; ++k) {
        if (k >= my_full) break;
        full_fn(k, base0 + k * NW * C);
      }
      if (my_tail) tail_fn(tail_base);
    }
  };

  Real sl_reg[SS ? 1 : R * V];
  Real* sl_sm = reinterpret_cast<Real*>(smem + L.slack_off);
  auto slack_get = [&](int k, int base, Real (&s)[V]) {
    if constexpr (SS) {
      vload<Real, V>(sl_sm + base, s);
    } else {
#pragma unroll
      for (int v = 0; v < V; ++v) s[v] = sl_reg[k * V + v];
    }
  };
  auto slack_put = [&](int k, int base, const Real (&s)[V]) {
    if constexpr (SS) {
      vstore<Real, V>(sl_sm + base, s);
    } else {
#pragma unroll
      for (int v = 0; v < V; ++v) sl_reg[k * V + v] = s[v];
    }
  };
  // Slack of row r of the partial chunk.
  Real* tail_sl = reinterpret_cast<Real*>(smem + L.tail_off) - n_full * C;
  auto slack_tail = [&](int r) -> Real& {
    if constexpr (SS) return sl_sm[r];
    else return tail_sl[r];
  };

  auto recompute = [&]() {
    for_chunks(
        [&](int k, int base) {
          double acc[V];
#pragma unroll
          for (int v = 0; v < V; ++v) acc[v] = 0.0;
          const double* Ar = a.A64 + base;
          // Unrolled so that the loads of several columns are in flight
          // ahead of the (sequential, order-preserving) fma chain.
#pragma unroll 4
          for (int j = 0; j < d; ++j) {
            const double xj = xs[j];
            const double* Aj = Ar + static_cast<size_t>(j) * lda;
#pragma unroll
            for (int v = 0; v < V; ++v) acc[v] = __fma_rn(Aj[v], xj, acc[v]);
          }
          Real s[V];
#pragma unroll
          for (int v = 0; v < V; ++v) s[v] = T::from64(__dsub_rn(a.b[base + v], acc[v]));
          slack_put(k, base, s);
        },
        [&](int base) {
#pragma unroll
          for (int v = 0; v < V; ++v) {
            const int r = base + v;
            if (r < m) {
              double acc = 0.0;
              const double* Ar = a.A64 + r;
              for (int j = 0; j < d; ++j) acc = __fma_rn(Ar[static_cast<size_t>(j) * lda], xs[j], acc);
              slack_tail(r) = T::from64(__dsub_rn(a.b[r], acc));
            }
          }
        });
  };
  if (a.slack_in) {
    // the slack at step t_first, computed outside the kernel
    const Real* si = static_cast<const Real*>(a.slack_in) + static_cast<size_t>(chain_local) * m;
    for_chunks(
        [&](int k, int base) {
          Real sv[V];
#pragma unroll
          for (int v = 0; v < V; ++v) sv[v] = si[base + v];
          slack_put(k, base, sv);
        },
        [&](int base) {
#pragma unroll
          for (int v = 0; v < V; ++v)
            if (base + v < m) slack_tail(base + v) = si[base + v];
        });
  } else {
    recompute();
  }

  const long long total = launch_steps(a);
  // Ring position (mirrors the producer), phase parity of the slot's fill,
  // and step counters that replace the global step's remainders modulo
  // thinning and resync; out_row is the next saved sample's row.
  int slot = 0;
  uint32_t parity = 0;
  int thin_ctr = static_cast<int>(a.t_first % a.thinning);
  int resync_ctr = a.resync > 0 ? static_cast<int>(a.t_first % a.resync) : 0;
  int rbuf = 0;
  size_t out_row = static_cast<size_t>(gchain) +
                   static_cast<size_t>((a.t_first + a.thinning - 1) / a.thinning) * a.out_nchains;
  unsigned long long w_full = 0;
  const unsigned long long c_start = TIMING ? clock64() : 0ull;
  Real ae_prev[FUSED ? R * V : 1];   // step t-1's column values of this lane's rows
  Real ae_prev_tail[FUSED ? V : 1];  // ... of its rows in the partial chunk
  bool pending = false;              // step t-1's slack update not applied yet
  Real alpha_prev = Real(0);
  for (long long t = 0; t < total; ++t) {
    const int sa = slot;
    const unsigned long long w0 = (TIMING && a.wait_cycles) ? clock64() : 0ull;
    bool ok = mbar_wait_bounded(&full[sa], parity, a.timeout_ns);
    if (TIMING && a.wait_cycles) w_full += clock64() - w0;
    int kind = kCoord, ei = 0, ej = 0, sb = -1, kq = 0;
    Real cir = Real(1), cjr = Real(0);
    UT uu = UT(0.5);
    double cix = 1.0, cjx = 0.0;  // the coefficients as the x update uses them
    if (ok) {
      const StepMeta& M = meta[sa];
      const int4 h0 = *reinterpret_cast<const int4*>(&M.kind);
      const int4 h1 = *reinterpret_cast<const int4*>(&M.k);
      kind = h0.x;
      ei = h0.y;
      ej = h0.z;
      sb = h0.w;
      kq = h1.x;
      if constexpr (sizeof(Real) == 4) {
        cir = __int_as_float(h1.y);
        cjr = __int_as_float(h1.z);
        uu = __int_as_float(h1.w);
        cix = static_cast<double>(cir);
        cjx = static_cast<double>(cjr);
      } else {
        cir = M.ci;
        cjr = M.cj;
        uu = M.u;
        cix = cir;
        cjx = cjr;
      }
      if (++slot == S) {
        slot = 0;
        parity ^= 1u;
      }
      if (kind == kPair) {
        ok = mbar_wait_bounded(&full[sb], parity, a.timeout_ns);
        if (++slot == S) {
          slot = 0;
          parity ^= 1u;
        }
      }
    }
    // Uniform across every consumer warp (a named barrier follows), whatever `ok` is.
    if (a.resync > 0) {
      // (the launch's first step starts from the slack computed before the loop)
      if (resync_ctr == 0 && t != 0) {
        named_bar_sync(2, NT);  // every owner's x update of the previous step is visible
        recompute();
        pending = false;        // the recompute already holds step t-1's move
      }
      if (++resync_ctr == a.resync) resync_ctr = 0;
    }
    // Row passes, specialised once per step on the (warp-uniform) kind and
    // on where the column lives, so the per-row code is straight-line.
    // ae = A u for row r is evaluated identically in the ratio pass and the
    // slack update (the slot stays resident until the step releases it).
    const Real* sca = reinterpret_cast<const Real*>(smem + L.slot_off + static_cast<size_t>(sa) * L.slot_bytes);
    const Real* scb = reinterpret_cast<const Real*>(smem + L.slot_off +
                                                    static_cast<size_t>(sb < 0 ? 0 : sb) * L.slot_bytes);
    auto ks_at = [&](int r) -> Real {
      const StepMeta& M = meta[sa];
      Real acc = Real(0);
      for (int q = 0; q < kq; ++q) acc = T::ks_acc(acc, A[r + static_cast<size_t>(M.ks_idx[q]) * lda], M.ks_coef[q]);
      return acc;
    };
    // pass(vec, one): vec(base, ae[V]) fills a full chunk's V values, one(r)
    // returns row r's value.
    auto for_kind = [&](auto&& pass) {
      if (kind == kCoord) {
        const Real* col = direct ? A + static_cast<size_t>(ei) * lda : sca;
        pass([&](int base, Real(&o)[V]) { vload<Real, V>(col + base, o); }, [&](int r) -> Real { return col[r]; });
      } else if (kind == kPair) {
        const Real* ca = direct ? A + static_cast<size_t>(ei) * lda : sca;
        const Real* cb = direct ? A + static_cast<size_t>(ej) * lda : scb;
        pass(
            [&](int base, Real(&o)[V]) {
              Real x1[V], x2[V];
              vload<Real, V>(ca + base, x1);
              vload<Real, V>(cb + base, x2);
#pragma unroll
              for (int v = 0; v < V; ++v) o[v] = T::pair_ae_r(x1[v], x2[v], cir, cjr);
            },
            [&](int r) -> Real { return T::pair_ae_r(ca[r], cb[r], cir, cjr); });
      } else {
        pass(
            [&](int base, Real(&o)[V]) {
#pragma unroll
              for (int v = 0; v < V; ++v) o[v] = ks_at(base + v);
            },
            ks_at);
      }
    };
    // Cross-warp combination of (hi, lo, lo2): lane 0 of each warp posts its
    // warp's values; after one barrier lane l of every warp picks up warp l's
    // entry and a second warp reduction yields the chain's.  The two halves
    // of `red` alternate between consecutive steps.
    Acc hi = T::acc_hi0(), lo = T::acc_lo0(), lo2 = T::acc_lo20();
    if (ok) {
      for_kind([&](auto&& vec, auto&& one) {
        for_chunks(
            [&](int k, int base) {
              Real ae[V], s[V];
              vec(base, ae);
              slack_get(k, base, s);
              if constexpr (FUSED) {
                if (pending) {
#pragma unroll
                  for (int v = 0; v < V; ++v) s[v] = T::slack_update(s[v], alpha_prev, ae_prev[k * V + v]);
                  slack_put(k, base, s);
                }
#pragma unroll
                for (int v = 0; v < V; ++v) ae_prev[k * V + v] = ae[v];
              }
#pragma unroll
              for (int v = 0; v < V; ++v) T::acc(hi, lo, lo2, T::ratio(ae[v], s[v]));
            },
            [&](int base) {
#pragma unroll
              for (int v = 0; v < V; ++v) {
                const int r = base + v;
                if (r < m) {
                  const Real ae = one(r);
                  if constexpr (FUSED) {
                    if (pending) slack_tail(r) = T::slack_update(slack_tail(r), alpha_prev, ae_prev_tail[v]);
                    ae_prev_tail[v] = ae;
                  }
                  T::acc(hi, lo, lo2, T::ratio(ae, slack_tail(r)));
                }
              }
            });
      });
    }
    if constexpr (FUSED) {
      // The column is in registers now; a k-sparse step's record is still
      // read by its x update, so that slot is released at the end.
      if (ok && kind != kKSparse) {
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&empty[sa]);
          if (kind == kPair) mbar_arrive(&empty[sb]);
        }
      }
    }
    hi = T::red_hi(hi);
    lo = T::red_lo(lo);
    lo2 = T::red_lo2(lo2);
    if (NW > 1) {
      RedEntry* slotr = red + rbuf * NW;
      rbuf ^= 1;
      const int bad = __any_sync(0xffffffffu, !ok) ? 1 : 0;
      if (lane == 0) {
        slotr[warp].kmax = hi;
        slotr[warp].kmin = lo;
        slotr[warp].kmin2 = lo2;
        slotr[warp].abort = bad;
      }
      named_bar_sync(1, NT);
      Acc h = T::acc_hi0(), l = T::acc_lo0(), l2 = T::acc_lo20();
      int bflag = 0;
      if (lane < NW) {
        h = static_cast<Acc>(slotr[lane].kmax);
        l = static_cast<Acc>(slotr[lane].kmin);
        l2 = static_cast<Acc>(slotr[lane].kmin2);
        bflag = slotr[lane].abort;
      }
      hi = T::red_hi(h);
      lo = T::red_lo(l);
      lo2 = T::red_lo2(l2);
      ok = !__any_sync(0xffffffffu, bflag);
    } else {
      ok = !__any_sync(0xffffffffu, !ok);
    }
    if constexpr (CL) {
      // The CTA's values are uniform here.  Thread 0 writes them into every
      // CTA of the cluster, arrives on their barriers (releasing the writes)
      // and waits, bounded, for all entries of this step; one named barrier
      // hands the outcome to the other threads, so every warp takes the same
      // decision.  The abort flag travels with the values: all CTAs of the
      // chain leave at the same step.
      const int xb = static_cast<int>(t & 1);
      if (tid == 0) {
        ClusterXEntry* mine = cx->xbuf + xb * cx->size + cx->rank;
        for (uint32_t q = 0; q < cx->size; ++q) {
          const uint32_t ra = cluster_map(mine, q);
          cluster_st_v2(ra, static_cast<unsigned long long>(hi), static_cast<unsigned long long>(lo));
          cluster_st_v2(ra + 16, static_cast<unsigned long long>(lo2), ok ? 0ull : 1ull);
        }
        for (uint32_t q = 0; q < cx->size; ++q) mbar_arrive_remote(cluster_map(&cx->bar[xb], q));
        const bool w = mbar_wait_cluster_bounded(&cx->bar[xb], static_cast<uint32_t>((t >> 1) & 1), a.timeout_ns);
        cx->flag[xb] = w ? 1 : 0;
        if (!w) set_error(a.err, kDevTimeoutCluster, static_cast<int>(cx->rank), static_cast<int>(t), 0);
      }
      named_bar_sync(1, NT);
      const bool arrived = cx->flag[xb] != 0;
      Acc h = T::acc_hi0(), l = T::acc_lo0(), l2 = T::acc_lo20();
      int bflag = arrived ? 0 : 1;
      if (arrived && lane < static_cast<int>(cx->size)) {
        const ClusterXEntry& e = cx->xbuf[xb * cx->size + lane];
        h = static_cast<Acc>(e.hi);
        l = static_cast<Acc>(e.lo);
        l2 = static_cast<Acc>(e.lo2);
        bflag = e.abort != 0ull;
      }
      hi = T::red_hi(h);
      lo = T::red_lo(l);
      lo2 = T::red_lo2(l2);
      ok = !__any_sync(0xffffffffu, bflag);
    }
    if (!ok) {
      if (tid == 0) {
        set_error(a.err, kDevTimeoutFull, sa, static_cast<int>(parity), static_cast<int>(t));
        *abort_flag = 1;
      }
      return;
    }
    Real mx, mn;
    T::decode(hi, lo, lo2, mx, mn);
    const Real alpha = T::alpha(mx, mn, uu);
    const double a64 = static_cast<double>(alpha);
    // x update: entry j belongs to consumer thread j % NT.
    if (kind == kCoord) {
      if (ei % NT == tid) xs[ei] = __dadd_rn(xs[ei], a64);
    } else if (kind == kPair) {
      if (ei % NT == tid) xs[ei] = __fma_rn(a64, cix, xs[ei]);
      if (ej % NT == tid) xs[ej] = __fma_rn(a64, cjx, xs[ej]);
    } else {
      const StepMeta& M = meta[sa];
      for (int q = 0; q < kq; ++q) {
        const int idx = M.ks_idx[q];
        if (idx % NT == tid) xs[idx] = __fma_rn(a64, T::coef(M.ks_coef[q]), xs[idx]);
      }
    }
    if (thin_ctr == 0 && a.samples) {
      if (a.out_f64) {
        double* out = reinterpret_cast<double*>(a.samples) + out_row * d;
        for (int j = tid; j < d; j += NT) out[j] = xs[j];
      } else {
        float* out = reinterpret_cast<float*>(a.samples) + out_row * d;
        for (int j = tid; j < d; j += NT) out[j] = __double2float_rn(xs[j]);
      }
      out_row += static_cast<size_t>(a.out_nchains);
    }
    if (++thin_ctr == a.thinning) thin_ctr = 0;
    if constexpr (FUSED) {
      alpha_prev = alpha;
      pending = true;
      if (kind == kKSparse) {
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[sa]);
      }
      continue;
    }
    for_kind([&](auto&& vec, auto&& one) {
      for_chunks(
          [&](int k, int base) {
            Real ae[V], s[V];
            vec(base, ae);
            slack_get(k, base, s);
#pragma unroll
            for (int v = 0; v < V; ++v) s[v] = T::slack_update(s[v], alpha, ae[v]);
            slack_put(k, base, s);
          },
          [&](int base) {
#pragma unroll
            for (int v = 0; v < V; ++v) {
              const int r = base + v;
              if (r < m) slack_tail(r) = T::slack_update(slack_tail(r), alpha, one(r));
            }
          });
    });
    __syncwarp();
    if (lane == 0) {
      mbar_arrive(&empty[sa]);
      if (kind == kPair) mbar_arrive(&empty[sb]);
    }
  }
  if (a.X_final) {
    for (int j = tid; j < d; j += NT) a.X_final[static_cast<size_t>(chain_local) * a.ldx + j] = xs[j];
  }
  if (a.slack_final) {
    // the last step's pending update first (the fused order defers it)
    Real* so = static_cast<Real*>(a.slack_final) + static_cast<size_t>(chain_local) * m;
    for_chunks(
        [&](int k, int base) {
          if (UNI && base0 + k * NW * C >= m) return;  // a repeat of rows another lane owns
          Real s[V];
          slack_get(k, base, s);
          if constexpr (FUSED) {
            if (pending) {
#pragma unroll
              for (int v = 0; v < V; ++v) s[v] = T::slack_update(s[v], alpha_prev, ae_prev[k * V + v]);
            }
          }
#pragma unroll
          for (int v = 0; v < V; ++v) so[base + v] = s[v];
        },
        [&](int base) {
#pragma unroll
          for (int v = 0; v < V; ++v) {
            const int r = base + v;
            if (r < m) {
              Real sv = slack_tail(r);
              if constexpr (FUSED) {
                if (pending) sv = T::slack_update(sv, alpha_prev, ae_prev_tail[v]);
              }
              so[r] = sv;
            }
          }
        });
  }
  if (TIMING && a.wait_cycles && tid == 0) {
    a.wait_cycles[4 * chain_local + 0] = w_full;
    a.wait_cycles[4 * chain_local + 2] = clock64() - c_start;
  }
}

// Rows per lane per chunk of the single-model kernel: 16-byte vector
// accesses (FP32: 128-row chunks, four independent rows per lane between a
// column load and the extremes; FP64: 64-row chunks, whose slack fits the
// registers without spilling).
template <class Real>
constexpr int kStandaloneV = sizeof(Real) == 4 ? 4 : 2;
inline int standalone_v(int precision) { return precision == NAJA_PREC_FP64 ? 2 : 4; }
// A chain split over a cluster keeps 64-row chunks, so that small models
// still give every CTA of the cluster rows.
constexpr int kClusterV = 2;
// The batched kernel (FP32 only) runs several chains per SM and is bound by
// instruction issue, so it takes 16-byte accesses: 128-row chunks.
constexpr int kBatchV = 4;

template <class Real, int NT, int R, bool UNI = false>
__global__ void __launch_bounds__(NT + 32, 1)
    chr_kernel(const __grid_constant__ ChrArgs a, const __grid_constant__ Layout L) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int chain_local = blockIdx.x;
  if (threadIdx.x == 0) {
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.full_off);
    uint64_t* empty = reinterpret_cast<uint64_t*>(smem + L.empty_off);
    for (int s = 0; s < L.slots; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NT / 32);
    }
    *reinterpret_cast<volatile int*>(smem + L.flag_off) = 0;
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x >= NT) {
    if (threadIdx.x == NT) producer_entry<Real>(a, L, smem, chain_local);
    return;
  }
  // fused update where step t-1's column values (R V per lane) fit in 64
  // bytes of registers; larger capacities keep the two-pass order
  constexpr bool kFuse = R * kStandaloneV<Real> * sizeof(Real) <= 64;
  run_consumers<Real, NT, R, kStandaloneV<Real>, false, true, true, false, kFuse, UNI>(a, L, smem, chain_local);
}

// One chain split over a thread-block cluster of `size` CTAs: CTA `rank`
// owns the row chunks [nc rank / size, nc (rank + 1) / size) of the 32 V-row
// chunks, with its own column staging (producer), slack and FP64 recompute
// of those rows, a full copy of x and the same direction stream, so every
// CTA computes the same alpha from the cluster-wide extremes.  Only rank 0
// writes samples and final positions.  The kernel begins and ends with a
// barrier over the whole cluster: no CTA starts sending before every peer
// has initialised its barriers, and none leaves while a peer may still write
// into its shared memory.
template <class Real, int NT, int R>
__global__ void __launch_bounds__(NT + 32, 1)
    chr_cluster_kernel(const __grid_constant__ ChrArgs base, const __grid_constant__ Layout L) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ ChrArgs slice;
  __shared__ __align__(16) ClusterXEntry xbuf[2 * 8];
  __shared__ __align__(8) uint64_t xbar[2];
  __shared__ int xflag[2];
  const uint32_t rank = cluster_rank(), size = cluster_size();
  const int chain_local = static_cast<int>(blockIdx.x / size);
  constexpr int C = 32 * kClusterV;
  const int nc = (base.m + C - 1) / C;
  const int c0 = static_cast<int>(static_cast<long long>(nc) * rank / size);
  const int c1 = static_cast<int>(static_cast<long long>(nc) * (rank + 1) / size);
  const int row0 = c0 * C;
  if (threadIdx.x == 0) {
    ChrArgs a = base;
    a.A32 = base.A32 ? base.A32 + row0 : nullptr;
    a.A64 = base.A64 + row0;
    a.b = base.b + row0;
    a.m = min(c1 * C, base.m) - row0;
    if (rank != 0) {
      a.samples = nullptr;
      a.X_final = nullptr;
      a.wait_cycles = nullptr;
      a.slack_final = nullptr;
    }
    slice = a;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.full_off);
    uint64_t* empty = reinterpret_cast<uint64_t*>(smem + L.empty_off);
    for (int s = 0; s < L.slots; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NT / 32);
    }
    mbar_init(&xbar[0], size);
    mbar_init(&xbar[1], size);
    xflag[0] = xflag[1] = 0;
    *reinterpret_cast<volatile int*>(smem + L.flag_off) = 0;
    fence_mbar_init();
  }
  cluster_sync_all();
  const ClusterCtx cx{xbuf, xbar, xflag, rank, size};
  if (threadIdx.x >= NT) {
    if (threadIdx.x == NT) producer_entry<Real>(slice, L, smem, chain_local);
  } else {
    run_consumers<Real, NT, R, kClusterV, false, true, true, true>(slice, L, smem, chain_local, &cx);
  }
  cluster_sync_all();
}

// ------------------------------------------------------------- dispatch
template <class Real, int NT, int R>
int launch_one_cluster(const ChrArgs& a, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream) {
  auto kern = chr_cluster_kernel<Real, NT, R>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(cfg.smem));
  if (e != cudaSuccess) return NAJA_ERR_CUDA;
  const Layout L = make_layout(a.d, cfg.slice_lda, sizeof(Real), NT, cfg.slots);
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3(static_cast<unsigned>(nchains * cfg.cluster));
  lc.blockDim = dim3(NT + 32);
  lc.dynamicSmemBytes = cfg.smem;
  lc.stream = stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = static_cast<unsigned>(cfg.cluster);
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  e = cudaLaunchKernelEx(&lc, kern, a, L);
  return e == cudaSuccess ? NAJA_OK : NAJA_ERR_CUDA;
}

template <class Real, int NT, int R, bool UNI = false>
int launch_one(const ChrArgs& a, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream) {
  if constexpr (NT == 128 || NT == 256) {
    if (!UNI && cfg.cluster > 1) return launch_one_cluster<Real, NT, R>(a, nchains, cfg, stream);
  }
  if (cfg.cluster > 1) return NAJA_ERR_UNSUPPORTED;
  if (UNI && a.m % kStandaloneV<Real> != 0) return NAJA_ERR_UNSUPPORTED;
  auto kern = chr_kernel<Real, NT, R, UNI>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(cfg.smem));
  if (e != cudaSuccess) return NAJA_ERR_CUDA;
  const Layout L = make_layout(a.d, a.lda, sizeof(Real), NT, cfg.slots);
  kern<<<nchains, NT + 32, cfg.smem, stream>>>(a, L);
  return cudaGetLastError() == cudaSuccess ? NAJA_OK : NAJA_ERR_CUDA;
}

// cfg.rows = chunks per warp (template capacity).
template <class Real, int NT>
int launch_rows(const ChrArgs& a, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream) {
  if (cfg.uniform) {
    // cfg.rows = chunks of every warp (exact)
    switch (cfg.rows) {
      case 1: return launch_one<Real, NT, 1, true>(a, nchains, cfg, stream);
      case 2: return launch_one<Real, NT, 2, true>(a, nchains, cfg, stream);
      case 3: return launch_one<Real, NT, 3, true>(a, nchains, cfg, stream);
      case 4: return launch_one<Real, NT, 4, true>(a, nchains, cfg, stream);
      case 5: return launch_one<Real, NT, 5, true>(a, nchains, cfg, stream);
      case 6: return launch_one<Real, NT, 6, true>(a, nchains, cfg, stream);
      case 7: return launch_one<Real, NT, 7, true>(a, nchains, cfg, stream);
      case 8: return launch_one<Real, NT, 8, true>(a, nchains, cfg, stream);
      default: return NAJA_ERR_UNSUPPORTED;
    }
  }
  // cfg.rows = chunks per warp (template capacity)
  switch (cfg.rows) {
    case 1: return launch_one<Real, NT, 1>(a, nchains, cfg, stream);
    case 2: return launch_one<Real, NT, 2>(a, nchains, cfg, stream);
    case 4: return launch_one<Real, NT, 4>(a, nchains, cfg, stream);
    case 8: return launch_one<Real, NT, 8>(a, nchains, cfg, stream);
    case 16:
      if constexpr (NT <= 512) return launch_one<Real, NT, 16>(a, nchains, cfg, stream);
      break;
    default: break;
  }
  return NAJA_ERR_UNSUPPORTED;
}

}  // namespace
}  // namespace chr_detail
}  // namespace naja
