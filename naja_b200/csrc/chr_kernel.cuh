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
//   * The slack vector lives in the consumers' registers (thread t owns rows
//     t, t+NT, ...), so the only memory traffic per step is one column of A
//     (two for a pair step) plus the amortised sample write.
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

struct __align__(16) StepMeta {
  int kind;
  int ei;
  int ej;
  int slot_b;
  double ci;
  double cj;
  double u;
  int k;
  int pad;
  int ks_idx[32];
  double ks_coef[32];
};

struct RedEntry {
  unsigned long long kmax;
  unsigned long long kmin;
  int abort;
  int pad;
};

constexpr size_t kSmemBudget = 227 * 1024;
constexpr int kMaxSlots = 8;

__host__ __device__ inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

struct Layout {
  size_t x_off, slot_off, slot_bytes, meta_off, full_off, empty_off, red_off, flag_off, total;
  int slots;
  bool direct;
};

__host__ __device__ inline Layout make_layout(int d, int lda, int elt, int nthreads, int slots_req) {
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
  L.total = align_up(off, 128);
  L.slots = S;
  L.direct = direct;
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
__device__ bool draw_direction(Src& src, const ChrArgs& a, StepMeta& o) {
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
      o.ks_idx[t] = idx;
      o.ks_coef[t] = __dmul_rn(sign, inv_sqrt_k);
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
  __device__ static float pair_ae(float ai, float aj, double ci, double cj) {
    return __fmaf_rn(ai, static_cast<float>(ci), __fmul_rn(aj, static_cast<float>(cj)));
  }
  __device__ static float ks_acc(float acc, float av, double coef) {
    return __fmaf_rn(av, static_cast<float>(coef), acc);
  }
  // Ratio ae/s with the reference's special cases; a negative FP32 slack
  // counts as 0 (it can only come from FP32 rounding).
  __device__ static float ratio(float ae, float s) {
    if (s < 0.0f) s = 0.0f;
    if (s == 0.0f) return ae > 0.0f ? __int_as_float(0x7f800000) : (ae < 0.0f ? __int_as_float(0xff800000) : 0.0f);
    const float r = __fdiv_rn(ae, s);
    return isnan(r) ? 0.0f : r;
  }
  __device__ static float alpha(float mx, float mn, double u) {
    const float lo = __fdiv_rn(1.0f, mn), hi = __fdiv_rn(1.0f, mx);
    return __fmaf_rn(static_cast<float>(u), __fsub_rn(hi, lo), lo);
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
  __device__ static double pair_ae(double ai, double aj, double ci, double cj) {
    return __fma_rn(ai, ci, __dmul_rn(aj, cj));
  }
  __device__ static double ks_acc(double acc, double av, double coef) { return __fma_rn(av, coef, acc); }
  __device__ static double ratio(double ae, double s) {
    if (s == 0.0)
      return ae > 0.0 ? __longlong_as_double(0x7ff0000000000000ll)
                      : (ae < 0.0 ? __longlong_as_double(static_cast<long long>(0xfff0000000000000ull)) : 0.0);
    const double r = __ddiv_rn(ae, s);
    return isnan(r) ? 0.0 : r;
  }
  __device__ static double alpha(double mx, double mn, double u) {
    const double lo = __ddiv_rn(1.0, mn), hi = __ddiv_rn(1.0, mx);
    return __fma_rn(u, __dsub_rn(hi, lo), lo);
  }
  __device__ static double coef(double c) { return c; }
  __device__ static double slack_update(double s, double alpha, double ae) { return __fma_rn(-alpha, ae, s); }
  __device__ static double from64(double v) { return v; }
};


// ------------------------------------------------------------------ producer
// One thread: draws each step's direction ahead of the consumers, claims one
// ring slot per staged column (two for a pair step, one metadata-only slot
// for a k-sparse step), writes the step record and starts the bulk copy.
template <class Real, class Src>
__device__ __noinline__ void run_producer(const ChrArgs& a, Src& src, const Layout& L, unsigned char* smem) {
  StepMeta* meta = reinterpret_cast<StepMeta*>(smem + L.meta_off);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.full_off);
  uint64_t* empty = reinterpret_cast<uint64_t*>(smem + L.empty_off);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + L.flag_off);
  const Real* A = Tier<Real>::A(a);
  const uint32_t col_bytes = static_cast<uint32_t>(align_up(static_cast<size_t>(a.m) * sizeof(Real), 16));
  const int S = L.slots;
  const long long total = static_cast<long long>(a.nspc) * a.thinning;
  uint64_t g = 0;
  uint64_t last_use[kMaxSlots];
  bool used[kMaxSlots];
  for (int s = 0; s < kMaxSlots; ++s) used[s] = false;
  StepMeta dir;
  for (long long t = 0; t < total; ++t) {
    if (*abort_flag) break;
    src.begin_step(static_cast<uint64_t>(a.step_offset + t));
    if (!draw_direction(src, a, dir)) {
      set_error(a.err, kDevBadPair);
      *abort_flag = 1;
      break;
    }
    const int sa = static_cast<int>(g % S);
    const uint64_t ua = g / S;
    if (ua >= 1 && !mbar_wait_bounded(&empty[sa], static_cast<uint32_t>((ua - 1) & 1), a.timeout_ns)) {
      set_error(a.err, kDevTimeoutEmpty);
      *abort_flag = 1;
      break;
    }
    int sb = -1;
    uint64_t ub = 0;
    if (dir.kind == kPair) {
      sb = static_cast<int>((g + 1) % S);
      ub = (g + 1) / S;
      if (ub >= 1 && !mbar_wait_bounded(&empty[sb], static_cast<uint32_t>((ub - 1) & 1), a.timeout_ns)) {
        set_error(a.err, kDevTimeoutEmpty);
        *abort_flag = 1;
        break;
      }
    }
    g += (sb >= 0) ? 2 : 1;
    StepMeta& M = meta[sa];
    M.kind = dir.kind;
    M.ei = dir.ei;
    M.ej = dir.ej;
    M.slot_b = sb;
    M.ci = dir.ci;
    M.cj = dir.cj;
    M.u = dir.u;
    M.k = dir.k;
    if (dir.kind == kKSparse) {
      for (int q = 0; q < dir.k; ++q) {
        M.ks_idx[q] = dir.ks_idx[q];
        M.ks_coef[q] = dir.ks_coef[q];
      }
    }
    if (!L.direct && dir.kind != kKSparse) {
      used[sa] = true;
      last_use[sa] = ua;
      mbar_arrive_expect_tx(&full[sa], col_bytes);
      bulk_g2s(smem + L.slot_off + static_cast<size_t>(sa) * L.slot_bytes, A + static_cast<size_t>(dir.ei) * a.lda,
               col_bytes, &full[sa]);
      if (sb >= 0) {
        used[sb] = true;
        last_use[sb] = ub;
        mbar_arrive_expect_tx(&full[sb], col_bytes);
        bulk_g2s(smem + L.slot_off + static_cast<size_t>(sb) * L.slot_bytes,
                 A + static_cast<size_t>(dir.ej) * a.lda, col_bytes, &full[sb]);
      }
    } else {
      mbar_arrive(&full[sa]);
      if (sb >= 0) mbar_arrive(&full[sb]);
    }
  }
  // Drain: never leave the CTA with a bulk copy still writing into it.
  for (int s = 0; s < S; ++s) {
    if (used[s] && !mbar_wait_bounded(&full[s], static_cast<uint32_t>(last_use[s] & 1), a.timeout_ns)) {
      set_error(a.err, kDevTimeoutDrain);
    }
  }
}

template <class Real>
__device__ __noinline__ void producer_entry(const ChrArgs& a, const Layout& L, unsigned char* smem, int chain_local) {
  const int gchain = a.chain_base + chain_local;
  if (a.rng == 0) {
    PhiloxSource src;
    src.k0 = static_cast<uint32_t>(a.seed);
    src.k1 = static_cast<uint32_t>(a.seed >> 32);
    src.chain = static_cast<uint32_t>(gchain);
    run_producer<Real>(a, src, L, smem);
  } else {
    MrgSource src;
    curandStateMRG32k3a* states = reinterpret_cast<curandStateMRG32k3a*>(a.rng_state);
    if (states) {
      src.st = states[chain_local];
    } else {
      curand_init(a.seed, static_cast<unsigned long long>(gchain), 0ull, &src.st);
    }
    run_producer<Real>(a, src, L, smem);
    if (states) states[chain_local] = src.st;
  }
}

template <class Real, int NT, int R>
__device__ void run_consumers(const ChrArgs& a, const Layout& L, unsigned char* smem, int chain_local) {
  using T = Tier<Real>;
  using Key = typename T::Key;
  constexpr int NW = NT / 32;
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

  for (int j = tid; j < d; j += NT) xs[j] = a.X0[static_cast<size_t>(chain_local) * a.ldx + j];
  named_bar_sync(1, NT);

  Real sl[R];
  auto recompute = [&]() {
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int r = tid + k * NT;
      if (r < m) {
        double acc = 0.0;
        const double* Ar = a.A64 + r;
        for (int j = 0; j < d; ++j) acc = __fma_rn(Ar[static_cast<size_t>(j) * lda], xs[j], acc);
        sl[k] = T::from64(__dsub_rn(a.b[r], acc));
      } else {
        sl[k] = Real(0);
      }
    }
  };
  recompute();

  const long long total = static_cast<long long>(a.nspc) * a.thinning;
  uint64_t g = 0;
  for (long long t = 0; t < total; ++t) {
    const int sa = static_cast<int>(g % S);
    bool ok = mbar_wait_bounded(&full[sa], static_cast<uint32_t>((g / S) & 1), a.timeout_ns);
    int kind = kCoord, ei = 0, ej = 0, sb = -1, kq = 0;
    double ci = 1.0, cj = 0.0, u = 0.5;
    if (ok) {
      const StepMeta& M = meta[sa];
      kind = M.kind;
      ei = M.ei;
      ej = M.ej;
      sb = M.slot_b;
      ci = M.ci;
      cj = M.cj;
      u = M.u;
      kq = M.k;
      ++g;
      if (kind == kPair) {
        ok = mbar_wait_bounded(&full[sb], static_cast<uint32_t>((g / S) & 1), a.timeout_ns);
        ++g;
      }
    }
    // Uniform across every consumer warp (a named barrier follows), whatever `ok` is.
    if (a.resync > 0 && (t % a.resync) == 0) {
      named_bar_sync(2, NT);  // every owner's x update of step t-1 is visible
      recompute();
    }
    Key kmax = T::key(T::lowest()), kmin = T::key(T::highest());
    // Column(s) of this step: staged in the ring, or straight from L2/HBM.
    const Real* ca = L.direct ? A + static_cast<size_t>(ei) * lda
                              : reinterpret_cast<const Real*>(smem + L.slot_off + static_cast<size_t>(sa) * L.slot_bytes);
    const Real* cb = (kind == kPair)
                         ? (L.direct ? A + static_cast<size_t>(ej) * lda
                                     : reinterpret_cast<const Real*>(smem + L.slot_off +
                                                                     static_cast<size_t>(sb) * L.slot_bytes))
                         : ca;
    // ae = A u for row r; evaluated identically in the ratio pass and the
    // slack update (the slot stays resident until the step releases it).
    auto ae_of = [&](int r) -> Real {
      if (kind == kCoord) return ca[r];
      if (kind == kPair) return T::pair_ae(ca[r], cb[r], ci, cj);
      const StepMeta& M = meta[sa];
      Real acc = Real(0);
      for (int q = 0; q < kq; ++q) acc = T::ks_acc(acc, A[r + static_cast<size_t>(M.ks_idx[q]) * lda], M.ks_coef[q]);
      return acc;
    };
    if (ok) {
#pragma unroll
      for (int k = 0; k < R; ++k) {
        const int r = tid + k * NT;
        if (r < m) {
          const Real v = ae_of(r);
          const Key kv = T::key(T::ratio(v, sl[k]));
          kmax = kv > kmax ? kv : kmax;
          kmin = kv < kmin ? kv : kmin;
        }
      }
    }
    kmax = T::wmax(kmax);
    kmin = T::wmin(kmin);
    Real mx = T::unkey(kmax), mn = T::unkey(kmin);
    if (NW > 1) {
      RedEntry* slotr = red + (t & 1) * NW;
      const int bad = __any_sync(0xffffffffu, !ok) ? 1 : 0;
      if (lane == 0) {
        slotr[warp].kmax = kmax;
        slotr[warp].kmin = kmin;
        slotr[warp].abort = bad;
      }
      named_bar_sync(1, NT);
      int any_bad = 0;
#pragma unroll 4
      for (int w = 0; w < NW; ++w) {
        const Key a1 = static_cast<Key>(slotr[w].kmax), a2 = static_cast<Key>(slotr[w].kmin);
        kmax = a1 > kmax ? a1 : kmax;
        kmin = a2 < kmin ? a2 : kmin;
        any_bad |= slotr[w].abort;
      }
      if (any_bad) {
        if (tid == 0) {
          set_error(a.err, kDevTimeoutFull);
          *abort_flag = 1;
        }
        return;
      }
      mx = T::unkey(kmax);
      mn = T::unkey(kmin);
    } else if (__any_sync(0xffffffffu, !ok)) {
      if (lane == 0) {
        set_error(a.err, kDevTimeoutFull);
        *abort_flag = 1;
      }
      return;
    }
    const Real alpha = T::alpha(mx, mn, u);
    const double a64 = static_cast<double>(alpha);
    // x update: entry j belongs to consumer thread j % NT.
    if (kind == kCoord) {
      if (ei % NT == tid) xs[ei] = __dadd_rn(xs[ei], a64);
    } else if (kind == kPair) {
      if (ei % NT == tid) xs[ei] = __fma_rn(a64, T::coef(ci), xs[ei]);
      if (ej % NT == tid) xs[ej] = __fma_rn(a64, T::coef(cj), xs[ej]);
    } else {
      const StepMeta& M = meta[sa];
      for (int q = 0; q < kq; ++q) {
        const int idx = M.ks_idx[q];
        if (idx % NT == tid) xs[idx] = __fma_rn(a64, T::coef(M.ks_coef[q]), xs[idx]);
      }
    }
    if (t % a.thinning == 0) {
      const size_t row = static_cast<size_t>(t / a.thinning) * a.out_nchains + gchain;
      if (a.out_f64) {
        double* out = reinterpret_cast<double*>(a.samples) + row * d;
        for (int j = tid; j < d; j += NT) out[j] = xs[j];
      } else {
        float* out = reinterpret_cast<float*>(a.samples) + row * d;
        for (int j = tid; j < d; j += NT) out[j] = __double2float_rn(xs[j]);
      }
    }
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int r = tid + k * NT;
      if (r < m) sl[k] = T::slack_update(sl[k], alpha, ae_of(r));
    }
    __syncwarp();
    if (lane == 0) {
      mbar_arrive(&empty[sa]);
      if (kind == kPair) mbar_arrive(&empty[sb]);
    }
  }
  if (a.X_final) {
    for (int j = tid; j < d; j += NT) a.X_final[static_cast<size_t>(chain_local) * a.ldx + j] = xs[j];
  }
}

template <class Real, int NT, int R>
__global__ void __launch_bounds__(NT + 32, 1) chr_kernel(ChrArgs a, int slots) {
  extern __shared__ __align__(128) unsigned char smem[];
  const Layout L = make_layout(a.d, a.lda, sizeof(Real), NT, slots);
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
  run_consumers<Real, NT, R>(a, L, smem, chain_local);
}

// ------------------------------------------------------------- dispatch
template <class Real, int NT, int R>
int launch_one(const ChrArgs& a, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream) {
  auto kern = chr_kernel<Real, NT, R>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(cfg.smem));
  if (e != cudaSuccess) return NAJA_ERR_CUDA;
  kern<<<nchains, NT + 32, cfg.smem, stream>>>(a, cfg.slots);
  return cudaGetLastError() == cudaSuccess ? NAJA_OK : NAJA_ERR_CUDA;
}

template <class Real, int NT>
int launch_rows(const ChrArgs& a, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream) {
  switch (cfg.rows) {
    case 1: return launch_one<Real, NT, 1>(a, nchains, cfg, stream);
    case 2: return launch_one<Real, NT, 2>(a, nchains, cfg, stream);
    case 4: return launch_one<Real, NT, 4>(a, nchains, cfg, stream);
    case 8: return launch_one<Real, NT, 8>(a, nchains, cfg, stream);
    case 16: return launch_one<Real, NT, 16>(a, nchains, cfg, stream);
    case 32:
      if constexpr (NT <= 512) return launch_one<Real, NT, 32>(a, nchains, cfg, stream);
      break;
    default: break;
  }
  return NAJA_ERR_UNSUPPORTED;
}

}  // namespace
}  // namespace chr_detail
}  // namespace naja
