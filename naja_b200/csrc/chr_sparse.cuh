// Sparse-column CHR step kernel for sm_100a.
//
// Same steps, same arithmetic and the same results as chr_kernel (the
// reference's chrKernel, src/gpu/chr.cu:232-490 of quothbonney/naja), for
// constraint matrices whose columns are mostly zero: a step touches only
// the rows where its direction's column(s) of A are nonzero.
//
//   * The producer stages a column's compressed entries (value, row) into
//     the slot ring instead of the whole column.
//   * NW consumer warps per chain (1..16); entry e of a staged column goes to
//     consumer thread e % (32 NW).  The slack vector (m values, plus a
//     scratch row m that padding entries point at) lives in shared memory.
//     A step synchronises at one barrier after the column wait (every warp
//     agrees the column arrived; the previous step's slack writes become
//     visible) and one for the cross-warp max / min, plus two inside a pair
//     step.  With one warp every barrier is a __syncwarp.
//   * The chord ends are max / min over all m rows of ae/s.  A row with
//     ae = 0 contributes a signed zero (FP32 tier: +0; FP64 tier: +-0 by the
//     signs of ae and s), so when the extremes over the nonzero rows are
//     strictly positive (max) and strictly negative (min) the zero rows
//     cannot change them and the compressed pass is exact.  Otherwise (an
//     unbounded or degenerate chord) the step repeats the pass over all m
//     rows from the dense A.
//   * Slack rows with ae = 0 are not updated: s - alpha * (+-0) equals s
//     except for the sign of a zero slack, which neither tier's ratio
//     reads (a zero slack counts as +0) and which no later update can turn
//     into a different nonzero value.
//   * Pair steps combine the two columns in one of two ways (template SCAT,
//     same values either way):
//       scatter (single-model kernel, when it fits): column j is scattered
//         into a dense scratch column `ajd` (all zeros between steps), the
//         pass over column i's entries reads a_j there (0 where column j has
//         no entry) and marks the shared rows, the pass over column j's
//         entries skips the marked rows and clears the scratch -- two more
//         barriers per pair step and m values of shared memory;
//       bitmap (batched kernel, or when the scratch column does not fit):
//         both columns' rows are set in two bitmaps of m + 1 bits (atomicOr,
//         one barrier); an entry of column i whose row column j also holds
//         (its bit set) finds column j's value there by binary search in
//         column j's slot (rows ascend), and an entry of column j whose row
//         column i holds is left to that entry; the update pass clears the
//         bits.  2 (m + 1) bits instead of m + 1 values of shared memory, so
//         more chains fit on an SM, and only the few shared rows search.
//     ae = fma(a_i, c_i, a_j c_j) exactly as the dense kernel forms it.  The
//     combined values go to a shared array beside the slots; the staged
//     slots are only read.
//   * The FP64 recompute slack = b - A64 x runs over the rows of A64
//     stored by rows, columns ascending: the dense kernel's fma chain
//     without its zero terms (padding terms 0 * x_0 change at most the sign
//     of a zero sum), kSpRowGroup 16-byte entries loaded ahead of each
//     group of as many fmas.
#pragma once
#include "chr_kernel.cuh"

namespace naja {
namespace chr_detail {
namespace {

template <class Real>
struct SpEntry;
template <>
struct __align__(8) SpEntry<float> {
  float v;
  int r;
};
template <>
struct __align__(16) SpEntry<double> {
  double v;
  int r;
  int pad;
};
static_assert(sizeof(SpEntry<float>) == kSpEntryBytes32, "FP32 entry size");
static_assert(sizeof(SpEntry<double>) == kSpEntryBytes64, "FP64 entry size");

// Marker for a row shared by both columns of a pair step: -0, which no
// stored entry holds (stored values are nonzero).
__device__ __forceinline__ float sp_mark(float) { return __uint_as_float(0x80000000u); }
__device__ __forceinline__ double sp_mark(double) {
  return __longlong_as_double(static_cast<long long>(0x8000000000000000ull));
}
__device__ __forceinline__ bool sp_is_mark(float v) { return __float_as_uint(v) == 0x80000000u; }
__device__ __forceinline__ bool sp_is_mark(double v) {
  return static_cast<unsigned long long>(__double_as_longlong(v)) == 0x8000000000000000ull;
}

// 32-bit words of one row bitmap (rows 0..m, row m the padding row).
__host__ __device__ inline size_t sp_bitmap_words(int m) { return (static_cast<size_t>(m) + 32) / 32; }

// Shared memory of one chain: x (FP64), the column offsets, `slots` staged
// compressed columns of up to max_col entries, the step records and
// barriers, the cross-warp reduction entries, the abort flag followed by the
// arrival flags (2 x nw ints), slack (m + 1 values), with `scatter` the
// pair scratch column (m + 1 values), and a pair step's combined values
// (tail_off: one value per slot entry for column i's entries, then as many
// for column j's).
__host__ __device__ inline Layout make_sparse_layout(int d, int m, int elt, int eb, int max_col, int nw, int slots,
                                                     bool scatter = false) {
  Layout L;
  size_t off = 0;
  L.x_off = 0;
  off = align_up(static_cast<size_t>(d) * 8, 128);
  L.cs_off = off;
  off = align_up(off + static_cast<size_t>(d + 1) * 4, 128);
  L.slot_off = off;
  L.slot_bytes = align_up(static_cast<size_t>(max_col) * eb, 128);
  off += L.slot_bytes * slots;
  L.meta_off = off;
  off = align_up(off + sizeof(StepMeta) * slots, 16);
  L.full_off = off;
  off += 8 * static_cast<size_t>(slots);
  L.empty_off = off;
  off += 8 * static_cast<size_t>(slots);
  L.red_off = align_up(off, 16);
  off = L.red_off + sizeof(RedEntry) * 2 * nw;
  L.flag_off = align_up(off, 16);
  off = L.flag_off + 16 + 2 * static_cast<size_t>(nw) * 4;
  L.slack_off = align_up(off, 128);
  off = L.slack_off + static_cast<size_t>(m + 1) * elt;
  // the pair scratch column, or the two row bitmaps
  L.ajd_off = align_up(off, 16);
  off = L.ajd_off + (scatter ? static_cast<size_t>(m + 1) * elt : 2 * sp_bitmap_words(m) * sizeof(uint32_t));
  L.tail_off = align_up(off, 16);
  off = L.tail_off + 2 * (L.slot_bytes / eb) * elt;
  L.total = align_up(off, 128);
  L.slots = slots;
  L.direct = false;
  return L;
}

// Position of the first entry of a staged column (rows ascending) whose row
// is >= r, among its n entries.
template <class E>
__device__ __forceinline__ int sp_lower_bound(const E* col, int n, int r) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (col[mid].r < r) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Entries a consumer thread loads together in a coordinate step's passes.
constexpr int kSpBatch = 4;

// Barrier over the consumer warps (the producer warp never takes part).
template <int NW>
__device__ __forceinline__ void consumers_sync(uint32_t id) {
  if constexpr (NW == 1) {
    __syncwarp();
  } else {
    named_bar_sync(id, NW * 32);
  }
}

// The consumer warps of one chain.
template <class Real, int NW, bool SCAT>
__device__ void run_sparse_consumers(const ChrArgs& a, const SpArgs& sp, const Layout& L, unsigned char* smem,
                                     int chain_local) {
  using T = Tier<Real>;
  using Acc = typename T::Acc;
  using UT = typename T::UType;
  using E = SpEntry<Real>;
  using R64 = SpEntry<double>;
  constexpr int NT = 32 * NW;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  double* xs = reinterpret_cast<double*>(smem + L.x_off);
  const StepMeta* meta = reinterpret_cast<const StepMeta*>(smem + L.meta_off);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.full_off);
  uint64_t* empty = reinterpret_cast<uint64_t*>(smem + L.empty_off);
  RedEntry* red = reinterpret_cast<RedEntry*>(smem + L.red_off);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + L.flag_off);
  int* arrived = reinterpret_cast<int*>(smem + L.flag_off + 16);
  Real* slack = reinterpret_cast<Real*>(smem + L.slack_off);
  Real* ajd = reinterpret_cast<Real*>(smem + L.ajd_off);           // SCAT
  uint32_t* bits_j = reinterpret_cast<uint32_t*>(smem + L.ajd_off);  // !SCAT: rows of column j,
  const int nwords = static_cast<int>(sp_bitmap_words(a.m));
  uint32_t* bits_i = bits_j + nwords;                                 // then rows of column i
  Real* pv = reinterpret_cast<Real*>(smem + L.tail_off);  // combined values, column i's entries
  Real* qv = pv + L.slot_bytes / sizeof(E);                 // ... column j's entries
  const Real* A = T::A(a);
  const R64* rows = static_cast<const R64*>(sp.row_ent);
  const int m = a.m, d = a.d, lda = a.lda, S = L.slots;
  const int gchain = a.chain_base + chain_local;

  for (int j = tid; j < d; j += NT) xs[j] = a.X0[static_cast<size_t>(chain_local) * a.ldx + j];
  if constexpr (SCAT) {
    for (int r = tid; r <= m; r += NT) ajd[r] = Real(0);
  } else {
    for (int w = tid; w < 2 * nwords; w += NT) bits_j[w] = 0u;
  }
  consumers_sync<NW>(1);

  auto recompute = [&]() {
    for (int r = tid; r < m; r += NT) {
      double acc = 0.0;
      const int k1 = sp.row_start[r + 1];
      for (int k = sp.row_start[r]; k < k1; k += kSpRowGroup) {
        R64 e[kSpRowGroup];
#pragma unroll
        for (int u = 0; u < kSpRowGroup; ++u) e[u] = rows[k + u];
        double xv[kSpRowGroup];
#pragma unroll
        for (int u = 0; u < kSpRowGroup; ++u) xv[u] = xs[e[u].r];
#pragma unroll
        for (int u = 0; u < kSpRowGroup; ++u) acc = __fma_rn(e[u].v, xv[u], acc);
      }
      slack[r] = T::from64(__dsub_rn(a.b[r], acc));
    }
    if (tid == 0) slack[m] = Real(0);
  };
  if (a.slack_in) {
    const Real* si = static_cast<const Real*>(a.slack_in) + static_cast<size_t>(chain_local) * m;
    for (int r = tid; r < m; r += NT) slack[r] = si[r];
    if (tid == 0) slack[m] = Real(0);
  } else {
    recompute();
  }
  consumers_sync<NW>(1);

  // Cross-warp max / min: lane 0 of each warp posts, one barrier, every
  // warp reduces the posted entries.  The halves of `red` alternate.
  int rbuf = 0;
  auto reduce = [&](Acc& hi, Acc& lo, Acc& lo2) {
    hi = T::red_hi(hi);
    lo = T::red_lo(lo);
    lo2 = T::red_lo2(lo2);
    if constexpr (NW > 1) {
      RedEntry* slotr = red + rbuf * NW;
      rbuf ^= 1;
      if (lane == 0) {
        slotr[warp].kmax = hi;
        slotr[warp].kmin = lo;
        slotr[warp].kmin2 = lo2;
      }
      named_bar_sync(1, NT);
      Acc h = T::acc_hi0(), l = T::acc_lo0(), l2 = T::acc_lo20();
      if (lane < NW) {
        h = static_cast<Acc>(slotr[lane].kmax);
        l = static_cast<Acc>(slotr[lane].kmin);
        l2 = static_cast<Acc>(slotr[lane].kmin2);
      }
      hi = T::red_hi(h);
      lo = T::red_lo(l);
      lo2 = T::red_lo2(l2);
    }
  };

  // global step counters as in the dense kernel (ChrArgs::t_first)
  const long long total = launch_steps(a);
  int slot = 0;
  uint32_t parity = 0;
  int thin_ctr = static_cast<int>(a.t_first % a.thinning);
  int resync_ctr = a.resync > 0 ? static_cast<int>(a.t_first % a.resync) : 0;
  int abuf = 0;
  size_t out_row = static_cast<size_t>(gchain) +
                   static_cast<size_t>((a.t_first + a.thinning - 1) / a.thinning) * a.out_nchains;
  unsigned long long w_full = 0;
  const unsigned long long c_start = clock64();
  for (long long t = 0; t < total; ++t) {
    const int sa = slot;
    const unsigned long long w0 = a.wait_cycles ? clock64() : 0ull;
    bool ok = mbar_wait_bounded(&full[sa], parity, a.timeout_ns);
    if (a.wait_cycles) w_full += clock64() - w0;
    int kind = kCoord, ei = 0, ej = 0, sb = -1, na = 0, nb = 0;
    Real cir = Real(1), cjr = Real(0);
    UT uu = UT(0.5);
    double cix = 1.0, cjx = 0.0;
    if (ok) {
      const StepMeta& M = meta[sa];
      const int4 h0 = *reinterpret_cast<const int4*>(&M.kind);
      const int4 h1 = *reinterpret_cast<const int4*>(&M.k);
      const int2 hn = *reinterpret_cast<const int2*>(&M.na);
      kind = h0.x;
      ei = h0.y;
      ej = h0.z;
      sb = h0.w;
      na = hn.x;
      nb = hn.y;
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
    // Every warp agrees that the step's columns arrived before any barrier
    // that depends on the step's kind; this barrier also publishes the
    // previous step's slack writes.
    ok = __all_sync(0xffffffffu, ok);
    if constexpr (NW > 1) {
      int* af = arrived + abuf * NW;
      abuf ^= 1;
      if (lane == 0) af[warp] = ok ? 1 : 0;
      named_bar_sync(3, NT);
      ok = __all_sync(0xffffffffu, lane >= NW || af[lane] != 0);
    }
    if (!ok) {
      if (tid == 0) {
        set_error(a.err, kDevTimeoutFull, sa, static_cast<int>(parity), static_cast<int>(t));
        *abort_flag = 1;
      }
      return;
    }
    if (a.resync > 0) {
      // the recompute before the loop is step 0's
      if (resync_ctr == 0 && t != 0) {
        recompute();
        consumers_sync<NW>(2);
      }
      if (++resync_ctr == a.resync) resync_ctr = 0;
    }
    const E* ea = reinterpret_cast<const E*>(smem + L.slot_off + static_cast<size_t>(sa) * L.slot_bytes);
    const E* eb =
        reinterpret_cast<const E*>(smem + L.slot_off + static_cast<size_t>(sb < 0 ? 0 : sb) * L.slot_bytes);
    Acc hi = T::acc_hi0(), lo = T::acc_lo0(), lo2 = T::acc_lo20();
    if (kind == kPair && SCAT) {
#pragma unroll 4
      for (int e = tid; e < nb; e += NT) {
        const E q = eb[e];
        ajd[q.r] = q.v;
      }
      consumers_sync<NW>(3);
#pragma unroll 4
      for (int e = tid; e < na; e += NT) {
        const E q = ea[e];
        const Real w = ajd[q.r];
        const Real ae = T::pair_ae_r(q.v, w, cir, cjr);
        if (w != Real(0)) ajd[q.r] = sp_mark(Real(0));
        pv[e] = ae;
        T::acc(hi, lo, lo2, T::ratio(ae, slack[q.r]));
      }
      consumers_sync<NW>(3);
#pragma unroll 4
      for (int e = tid; e < nb; e += NT) {
        const E q = eb[e];
        const Real w = ajd[q.r];
        ajd[q.r] = Real(0);
        // a row shared with column i was taken with that entry: the marker
        // (-0) makes this entry's update a no-op below
        Real ae = sp_mark(Real(0));
        if (!sp_is_mark(w)) {
          ae = T::pair_ae_r(Real(0), q.v, cir, cjr);
          T::acc(hi, lo, lo2, T::ratio(ae, slack[q.r]));
        }
        qv[e] = ae;
      }
    } else if (kind == kPair) {
      for (int e = tid; e < nb; e += NT) {
        const int r = eb[e].r;
        atomicOr(&bits_j[r >> 5], 1u << (r & 31));
      }
      for (int e = tid; e < na; e += NT) {
        const int r = ea[e].r;
        atomicOr(&bits_i[r >> 5], 1u << (r & 31));
      }
      consumers_sync<NW>(3);
      // rows of column i, each with column j's value at that row (0 if none);
      // kSpBatch entries per thread at a time, loads first
      for (int e0 = tid; e0 < na; e0 += kSpBatch * NT) {
        E q[kSpBatch];
        uint32_t bw[kSpBatch];
        Real sv[kSpBatch];
#pragma unroll
        for (int u = 0; u < kSpBatch; ++u) q[u] = e0 + u * NT < na ? ea[e0 + u * NT] : E{Real(0), m};
#pragma unroll
        for (int u = 0; u < kSpBatch; ++u) {
          bw[u] = bits_j[q[u].r >> 5];
          sv[u] = slack[q[u].r];
        }
#pragma unroll
        for (int u = 0; u < kSpBatch; ++u) {
          const int e = e0 + u * NT;
          if (e < na) {
            Real w = Real(0);
            if ((bw[u] >> (q[u].r & 31)) & 1u) w = eb[sp_lower_bound(eb, nb, q[u].r)].v;
            const Real ae = T::pair_ae_r(q[u].v, w, cir, cjr);
            pv[e] = ae;
            T::acc(hi, lo, lo2, T::ratio(ae, sv[u]));
          }
        }
      }
      // rows of column j that column i does not hold; a shared row was taken
      // with column i's entry, and the marker (-0) makes this entry's update
      // a no-op below
      for (int e0 = tid; e0 < nb; e0 += kSpBatch * NT) {
        E q[kSpBatch];
        uint32_t bw[kSpBatch];
        Real sv[kSpBatch];
#pragma unroll
        for (int u = 0; u < kSpBatch; ++u) q[u] = e0 + u * NT < nb ? eb[e0 + u * NT] : E{Real(0), m};
#pragma unroll
        for (int u = 0; u < kSpBatch; ++u) {
          bw[u] = bits_i[q[u].r >> 5];
          sv[u] = slack[q[u].r];
        }
#pragma unroll
        for (int u = 0; u < kSpBatch; ++u) {
          const int e = e0 + u * NT;
          if (e < nb) {
            Real ae = sp_mark(Real(0));
            if (!((bw[u] >> (q[u].r & 31)) & 1u)) {
              ae = T::pair_ae_r(Real(0), q[u].v, cir, cjr);
              T::acc(hi, lo, lo2, T::ratio(ae, sv[u]));
            }
            qv[e] = ae;
          }
        }
      }
      // the update pass clears bits other threads tested: with more than one
      // warp the reduction's barrier orders the two, with one warp this
      if constexpr (NW == 1) __syncwarp();
    } else {
      // kSpBatch entries per thread at a time: their loads are all issued
      // before the first ratio needs one (the per-entry chain is load, load,
      // divide)
      for (int e0 = tid; e0 < na; e0 += kSpBatch * NT) {
        E q[kSpBatch];
        Real sv[kSpBatch];
#pragma unroll
        for (int u = 0; u < kSpBatch; ++u) {
          const int e = e0 + u * NT;
          q[u] = e < na ? ea[e] : E{Real(0), m};
        }
#pragma unroll
        for (int u = 0; u < kSpBatch; ++u) sv[u] = slack[q[u].r];
#pragma unroll
        for (int u = 0; u < kSpBatch; ++u)
          if (e0 + u * NT < na) T::acc(hi, lo, lo2, T::ratio(q[u].v, sv[u]));
      }
    }
    reduce(hi, lo, lo2);
    Real mx, mn;
    T::decode(hi, lo, lo2, mx, mn);
    if (!(mx > Real(0) && mn < Real(0))) {
      // Some zero row may hold an extreme: repeat the pass over all rows.
      hi = T::acc_hi0();
      lo = T::acc_lo0();
      lo2 = T::acc_lo20();
      const Real* ca = A + static_cast<size_t>(ei) * lda;
      if (kind == kPair) {
        const Real* cb = A + static_cast<size_t>(ej) * lda;
        for (int r = tid; r < m; r += NT) T::acc(hi, lo, lo2, T::ratio(T::pair_ae_r(ca[r], cb[r], cir, cjr), slack[r]));
      } else {
        for (int r = tid; r < m; r += NT) T::acc(hi, lo, lo2, T::ratio(ca[r], slack[r]));
      }
      reduce(hi, lo, lo2);
      T::decode(hi, lo, lo2, mx, mn);
    }
    const Real alpha = T::alpha(mx, mn, uu);
    const double a64 = static_cast<double>(alpha);
    if (kind == kCoord) {
      if (ei % NT == tid) xs[ei] = __dadd_rn(xs[ei], a64);
    } else {
      if (ei % NT == tid) xs[ei] = __fma_rn(a64, cix, xs[ei]);
      if (ej % NT == tid) xs[ej] = __fma_rn(a64, cjx, xs[ej]);
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
    // Slack update of the rows the step touched, each by the thread that
    // read its entry.  A pair step's rows take the combined values; an entry
    // holding the marker (a row already updated through column i, or a
    // combined value of -0, whose update would only change the sign of a
    // zero slack) is skipped.
    if (kind == kPair) {
      // (bitmap variant: every bit the step set is cleared here, after the
      // reduction's barrier, so the next pair step starts from zeros)
#pragma unroll 4
      for (int e = tid; e < na; e += NT) {
        const int r = ea[e].r;
        slack[r] = T::slack_update(slack[r], alpha, pv[e]);
        if constexpr (!SCAT) atomicAnd(&bits_i[r >> 5], ~(1u << (r & 31)));
      }
#pragma unroll 4
      for (int e = tid; e < nb; e += NT) {
        const Real ae = qv[e];
        const int r = eb[e].r;
        if (!sp_is_mark(ae)) slack[r] = T::slack_update(slack[r], alpha, ae);
        if constexpr (!SCAT) atomicAnd(&bits_j[r >> 5], ~(1u << (r & 31)));
      }
    } else {
      for (int e0 = tid; e0 < na; e0 += kSpBatch * NT) {
        E q[kSpBatch];
        Real sv[kSpBatch];
#pragma unroll
        for (int u = 0; u < kSpBatch; ++u) {
          const int e = e0 + u * NT;
          q[u] = e < na ? ea[e] : E{Real(0), m};
        }
#pragma unroll
        for (int u = 0; u < kSpBatch; ++u) sv[u] = slack[q[u].r];
        // entries past na stand for the scratch row m and are not written
#pragma unroll
        for (int u = 0; u < kSpBatch; ++u)
          if (e0 + u * NT < na) slack[q[u].r] = T::slack_update(sv[u], alpha, q[u].v);
      }
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
  if (a.slack_final) {
    consumers_sync<NW>(1);  // every thread's last slack writes are visible
    Real* so = static_cast<Real*>(a.slack_final) + static_cast<size_t>(chain_local) * m;
    for (int r = tid; r < m; r += NT) so[r] = slack[r];
  }
  if (a.wait_cycles && tid == 0) {
    a.wait_cycles[4 * chain_local + 0] = w_full;
    a.wait_cycles[4 * chain_local + 2] = clock64() - c_start;
  }
}

template <class Real, int NW, bool SCAT>
__global__ void __launch_bounds__(NW * 32 + 32, 1)
    chr_sparse_kernel(const __grid_constant__ ChrArgs a, const __grid_constant__ SpArgs sp,
                      const __grid_constant__ Layout L) {
  extern __shared__ __align__(128) unsigned char smem[];
  constexpr int NT = NW * 32;
  int* cs = reinterpret_cast<int*>(smem + L.cs_off);
  if (threadIdx.x == 0) {
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.full_off);
    uint64_t* empty = reinterpret_cast<uint64_t*>(smem + L.empty_off);
    for (int s = 0; s < L.slots; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NW);
    }
    *reinterpret_cast<volatile int*>(smem + L.flag_off) = 0;
    fence_mbar_init();
  }
  for (int j = threadIdx.x; j <= a.d; j += blockDim.x) cs[j] = sp.col_start[j];
  __syncthreads();
  if (threadIdx.x >= NT) {
    if (threadIdx.x == NT)
      producer_entry<Real, true>(a, L, smem, blockIdx.x, &sp, cs, static_cast<int>(sizeof(SpEntry<Real>)));
    return;
  }
  run_sparse_consumers<Real, NW, SCAT>(a, sp, L, smem, blockIdx.x);
}

template <class Real, int NW, bool SCAT>
int launch_sparse(const ChrArgs& a, const SpArgs& sp, int nchains, const ChrLaunchConfig& cfg, cudaStream_t stream) {
  auto kern = chr_sparse_kernel<Real, NW, SCAT>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(cfg.smem));
  if (e != cudaSuccess) return NAJA_ERR_CUDA;
  const Layout L =
      make_sparse_layout(a.d, a.m, sizeof(Real), sizeof(SpEntry<Real>), cfg.max_col, NW, cfg.slots, SCAT);
  kern<<<nchains, NW * 32 + 32, cfg.smem, stream>>>(a, sp, L);
  return cudaGetLastError() == cudaSuccess ? NAJA_OK : NAJA_ERR_CUDA;
}

template <class Real>
int launch_sparse_nw(const ChrArgs& a, const SpArgs& sp, int nchains, const ChrLaunchConfig& cfg,
                     cudaStream_t stream) {
  const bool sc = cfg.pair_scatter != 0;
  switch (cfg.threads) {
    case 32: return sc ? launch_sparse<Real, 1, true>(a, sp, nchains, cfg, stream)
                       : launch_sparse<Real, 1, false>(a, sp, nchains, cfg, stream);
    case 64: return sc ? launch_sparse<Real, 2, true>(a, sp, nchains, cfg, stream)
                       : launch_sparse<Real, 2, false>(a, sp, nchains, cfg, stream);
    case 128: return sc ? launch_sparse<Real, 4, true>(a, sp, nchains, cfg, stream)
                        : launch_sparse<Real, 4, false>(a, sp, nchains, cfg, stream);
    case 256: return sc ? launch_sparse<Real, 8, true>(a, sp, nchains, cfg, stream)
                        : launch_sparse<Real, 8, false>(a, sp, nchains, cfg, stream);
    case 512: return sc ? launch_sparse<Real, 16, true>(a, sp, nchains, cfg, stream)
                        : launch_sparse<Real, 16, false>(a, sp, nchains, cfg, stream);
    default: return NAJA_ERR_UNSUPPORTED;
  }
}

}  // namespace
}  // namespace chr_detail
}  // namespace naja

namespace naja {
namespace chr_detail {
namespace {

// Batched multi-model run on the compressed-column kernel: the persistent
// item loop of chr_batched_kernel (one item = one chain of one model; the
// CTA re-initialises its mbarriers between items, after the producer has
// drained its copies and every consumer has released its slots), with each
// model's compressed columns and FP32 tier.  Layout sized for the largest
// model and the longest column of any model.
template <int NW>
__global__ void __launch_bounds__(NW * 32 + 32, NW >= 8 ? 2 : (NW == 4 ? 4 : 6))
    chr_batched_sparse_kernel(const __grid_constant__ ChrArgs base, const __grid_constant__ Layout L,
                              const ModelDesc* __restrict__ models, const int* __restrict__ item_model,
                              const int* __restrict__ item_chain, int nitems) {
  using Real = float;
  constexpr int NT = NW * 32;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ ChrArgs item_args;
  __shared__ SpArgs item_sp;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.full_off);
  uint64_t* empty = reinterpret_cast<uint64_t*>(smem + L.empty_off);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + L.flag_off);
  int* cs = reinterpret_cast<int*>(smem + L.cs_off);
  if (threadIdx.x == 0) *abort_flag = 0;
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    const int ch = item_chain[item];
    if (threadIdx.x == 0) {
      for (int s = 0; s < L.slots; ++s) {
        mbar_init(&full[s], 1);
        mbar_init(&empty[s], NW);
      }
      fence_mbar_init();
      const ModelDesc& md = models[item_model[item]];
      ChrArgs a = base;
      a.A32 = md.A32;
      a.A64 = md.A64;
      a.lda = md.lda;
      a.m = md.m;
      a.b = md.b;
      a.X0 = md.X0;
      a.ldx = md.ldx;
      a.samples = md.samples;
      a.X_final = md.X_final;
      a.seed = md.seed;
      a.chain_base = 0;
      a.rng_state = nullptr;
      a.wait_cycles = nullptr;
      a.slack_final = nullptr;
      item_args = a;
      item_sp = md.sp;
    }
    __syncthreads();
    if (*abort_flag) break;  // every thread reads it after the barrier
    for (int j = threadIdx.x; j <= item_args.d; j += blockDim.x) cs[j] = item_sp.col_start[j];
    __syncthreads();
    if (threadIdx.x >= NT) {
      if (threadIdx.x == NT)
        producer_entry<Real, true>(item_args, L, smem, ch, &item_sp, cs, static_cast<int>(sizeof(SpEntry<Real>)));
    } else {
      run_sparse_consumers<Real, NW, false>(item_args, item_sp, L, smem, ch);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int s = 0; s < L.slots; ++s) {
        mbar_inval(&full[s]);
        mbar_inval(&empty[s]);
      }
    }
  }
}

template <int NW>
int batch_sparse_one(const ChrArgs* base, const ModelDesc* models, const int* im, const int* ic, int nitems,
                     const BatchConfig& cfg, cudaStream_t stream, int* occ_out) {
  auto kern = chr_batched_sparse_kernel<NW>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(cfg.smem));
  if (e != cudaSuccess) return NAJA_ERR_CUDA;
  int occ = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, NW * 32 + 32, cfg.smem);
  if (e != cudaSuccess) return NAJA_ERR_CUDA;
  if (occ_out) {
    *occ_out = occ;
    return NAJA_OK;
  }
  if (occ < 1) return NAJA_ERR_UNSUPPORTED;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int per_sm = cfg.ctas_per_sm > 0 ? (cfg.ctas_per_sm < occ ? cfg.ctas_per_sm : occ) : occ;
  const int grid = nitems < sms * per_sm ? nitems : sms * per_sm;
  const Layout L = make_sparse_layout(base->d, cfg.lda_max, sizeof(float), sizeof(SpEntry<float>), cfg.max_col, NW,
                                      cfg.slots);
  kern<<<grid, NW * 32 + 32, cfg.smem, stream>>>(*base, L, models, im, ic, nitems);
  return cudaGetLastError() == cudaSuccess ? NAJA_OK : NAJA_ERR_CUDA;
}

}  // namespace
}  // namespace chr_detail
}  // namespace naja
