// Split-precision tensor-core backmap V = Y T^T + shift on sm_100a (tcgen05).
//
// GEMM view: D (M x N) = A (M x K) B (N x K)^T with A = samples Y (K-major,
// one row per sample), B = T (K-major after a transpose), K = d.  FP32 values
// are carried by two lower-precision terms, x = hi + lo, and the product is
// taken as hi*hi + hi*lo + lo*hi (the lo*lo term is below the terms' own
// rounding), accumulated in FP32 in tensor memory:
//   BF16X3 : hi = bf16(x), lo = bf16(x - hi)            (kind::f16, BF16 in)
//   TF32X3 : hi = tf32(x), lo = tf32(x - hi)            (kind::tf32)
//
// Organisation (one CTA per SM, persistent over 128 x 256 output tiles,
// tiles ordered n-fastest so a sample block stays in L2 across its n tiles):
//   warp 4, one thread : TMA producer.  2-D tiled bulk-tensor loads with
//                        128-byte swizzle of A_hi, A_lo, B_hi, B_lo for one
//                        128-byte K slice into a 2-stage shared-memory ring.
//   warp 5, one thread : MMA issuer.  Per stage 4 K-steps x 3 tcgen05.mma
//                        into one of two 128 x 256 FP32 accumulators in TMEM
//                        (512 columns; tiles alternate), so a tile's MMAs run
//                        while the epilogue drains the previous tile; the
//                        stage is released with tcgen05.commit.
//   warps 0-3          : epilogue.  tcgen05.ld of their 32 TMEM lanes, 32 x 32
//                        blocks transposed through shared memory, + shift,
//                        stores of 32 consecutive values of a row each.
// Every wait is bounded (global timer); on expiry the CTA records an error,
// stops issuing, drains its own copies / MMAs and frees TMEM before exiting.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/naja_chr.h"
#include "capi_internal.cuh"
#include "common.cuh"

namespace naja {
namespace {

constexpr int kTileM = 128;
constexpr int kTileN = 256;
constexpr int kSliceBytes = 128;  // K extent of one stage, in bytes per row
constexpr int kStages = 2;
constexpr int kThreads = 192;     // warps 0-3 epilogue, 4 producer, 5 MMA
constexpr uint32_t kTmemCols = 512;  // two 256-column accumulators
constexpr uint64_t kTimeoutNs = 5ull * 1000 * 1000 * 1000;

constexpr uint32_t kATileBytes = kTileM * kSliceBytes;  // 16 KB
constexpr uint32_t kBTileBytes = kTileN * kSliceBytes;  // 32 KB
constexpr uint32_t kStageBytes = 2 * kATileBytes + 2 * kBTileBytes;

enum TcError : int { kTcTimeoutLoad = 11, kTcTimeoutSlot = 12, kTcTimeoutAcc = 13, kTcTimeoutEpi = 14 };

struct TcArgs {
  int n, kslices;
  long long N;
  int tiles_n;
  long long tiles;
  const double* shift;
  void* V;
  int v_f64;
  int* err;
};

// ------------------------------------------------------------ PTX wrappers
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// K-major, 128-byte-swizzled operand: 8-row core groups 1024 B apart.
__device__ __forceinline__ uint64_t umma_desc_sw128(const void* smem) {
  const uint64_t addr = smem_u32(smem);
  uint64_t d = 0;
  d |= (addr >> 4) & 0x3FFFull;              // start address
  d |= static_cast<uint64_t>(1) << 16;        // leading byte offset (unused with swizzle)
  d |= static_cast<uint64_t>(1024 >> 4) << 32;  // stride byte offset
  d |= static_cast<uint64_t>(1) << 46;        // descriptor version (sm100)
  d |= static_cast<uint64_t>(2) << 61;        // SWIZZLE_128B
  return d;
}

template <bool TF32>
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
  if constexpr (TF32) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
  }
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ------------------------------------------------------------------ kernel
template <bool TF32>
__global__ void __launch_bounds__(kThreads, 1)
    backmap_tc_kernel(const __grid_constant__ CUtensorMap mAhi, const __grid_constant__ CUtensorMap mAlo,
                      const __grid_constant__ CUtensorMap mBhi, const __grid_constant__ CUtensorMap mBlo, TcArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte alignment for the swizzled tiles
  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* acc_full = empty + kStages;  // [2]
  uint64_t* acc_empty = acc_full + 2;    // [2]
  uint64_t* drain_bar = acc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain_bar + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  // epilogue staging: one 32 x 33 float block per epilogue warp
  float* stage_out = reinterpret_cast<float*>(smem + kStages * kStageBytes + 256);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&acc_full[0], 1);
    mbar_init(&acc_full[1], 1);
    mbar_init(&acc_empty[0], 4);
    mbar_init(&acc_empty[1], 4);
    mbar_init(drain_bar, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  const int K = a.kslices;
  if (warp == 4) {
    if (lane == 0) {
      // ---------------- TMA producer
      int stage = 0;
      uint32_t round = 0;
      uint32_t last_parity = 0, used = 0;
      const int elem_per_slice = TF32 ? 32 : 64;
      for (long long tile = blockIdx.x; tile < a.tiles && !*abort_flag; tile += gridDim.x) {
        const int tm = static_cast<int>(tile / a.tiles_n), tn = static_cast<int>(tile % a.tiles_n);
        for (int ks = 0; ks < K; ++ks) {
          if (round >= 1 && !mbar_wait_bounded(&empty[stage], (round - 1) & 1u, kTimeoutNs)) {
            set_error(a.err, kTcTimeoutSlot, static_cast<int>(blockIdx.x), stage, ks);
            *abort_flag = 1;
            break;
          }
          unsigned char* st = smem + stage * kStageBytes;
          mbar_arrive_expect_tx(&full[stage], kStageBytes);
          const int x = ks * elem_per_slice;
          tma_load_2d(st, &mAhi, x, tm * kTileM, &full[stage]);
          tma_load_2d(st + kATileBytes, &mAlo, x, tm * kTileM, &full[stage]);
          tma_load_2d(st + 2 * kATileBytes, &mBhi, x, tn * kTileN, &full[stage]);
          tma_load_2d(st + 2 * kATileBytes + kBTileBytes, &mBlo, x, tn * kTileN, &full[stage]);
          used |= 1u << stage;
          last_parity = (last_parity & ~(1u << stage)) | ((round & 1u) << stage);
          if (++stage == kStages) {
            stage = 0;
            ++round;
          }
        }
      }
      // drain: every issued load has landed before the CTA may exit
      for (int s = 0; s < kStages; ++s)
        if (((used >> s) & 1u) && !mbar_wait_bounded(&full[s], (last_parity >> s) & 1u, kTimeoutNs))
          set_error(a.err, kTcTimeoutLoad, static_cast<int>(blockIdx.x), s, -1);
    }
  } else if (warp == 5) {
    if (lane == 0) {
      // ---------------- MMA issuer
      constexpr uint32_t fmt = TF32 ? 2u : 1u;
      const uint32_t idesc = (1u << 4) | (fmt << 7) | (fmt << 10) | (static_cast<uint32_t>(kTileN >> 3) << 17) |
                             (static_cast<uint32_t>(kTileM >> 4) << 24);
      constexpr int ksteps = 4;             // 4 MMAs of 32 bytes of K per 128-byte slice
      int stage = 0;
      uint32_t parity = 0;
      uint32_t acc_round = 0;  // tiles issued by this CTA; accumulator acc_round & 1
      bool issued = false;
      for (long long tile = blockIdx.x; tile < a.tiles && !*abort_flag; tile += gridDim.x) {
        const uint32_t buf = acc_round & 1u, use = acc_round >> 1;
        const uint32_t tacc = tmem + buf * static_cast<uint32_t>(kTileN);
        // the epilogue has read this accumulator's previous tile (two tiles back)
        if (use >= 1 && !mbar_wait_bounded(&acc_empty[buf], (use - 1) & 1u, kTimeoutNs)) {
          set_error(a.err, kTcTimeoutEpi, static_cast<int>(blockIdx.x), static_cast<int>(acc_round), -1);
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        bool ok = true;
        for (int ks = 0; ks < K; ++ks) {
          if (!mbar_wait_bounded(&full[stage], parity, kTimeoutNs)) {
            set_error(a.err, kTcTimeoutLoad, static_cast<int>(blockIdx.x), stage, ks);
            *abort_flag = 1;
            ok = false;
            break;
          }
          tc_fence_after();
          unsigned char* st = smem + stage * kStageBytes;
          const unsigned char* Ahi = st;
          const unsigned char* Alo = st + kATileBytes;
          const unsigned char* Bhi = st + 2 * kATileBytes;
          const unsigned char* Blo = st + 2 * kATileBytes + kBTileBytes;
#pragma unroll
          for (int kk = 0; kk < ksteps; ++kk) {
            const uint64_t ah = umma_desc_sw128(Ahi + kk * 32), al = umma_desc_sw128(Alo + kk * 32);
            const uint64_t bh = umma_desc_sw128(Bhi + kk * 32), bl = umma_desc_sw128(Blo + kk * 32);
            const uint32_t acc = (ks > 0 || kk > 0) ? 1u : 0u;
            umma<TF32>(tacc, ah, bh, idesc, acc);
            umma<TF32>(tacc, ah, bl, idesc, 1u);
            umma<TF32>(tacc, al, bh, idesc, 1u);
          }
          issued = true;
          umma_commit(&empty[stage]);  // the stage is free once these MMAs have read it
          if (++stage == kStages) {
            stage = 0;
            parity ^= 1u;
          }
        }
        if (!ok) break;
        umma_commit(&acc_full[buf]);  // accumulator complete
        ++acc_round;
      }
      if (issued) {
        // every MMA of this CTA has finished before TMEM is released
        umma_commit(drain_bar);
        if (!mbar_wait_bounded(drain_bar, 0u, kTimeoutNs)) set_error(a.err, kTcTimeoutAcc, static_cast<int>(blockIdx.x), -1, -1);
      }
    }
  } else {
    // ---------------- epilogue, warps 0-3: TMEM lanes 32*warp .. 32*warp+31
    // Each 32 x 32 block goes through shared memory so that every store
    // instruction writes 32 consecutive values of one output row.  The
    // other accumulator takes the next tile's MMAs meanwhile.
    float* stg = stage_out + warp * (32 * 33);
    uint32_t acc_round = 0;
    for (long long tile = blockIdx.x; tile < a.tiles; tile += gridDim.x) {
      const uint32_t buf = acc_round & 1u, use = acc_round >> 1;
      bool ok = mbar_wait_bounded(&acc_full[buf], use & 1u, kTimeoutNs);
      if (!__all_sync(0xffffffffu, ok)) {
        if (lane == 0) set_error(a.err, kTcTimeoutAcc, static_cast<int>(blockIdx.x), warp, static_cast<int>(acc_round));
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
      const int tm = static_cast<int>(tile / a.tiles_n), tn = static_cast<int>(tile % a.tiles_n);
      const long long row_base = static_cast<long long>(tm) * kTileM + warp * 32;
      const int col0 = tn * kTileN;
#pragma unroll 1
      for (int c = 0; c < kTileN; c += 32) {
        uint32_t r[32];
        tmem_ld32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + buf * static_cast<uint32_t>(kTileN) +
                      static_cast<uint32_t>(c),
                  r);
#pragma unroll
        for (int q = 0; q < 32; ++q) stg[lane * 33 + q] = __uint_as_float(r[q]);
        __syncwarp();
        const int i = col0 + c + lane;
        const bool col_ok = i < a.n;
        const double sh = col_ok ? a.shift[i] : 0.0;
        if (a.v_f64) {
#pragma unroll 4
          for (int j = 0; j < 32; ++j) {
            const long long row = row_base + j;
            if (row < a.N && col_ok)
              reinterpret_cast<double*>(a.V)[row * a.n + i] = static_cast<double>(stg[j * 33 + lane]) + sh;
          }
        } else {
#pragma unroll 4
          for (int j = 0; j < 32; ++j) {
            const long long row = row_base + j;
            if (row < a.N && col_ok)
              reinterpret_cast<float*>(a.V)[row * a.n + i] =
                  static_cast<float>(static_cast<double>(stg[j * 33 + lane]) + sh);
          }
        }
        __syncwarp();
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[buf]);
      ++acc_round;
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// ----------------------------------------------------------- operand split
// Y (N x d, row-major, float or double) -> hi, lo (N x dp, row-major), zero
// for k >= d.  T (n x d column-major, ldt) -> hi, lo (n x dp row-major).
template <class YT, bool TF32>
__global__ void split_rows_kernel(const YT* __restrict__ Y, long long N, int d, int dp, void* hi, void* lo) {
  const long long total = N * dp;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long s = e / dp;
    const int k = static_cast<int>(e % dp);
    const float x = (k < d) ? static_cast<float>(Y[s * d + k]) : 0.0f;
    if constexpr (TF32) {
      uint32_t h;
      asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
      const float hf = __uint_as_float(h);
      uint32_t l;
      asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(x - hf));
      reinterpret_cast<uint32_t*>(hi)[e] = h;
      reinterpret_cast<uint32_t*>(lo)[e] = l;
    } else {
      const __nv_bfloat16 h = __float2bfloat16_rn(x);
      const __nv_bfloat16 l = __float2bfloat16_rn(x - __bfloat162float(h));
      reinterpret_cast<__nv_bfloat16*>(hi)[e] = h;
      reinterpret_cast<__nv_bfloat16*>(lo)[e] = l;
    }
  }
}

template <bool TF32>
__global__ void split_T_kernel(const double* __restrict__ T, int ldt, int n, int d, int dp, void* hi, void* lo) {
  const long long total = static_cast<long long>(n) * dp;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e / dp);
    const int k = static_cast<int>(e % dp);
    const float x = (k < d) ? static_cast<float>(T[static_cast<long long>(k) * ldt + i]) : 0.0f;
    if constexpr (TF32) {
      uint32_t h;
      asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
      uint32_t l;
      asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(x - __uint_as_float(h)));
      reinterpret_cast<uint32_t*>(hi)[e] = h;
      reinterpret_cast<uint32_t*>(lo)[e] = l;
    } else {
      const __nv_bfloat16 h = __float2bfloat16_rn(x);
      reinterpret_cast<__nv_bfloat16*>(hi)[e] = h;
      reinterpret_cast<__nv_bfloat16*>(lo)[e] = __float2bfloat16_rn(x - __bfloat162float(h));
    }
  }
}

// ------------------------------------------------------------ tensor maps
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// 2-D map over a row-major rows x dp matrix; box = box_rows x (128 bytes).
bool make_map(CUtensorMap* m, void* base, bool tf32, long long rows, int dp, int box_rows) {
  auto fn = encode_fn();
  if (!fn) return false;
  const CUtensorMapDataType dt = tf32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
  const int esz = tf32 ? 4 : 2;
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(dp), static_cast<cuuint64_t>(rows)};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(dp) * esz};
  cuuint32_t box[2] = {static_cast<cuuint32_t>(kSliceBytes / esz), static_cast<cuuint32_t>(box_rows)};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, dt, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace

size_t backmap_tc_operand_bytes(long long rows, int d, int mode) {
  const size_t esz = mode == NAJA_BACKMAP_TF32X3 ? 4 : 2;
  const size_t dp = static_cast<size_t>((d + 63) / 64 * 64);
  return (static_cast<size_t>(rows) * dp * esz + 1023) / 1024 * 1024;
}

int backmap_tc_split_T(int n, int d, const double* T, int ldt, void* Th, void* Tl, int mode, cudaStream_t stream) {
  const int dp = (d + 63) / 64 * 64;
  const int sblocks = 148 * 8;
  if (mode == NAJA_BACKMAP_TF32X3)
    split_T_kernel<true><<<sblocks, 256, 0, stream>>>(T, ldt, n, d, dp, Th, Tl);
  else
    split_T_kernel<false><<<sblocks, 256, 0, stream>>>(T, ldt, n, d, dp, Th, Tl);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("backmap: split launch failed: ") + cudaGetErrorString(e));
  return NAJA_OK;
}

int backmap_tc_enqueue(int n, int d, long long N, const void* Y, int y_dtype, const void* Th, const void* Tl, void* Yh,
                       void* Yl, const double* shift, void* V, int v_dtype, int mode, int* err, cudaStream_t stream) {
  const bool tf32 = mode == NAJA_BACKMAP_TF32X3;
  const int esz = tf32 ? 4 : 2;
  const int dp = (d + 63) / 64 * 64;
  const int sblocks = 148 * 8;
  if (tf32) {
    if (y_dtype == NAJA_DTYPE_F64)
      split_rows_kernel<double, true><<<sblocks, 256, 0, stream>>>(static_cast<const double*>(Y), N, d, dp, Yh, Yl);
    else
      split_rows_kernel<float, true><<<sblocks, 256, 0, stream>>>(static_cast<const float*>(Y), N, d, dp, Yh, Yl);
  } else {
    if (y_dtype == NAJA_DTYPE_F64)
      split_rows_kernel<double, false><<<sblocks, 256, 0, stream>>>(static_cast<const double*>(Y), N, d, dp, Yh, Yl);
    else
      split_rows_kernel<float, false><<<sblocks, 256, 0, stream>>>(static_cast<const float*>(Y), N, d, dp, Yh, Yl);
  }
  CUtensorMap mAh, mAl, mBh, mBl;
  if (!make_map(&mAh, Yh, tf32, N, dp, kTileM) || !make_map(&mAl, Yl, tf32, N, dp, kTileM) ||
      !make_map(&mBh, const_cast<void*>(Th), tf32, n, dp, kTileN) ||
      !make_map(&mBl, const_cast<void*>(Tl), tf32, n, dp, kTileN))
    return fail(NAJA_ERR_CUDA, "backmap: cuTensorMapEncodeTiled failed");
  TcArgs a;
  a.n = n;
  a.kslices = dp * esz / kSliceBytes;
  a.N = N;
  a.tiles_n = (n + kTileN - 1) / kTileN;
  a.tiles = ((N + kTileM - 1) / kTileM) * a.tiles_n;
  a.shift = shift;
  a.V = V;
  a.v_f64 = v_dtype == NAJA_DTYPE_F64;
  a.err = err;
  const size_t smem = kStages * kStageBytes + 1024 + 256 + 4 * 32 * 33 * sizeof(float);
  int sms = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = static_cast<int>(std::min<long long>(sms, a.tiles));
  auto kern = tf32 ? backmap_tc_kernel<true> : backmap_tc_kernel<false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("backmap: ") + cudaGetErrorString(e));
  kern<<<grid, kThreads, smem, stream>>>(mAh, mAl, mBh, mBl, a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("backmap: launch failed: ") + cudaGetErrorString(e));
  return NAJA_OK;
}

int backmap_tc_read_error(const int* err, cudaStream_t stream, const char* who) {
  int w[4] = {0, 0, 0, 0};
  cudaError_t e = cudaMemcpyAsync(w, err, sizeof(w), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string(who) + ": " + cudaGetErrorString(e));
  if (w[0] != 0)
    return fail(NAJA_ERR_DEVICE, std::string(who) + ": tensor-core pipeline gave up a bounded wait (code " +
                                     std::to_string(w[0]) + ", " + std::to_string(w[1]) + ", " + std::to_string(w[2]) +
                                     ", " + std::to_string(w[3]) + ")");
  return NAJA_OK;
}

int backmap_tc(int n, int d, long long N, const double* T, int ldt, const double* shift, const void* Y, int y_dtype,
               void* V, int v_dtype, int mode, cudaStream_t stream) {
  const size_t ybytes = backmap_tc_operand_bytes(N, d, mode), tbytes = backmap_tc_operand_bytes(n, d, mode);
  DeviceBuffer bYh, bYl, bTh, bTl, berr;
  int st;
  if ((st = bYh.alloc(ybytes, stream)) || (st = bYl.alloc(ybytes, stream)) || (st = bTh.alloc(tbytes, stream)) ||
      (st = bTl.alloc(tbytes, stream)) || (st = berr.alloc(4 * sizeof(int), stream)))
    return st;
  int* err = static_cast<int*>(berr.ptr);
  cudaError_t e = cudaMemsetAsync(err, 0, 4 * sizeof(int), stream);
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("backmap: ") + cudaGetErrorString(e));
  if ((st = backmap_tc_split_T(n, d, T, ldt, bTh.ptr, bTl.ptr, mode, stream))) return st;
  if ((st = backmap_tc_enqueue(n, d, N, Y, y_dtype, bTh.ptr, bTl.ptr, bYh.ptr, bYl.ptr, shift, V, v_dtype, mode, err,
                               stream)))
    return st;
  return backmap_tc_read_error(err, stream, "backmap");
}

// ----------------------------------------------------------------------
// Allocation-free variant (naja_backmap_noalloc).
//
// Some callers cannot allocate device memory at the point they need the
// backmap: a service that reserves its whole device-memory budget up front
// and forbids allocations in its request path, or a host framework whose
// allocator owns the device and must not see cudaMalloc/cudaFree (which may
// also synchronise the device) from a library.  For them the split operands
// live in one file-scope device array of fixed size instead of per-call
// buffers.  The array exists once per device that loads this library and is
// held until the process exits.  Its device address is looked up once per
// device (cudaGetSymbolAddress, with that device current) on the first call
// made on that device; that first call should therefore come before any
// stream capture.  After cudaDeviceReset the cached address is stale: a
// process that resets a device must not call this entry point on it again.
// Every call reuses the same array: the error words are cleared by each call,
// and calls whose work overlaps on the GPU (different streams, or different
// host threads on one device) race on the array, so the caller serialises
// them.
constexpr size_t kNoAllocScratchBytes = 64ull << 20;  // 64 MiB
constexpr int kNoAllocMaxDevices = 64;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[kNoAllocMaxDevices] = {};

int noalloc_scratch(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("naja_backmap_noalloc: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(NAJA_ERR_UNSUPPORTED, "naja_backmap_noalloc: device index too large");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(NAJA_ERR_CUDA, std::string("naja_backmap_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return NAJA_OK;
}
}  // namespace

int backmap_tc_noalloc(int n, int d, long long N, const double* T, int ldt, const double* shift, const void* Y,
                       int y_dtype, void* V, int v_dtype, int mode, cudaStream_t stream) {
  // scratch layout: [error words | Y hi | Y lo | T hi | T lo], each 1024-aligned
  const size_t ybytes = backmap_tc_operand_bytes(N, d, mode), tbytes = backmap_tc_operand_bytes(n, d, mode);
  const size_t need = 1024 + 2 * ybytes + 2 * tbytes;
  if (need > kNoAllocScratchBytes)
    return fail(NAJA_ERR_INVALID_ARGUMENT,
                "naja_backmap_noalloc: this shape needs " + std::to_string(need) + " bytes of scratch, more than the " +
                    std::to_string(kNoAllocScratchBytes) + " the library reserves; pass fewer samples per call");
  unsigned char* base = nullptr;
  int st = noalloc_scratch(&base);
  if (st) return st;
  int* err = reinterpret_cast<int*>(base);
  void* Yh = base + 1024;
  void* Yl = base + 1024 + ybytes;
  void* Th = base + 1024 + 2 * ybytes;
  void* Tl = base + 1024 + 2 * ybytes + tbytes;
  cudaError_t e = cudaMemsetAsync(err, 0, 4 * sizeof(int), stream);
  if (e != cudaSuccess) return fail(NAJA_ERR_CUDA, std::string("naja_backmap_noalloc: ") + cudaGetErrorString(e));
  if ((st = backmap_tc_split_T(n, d, T, ldt, Th, Tl, mode, stream))) return st;
  if ((st = backmap_tc_enqueue(n, d, N, Y, y_dtype, Th, Tl, Yh, Yl, shift, V, v_dtype, mode, err, stream))) return st;
  return backmap_tc_read_error(err, stream, "naja_backmap_noalloc");
}

}  // namespace naja
