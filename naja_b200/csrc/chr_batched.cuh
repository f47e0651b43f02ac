// Batched multi-model CHR: one persistent launch over many conditioned
// models with uneven row counts and their chains.
//
// The grid holds a fixed number of CTAs per SM; CTA i takes work items
// i, i + grid, ... where an item is one chain of one model.  Each item runs
// the same producer / consumer pipeline as the single-model kernel (so a
// model in a batch reproduces its standalone run bit for bit); between items
// the CTA's mbarriers are invalidated and re-initialised, which is safe
// because an item ends only after its producer has drained every bulk copy
// and every consumer has released every slot.  The shared-memory layout is
// sized for the largest model; the slack vector may live in shared memory so
// that several chains share an SM without register pressure.
#pragma once
#include "chr_kernel.cuh"

namespace naja {
namespace chr_detail {
namespace {

template <int NT, int R, bool SS>
__global__ void __launch_bounds__(NT + 32, NT >= 512 ? 2 : (NT == 256 ? 3 : 4))
    chr_batched_kernel(const __grid_constant__ ChrArgs base, const __grid_constant__ Layout L,
                       const ModelDesc* __restrict__ models, const int* __restrict__ item_model,
                       const int* __restrict__ item_chain, int nitems) {
  using Real = float;
  extern __shared__ __align__(128) unsigned char smem[];
  // The current item's arguments: shared memory rather than a local copy,
  // which the out-of-line producer call would force onto the stack.
  __shared__ ChrArgs item_args;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.full_off);
  uint64_t* empty = reinterpret_cast<uint64_t*>(smem + L.empty_off);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + L.flag_off);
  if (threadIdx.x == 0) *abort_flag = 0;
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    const int ch = item_chain[item];
    if (threadIdx.x == 0) {
      for (int s = 0; s < L.slots; ++s) {
        mbar_init(&full[s], 1);
        mbar_init(&empty[s], NT / 32);
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
    }
    __syncthreads();
    if (*abort_flag) break;  // every thread reads it after the barrier
    if (threadIdx.x >= NT) {
      if (threadIdx.x == NT) producer_entry<Real>(item_args, L, smem, ch);
    } else {
      run_consumers<Real, NT, R, kBatchV, SS, false>(item_args, L, smem, ch);
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

template <int NT, int R, bool SS>
int batch_launch_one(const ChrArgs& base, const ModelDesc* models, const int* im, const int* ic, int nitems,
                     const BatchConfig& cfg, cudaStream_t stream) {
  auto kern = chr_batched_kernel<NT, R, SS>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(cfg.smem));
  if (e != cudaSuccess) return NAJA_ERR_CUDA;
  int occ = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, NT + 32, cfg.smem);
  if (e != cudaSuccess || occ < 1) return NAJA_ERR_UNSUPPORTED;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int per_sm = cfg.ctas_per_sm > 0 ? (cfg.ctas_per_sm < occ ? cfg.ctas_per_sm : occ) : occ;
  const int grid = nitems < sms * per_sm ? nitems : sms * per_sm;
  const Layout L = make_layout(base.d, cfg.lda_max, sizeof(float), NT, cfg.slots, SS ? cfg.lda_max : 0);
  kern<<<grid, NT + 32, cfg.smem, stream>>>(base, L, models, im, ic, nitems);
  return cudaGetLastError() == cudaSuccess ? NAJA_OK : NAJA_ERR_CUDA;
}

template <int NT, int R, bool SS>
int batch_occupancy_one(const BatchConfig& cfg, int* out) {
  auto kern = chr_batched_kernel<NT, R, SS>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(cfg.smem));
  if (e != cudaSuccess) return NAJA_ERR_CUDA;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, kern, NT + 32, cfg.smem);
  return e == cudaSuccess ? NAJA_OK : NAJA_ERR_CUDA;
}

// Dispatch over the instantiated (chunks per warp, slack store) pairs of one
// thread count.
template <int NT>
int batch_dispatch(const ChrArgs* base, const ModelDesc* models, const int* im, const int* ic, int nitems,
                   const BatchConfig& cfg, cudaStream_t stream, int* occ_out) {
#define NAJA_BATCH_CASE(RR, SSV)                                                            \
  if (cfg.rows == RR && cfg.slack_smem == (SSV ? 1 : 0))                                    \
    return occ_out ? batch_occupancy_one<NT, RR, SSV>(cfg, occ_out)                         \
                   : batch_launch_one<NT, RR, SSV>(*base, models, im, ic, nitems, cfg, stream);
  // The capacities listed in batch_chunk_capacities (chr.cuh).
  if constexpr (NT == 512) {
    NAJA_BATCH_CASE(4, true)
    NAJA_BATCH_CASE(8, true)
    NAJA_BATCH_CASE(4, false)
    NAJA_BATCH_CASE(8, false)
  } else if constexpr (NT == 256) {
    NAJA_BATCH_CASE(4, true)
    NAJA_BATCH_CASE(8, true)
    NAJA_BATCH_CASE(16, true)
    NAJA_BATCH_CASE(6, false)
    NAJA_BATCH_CASE(8, false)
    NAJA_BATCH_CASE(12, false)
  } else {
    NAJA_BATCH_CASE(12, true)
    NAJA_BATCH_CASE(16, true)
    NAJA_BATCH_CASE(12, false)
    NAJA_BATCH_CASE(16, false)
  }
#undef NAJA_BATCH_CASE
  return NAJA_ERR_UNSUPPORTED;
}

}  // namespace
}  // namespace chr_detail
}  // namespace naja
