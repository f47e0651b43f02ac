// One consumer-thread-count slice of the batched CHR kernel's instantiations
// (NAJA_CHR_NT is set by the build).
#include "chr_batched.cuh"

#define NAJA_CAT2_(a, b) a##_##b
#define NAJA_CAT2(a, b) NAJA_CAT2_(a, b)

namespace naja {
int NAJA_CAT2(chr_batch_dispatch, NAJA_CHR_NT)(const ChrArgs* base, const ModelDesc* models, const int* im,
                                              const int* ic, int nitems, const BatchConfig& cfg, cudaStream_t stream,
                                              int* occ_out) {
  return chr_detail::batch_dispatch<NAJA_CHR_NT>(base, models, im, ic, nitems, cfg, stream, occ_out);
}
}  // namespace naja
