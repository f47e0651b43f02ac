// One (element type, consumer thread count) slice of the CHR step kernel's
// instantiations, compiled as its own translation unit so that the build
// runs in parallel.  NAJA_CHR_REAL and NAJA_CHR_NT are set by the build.
#include "chr_kernel.cuh"

#ifndef NAJA_CHR_REAL
#error "NAJA_CHR_REAL must be defined"
#endif
#define NAJA_CAT3_(a, b, c) a##_##b##_##c
#define NAJA_CAT3(a, b, c) NAJA_CAT3_(a, b, c)

namespace naja {
int NAJA_CAT3(chr_launch, NAJA_CHR_REAL, NAJA_CHR_NT)(const ChrArgs& a, int nchains, const ChrLaunchConfig& cfg,
                                                    cudaStream_t stream) {
  return chr_detail::launch_rows<NAJA_CHR_REAL, NAJA_CHR_NT>(a, nchains, cfg, stream);
}
}  // namespace naja
