// Split-precision tensor-core backmap (tcgen05).  Placeholder entry point
// until the tcgen05 GEMM lands: reports UNSUPPORTED rather than computing
// anything on another path.
#include <cuda_runtime.h>

#include "../../include/naja_chr.h"
#include "capi_internal.cuh"

namespace naja {

int backmap_tc(int, int, long long, const double*, int, const double*, const void*, int, void*, int, int,
               cudaStream_t) {
  return fail(NAJA_ERR_UNSUPPORTED, "backmap: tensor-core modes are not built yet");
}

}  // namespace naja
