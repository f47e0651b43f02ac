"""B200-native coordinate hit-and-run sampler (drop-in for quothbonney/naja's
GPU CHR path).  The compute lives in libnaja_b200.so (sm_100a CUDA behind
the C ABI of include/naja_chr.h); this package is its Python mirror."""
from ._lib import InvalidArgument, NajaError, load  # noqa: F401
from .sampler import Polytope, backmap, coordinate_hit_and_run, CoordinateHitAndRun, mrg_tape  # noqa: F401

__all__ = ["Polytope", "backmap", "coordinate_hit_and_run", "CoordinateHitAndRun", "mrg_tape", "load",
           "NajaError", "InvalidArgument"]
