"""ctypes binding of libnaja_b200.so (the C ABI in include/naja_chr.h and
include/naja_mlp.h).

There is no fallback: if the shared library is missing or a symbol is
absent, loading raises.  Build it with `python -m naja_b200.build`.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libnaja_b200.so"

NAJA_OK = 0
NAJA_ERR_INVALID_ARGUMENT = 1
NAJA_ERR_RUNTIME = 2
NAJA_ERR_CUDA = 3
NAJA_ERR_NO_MEMORY = 4
NAJA_ERR_UNSUPPORTED = 5
NAJA_ERR_DEVICE = 6

PREC_FP32 = 0
PREC_FP64 = 1
RNG_PHILOX = 0
RNG_REF_MRG = 1
DTYPE_F32 = 0
DTYPE_F64 = 1
SPARSE_AUTO = 0     # compressed columns when A is at most 1/4 nonzero and they fit
SPARSE_DENSE = 1    # every row of A every step
SPARSE_COLUMNS = 2  # only the nonzero rows of the step's column(s)
BACKMAP_FP64 = 0
BACKMAP_BF16X3 = 1
BACKMAP_TF32X3 = 2

# Every entry point include/naja_chr.h declares.
EXPORTED = (
    "naja_chr_params_default",
    "naja_polytope_create",
    "naja_polytope_destroy",
    "naja_polytope_shape",
    "naja_polytope_check",
    "naja_chr_run",
    "naja_chr_kernel_choice",
    "naja_backmap",
    "naja_backmap_noalloc",
    "naja_validate",
    "naja_last_error",
    "naja_mrg_state_bytes",
    "naja_mrg_tape",
    "naja_mrg_init_states",
    "naja_version",
    "naja_chr_run_batched",
    "naja_batch_occupancy",
    "naja_chr_capture_batched",
    "naja_graph_launch",
    "naja_graph_check",
    "naja_graph_destroy",
    "naja_chr_run_backmapped",
)

# Every entry point include/naja_mlp.h declares.
EXPORTED_MLP = (
    "naja_gemm_bf16",
    "naja_mlp_check",
    "naja_cast_bf16",
    "naja_gelu_backward",
    "naja_mse_grad",
    "naja_col_sum",
    "naja_adam",
)


class GemmEpilogue(C.Structure):
    """Mirror of `naja_gemm_epilogue`."""

    _fields_ = [
        ("bias", C.c_void_p),
        ("c_f32", C.c_void_p),
        ("ldc", C.c_int),
        ("accumulate", C.c_int),
        ("act", C.c_void_p),
        ("ld_act", C.c_int),
        ("act_t", C.c_void_p),
        ("ld_act_t", C.c_int),
        ("gelu", C.c_int),
    ]


class ChrParams(C.Structure):
    """Mirror of `naja_chr_params`."""

    _fields_ = [
        ("nspc", C.c_int),
        ("thinning", C.c_int),
        ("nchains", C.c_int),
        ("tpb", C.c_int),
        ("seed", C.c_ulonglong),
        ("pair_prob", C.c_double),
        ("resync_interval", C.c_int),
        ("ksparse_prob", C.c_double),
        ("ksparse_k", C.c_int),
        ("pair_mode", C.c_int),
        ("pair_i", C.c_void_p),
        ("pair_j", C.c_void_p),
        ("pair_c", C.c_void_p),
        ("pair_s", C.c_void_p),
        ("n_pairs", C.c_int),
        ("precision", C.c_int),
        ("rng", C.c_int),
        ("out_dtype", C.c_int),
        ("chain_base", C.c_int),
        ("out_nchains", C.c_int),
        ("step_offset", C.c_longlong),
        ("max_slots", C.c_int),
        ("rng_state", C.c_void_p),
        ("wait_cycles", C.c_void_p),
        ("cluster", C.c_int),
        ("sparse", C.c_int),
        ("slack_final", C.c_void_p),
    ]


class BatchConfig(C.Structure):
    """Mirror of `naja_batch_config`."""

    _fields_ = [("threads", C.c_int), ("slots", C.c_int), ("slack_smem", C.c_int), ("ctas_per_sm", C.c_int),
                ("sparse", C.c_int)]


class NajaError(RuntimeError):
    """A non-zero status from the C ABI, with the library's message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class InvalidArgument(NajaError, ValueError):
    """Status NAJA_ERR_INVALID_ARGUMENT (the reference's std::invalid_argument)."""


_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m naja_b200.build`")
    lib = C.CDLL(str(LIB_PATH))
    for name in EXPORTED + EXPORTED_MLP:
        if not hasattr(lib, name):
            raise ImportError(f"{LIB_PATH} does not export {name}")
    vp, i, ll, d, ull = C.c_void_p, C.c_int, C.c_longlong, C.c_double, C.c_ulonglong
    lib.naja_chr_params_default.argtypes = [C.POINTER(ChrParams)]
    lib.naja_chr_params_default.restype = None
    lib.naja_polytope_create.argtypes = [i, i, i, vp, i, vp, C.POINTER(vp)]
    lib.naja_polytope_destroy.argtypes = [vp]
    lib.naja_polytope_shape.argtypes = [vp, C.POINTER(i), C.POINTER(i)]
    lib.naja_polytope_check.argtypes = [vp]
    lib.naja_chr_run.argtypes = [vp, C.POINTER(ChrParams), vp, i, vp, vp, vp]
    lib.naja_chr_kernel_choice.argtypes = [vp, C.POINTER(ChrParams), C.POINTER(i), C.POINTER(i), C.POINTER(i),
                                           C.POINTER(C.c_size_t)]
    lib.naja_chr_kernel_choice.restype = i
    lib.naja_backmap.argtypes = [i, i, ll, vp, i, vp, vp, i, vp, i, i, vp]
    lib.naja_backmap_noalloc.argtypes = [i, i, ll, vp, i, vp, vp, i, vp, i, i, vp]
    lib.naja_validate.argtypes = [vp, ll, i, i, i, vp, vp, vp]
    lib.naja_last_error.restype = C.c_char_p
    lib.naja_last_error.argtypes = []
    lib.naja_mrg_state_bytes.restype = C.c_size_t
    lib.naja_mrg_tape.argtypes = [i, ull, i, i, ll, vp]
    lib.naja_mrg_init_states.argtypes = [i, ull, i, i, vp]
    lib.naja_version.restype = C.c_char_p
    pp = C.POINTER(C.c_void_p)
    lib.naja_chr_run_batched.argtypes = [i, pp, C.POINTER(ChrParams), pp, i, pp, vp, ull, C.POINTER(BatchConfig), vp]
    lib.naja_batch_occupancy.argtypes = [i, pp, C.POINTER(BatchConfig), C.POINTER(i)]
    lib.naja_chr_capture_batched.argtypes = [i, pp, C.POINTER(ChrParams), pp, i, pp, vp, ull, C.POINTER(BatchConfig),
                                             C.POINTER(vp)]
    lib.naja_graph_launch.argtypes = [vp, vp]
    lib.naja_graph_check.argtypes = [vp]
    lib.naja_graph_destroy.argtypes = [vp]
    lib.naja_chr_run_backmapped.argtypes = [vp, C.POINTER(ChrParams), vp, i, i, vp, i, vp, i, vp, i, vp, vp, i, vp]
    f = C.c_float
    lib.naja_gemm_bf16.argtypes = [i, i, i, vp, i, vp, i, C.POINTER(GemmEpilogue), vp]
    lib.naja_mlp_check.argtypes = [vp]
    lib.naja_cast_bf16.argtypes = [i, i, vp, i, vp, i, vp, i, vp]
    lib.naja_gelu_backward.argtypes = [i, i, vp, vp, i, vp, vp, i, vp, i, vp]
    lib.naja_mse_grad.argtypes = [i, i, vp, vp, i, vp, vp, vp, vp, i, vp, i, vp]
    lib.naja_col_sum.argtypes = [i, i, vp, i, vp, vp]
    lib.naja_adam.argtypes = [i, i, vp, vp, vp, vp, i, f, f, f, f, i, vp, i, vp, i, vp]
    for name in EXPORTED_MLP:
        getattr(lib, name).restype = C.c_int
    for name in EXPORTED:
        f = getattr(lib, name)
        if f.restype is C.c_int or name in ("naja_polytope_create", "naja_polytope_destroy", "naja_polytope_shape",
                                               "naja_polytope_check", "naja_chr_run", "naja_backmap", "naja_backmap_noalloc",
                                               "naja_validate", "naja_mrg_tape", "naja_mrg_init_states",
                                               "naja_chr_run_batched", "naja_batch_occupancy",
                                               "naja_chr_capture_batched", "naja_graph_launch", "naja_graph_check",
                                               "naja_graph_destroy", "naja_chr_run_backmapped"):
            f.restype = C.c_int
    _lib = lib
    return lib


def check(status: int) -> None:
    if status == NAJA_OK:
        return
    msg = load().naja_last_error().decode(errors="replace")
    if status == NAJA_ERR_INVALID_ARGUMENT:
        raise InvalidArgument(status, msg)
    raise NajaError(status, msg)
