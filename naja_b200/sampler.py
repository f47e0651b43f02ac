"""Python mirror of the reference's GPU sampler API over the C ABI.

`Polytope` uploads A y <= b once (naja_polytope_create) and runs chains
on it (naja_chr_run); `coordinate_hit_and_run` is the one-shot call with the
argument list of naja::gpu::CoordinateHitAndRun (src/gpu/gpusamplers.h:30-46
of quothbonney/naja).  Arrays may be numpy (host) or torch tensors (host or
CUDA); host buffers are staged by the library, CUDA tensors are used in
place on the current torch stream.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import ChrParams, check, load

try:  # torch is optional for host-only callers
    import torch
except Exception:  # pragma: no cover - torch is present in this image
    torch = None

_PREC = {"fp32": _lib.PREC_FP32, "fp64": _lib.PREC_FP64}
_RNG = {"philox": _lib.RNG_PHILOX, "mrg": _lib.RNG_REF_MRG, "ref_mrg": _lib.RNG_REF_MRG}
_SPARSE = {"auto": _lib.SPARSE_AUTO, "dense": _lib.SPARSE_DENSE, "columns": _lib.SPARSE_COLUMNS}
_BACKMAP = {"fp64": _lib.BACKMAP_FP64, "bf16x3": _lib.BACKMAP_BF16X3, "tf32x3": _lib.BACKMAP_TF32X3}


def _is_torch(x) -> bool:
    return torch is not None and isinstance(x, torch.Tensor)


def _ptr(x):
    """Raw pointer of a numpy array / torch tensor (None -> NULL)."""
    if x is None:
        return None
    if _is_torch(x):
        return C.c_void_p(x.data_ptr())
    return C.c_void_p(x.ctypes.data)


def _stream_of(*arrays):
    for a in arrays:
        if _is_torch(a) and a.is_cuda:
            return C.c_void_p(torch.cuda.current_stream(a.device).cuda_stream)
    return None


def _f64_colmajor(A) -> np.ndarray:
    return np.asfortranarray(np.asarray(A, dtype=np.float64))


@dataclass
class Tier:
    """Arithmetic and RNG tier of a run."""

    precision: str = "fp32"
    rng: str = "philox"


class Polytope:
    """Device-resident polytope {y : A y <= b} (FP64 and FP32 copies of A)."""

    def __init__(self, A, b, device: int = 0):
        lib = load()
        self.device = device
        if _is_torch(A) and A.is_cuda:
            At = A.to(torch.float64).t().contiguous()  # column-major A == row-major A^T
            m, d = A.shape
            self._keep = (At,)
            ap, lda = C.c_void_p(At.data_ptr()), m
        else:
            An = _f64_colmajor(A)
            m, d = An.shape
            self._keep = (An,)
            ap, lda = _ptr(An), m
        if _is_torch(b):
            bb = b.to(torch.float64).contiguous()
        else:
            bb = np.ascontiguousarray(np.asarray(b, dtype=np.float64).reshape(-1))
        if bb.shape[0] != m:
            raise _lib.InvalidArgument(1, f"dimension mismatch: rhs vector size ({bb.shape[0]}) != rows ({m})")
        self.m, self.d = int(m), int(d)
        h = C.c_void_p()
        check(lib.naja_polytope_create(device, self.m, self.d, ap, lda, _ptr(bb), C.byref(h)))
        self._h = h
        self._keep = None

    def close(self):
        if getattr(self, "_h", None):
            load().naja_polytope_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self):
        """Synchronises the device and raises a device-side error word."""
        check(load().naja_polytope_check(self._h))

    def params(self, nspc, thinning, nchains, *, tpb=-1, seed=0, pair_prob=0.0, resync_interval=0,
               ksparse_prob=0.0, ksparse_k=8, pair_mode=1, pairs=None, precision="fp32", rng="philox",
               out_dtype="f32", chain_base=0, out_nchains=0, step_offset=0, max_slots=0, rng_state=None,
               wait_cycles=None, cluster=0, sparse="auto", slack_final=None):
        p = ChrParams()
        load().naja_chr_params_default(C.byref(p))
        p.nspc, p.thinning, p.nchains, p.tpb = int(nspc), int(thinning), int(nchains), int(tpb)
        p.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        p.pair_prob, p.resync_interval = float(pair_prob), int(resync_interval)
        p.ksparse_prob, p.ksparse_k, p.pair_mode = float(ksparse_prob), int(ksparse_k), int(pair_mode)
        keep = []
        if pairs is not None:
            pi, pj, pc, ps = pairs
            arrs = []
            for a, dt in ((pi, np.int32), (pj, np.int32), (pc, np.float64), (ps, np.float64)):
                if _is_torch(a):
                    arrs.append(a.to({np.int32: torch.int32, np.float64: torch.float64}[dt]).contiguous())
                else:
                    arrs.append(np.ascontiguousarray(np.asarray(a, dtype=dt)))
            keep += arrs
            p.pair_i, p.pair_j, p.pair_c, p.pair_s = [(_ptr(a).value) for a in arrs]
            p.n_pairs = int(len(arrs[0]))
        p.precision = _PREC[precision]
        p.rng = _RNG[rng]
        p.out_dtype = _lib.DTYPE_F64 if out_dtype in ("f64", "float64", np.float64) else _lib.DTYPE_F32
        p.chain_base, p.out_nchains, p.step_offset = int(chain_base), int(out_nchains), int(step_offset)
        p.max_slots = int(max_slots)
        if rng_state is not None:
            p.rng_state = _ptr(rng_state).value
        if wait_cycles is not None:
            p.wait_cycles = _ptr(wait_cycles).value
        p.cluster = int(cluster)
        p.sparse = _SPARSE[sparse]
        if slack_final is not None:
            p.slack_final = _ptr(slack_final).value
        return p, keep

    def kernel_choice(self, nspc, thinning, nchains, **kw):
        """The step kernel a run with these arguments launches:
        dict(kernel="columns" | "dense", threads, slots, smem)."""
        p, keep = self.params(nspc, thinning, nchains, **kw)
        sk, th, sl, sm = C.c_int(), C.c_int(), C.c_int(), C.c_size_t()
        check(load().naja_chr_kernel_choice(self._h, C.byref(p), C.byref(sk), C.byref(th), C.byref(sl), C.byref(sm)))
        del keep
        return {"kernel": "columns" if sk.value else "dense", "threads": th.value, "slots": sl.value,
                "smem": sm.value}

    def run(self, X0, nspc, thinning, nchains=None, *, out=None, X_final=None, stream=None, **kw):
        """Runs the chains; returns the (nspc*out_nchains, d) sample matrix.

        X0: (nchains, d) start points (row = chain, the bytes of the
        reference's d x nchains X matrix) or one (d,) point for all chains.
        """
        lib = load()
        if _is_torch(X0):
            X = X0.to(torch.float64)
            if X.dim() == 1:
                X = X.expand(int(nchains), -1)
            X = X.contiguous()
        else:
            X = np.asarray(X0, dtype=np.float64)
            if X.ndim == 1:
                X = np.broadcast_to(X, (int(nchains), X.shape[0]))
            X = np.ascontiguousarray(X)
        nchains = int(X.shape[0]) if nchains is None else int(nchains)
        if X.shape[1] != self.d:
            raise _lib.InvalidArgument(1, f"dimension mismatch: start point size ({X.shape[1]}) != cols ({self.d})")
        p, keep = self.params(nspc, thinning, nchains, **kw)
        rows = int(nspc) * (p.out_nchains or nchains)
        if out is None:
            dt = np.float64 if p.out_dtype == _lib.DTYPE_F64 else np.float32
            out = np.empty((rows, self.d), dtype=dt)
        if stream is None:
            stream = _stream_of(out, X, X_final)
        check(lib.naja_chr_run(self._h, C.byref(p), _ptr(X), self.d, _ptr(out), _ptr(X_final), stream))
        del keep
        return out


def coordinate_hit_and_run(A, b, X, nspc, thinning, nchains, tpb_ss=-1, seed=0, pair_prob=0.0,
                           resync_interval=0, ksparse_prob=0.0, ksparse_k=8, pair_mode=1, pair_i=None,
                           pair_j=None, pair_c=None, pair_s=None, **tier):
    """One-shot sampler with naja::gpu::CoordinateHitAndRun's arguments.

    X is the reference's d x nchains start matrix (numpy (d, nchains)).
    Returns the (nchains*nspc, d) sample matrix (the reference's
    d x (nchains*nspc) column-major result, byte for byte).
    """
    P = Polytope(A, b)
    try:
        X0 = np.asarray(X, dtype=np.float64)
        X0 = X0.T if X0.ndim == 2 else X0
        pairs = None if pair_i is None else (pair_i, pair_j, pair_c, pair_s)
        return P.run(X0, nspc, thinning, nchains, tpb=tpb_ss, seed=seed, pair_prob=pair_prob,
                     resync_interval=resync_interval, ksparse_prob=ksparse_prob, ksparse_k=ksparse_k,
                     pair_mode=pair_mode, pairs=pairs, **tier)
    finally:
        P.close()


CoordinateHitAndRun = coordinate_hit_and_run


def backmap(T, shift, Y, mode="bf16x3", out=None, out_dtype=np.float32, stream=None):
    """V = T Y + shift for the (N, d) sample matrix Y; returns (N, n)."""
    lib = load()
    Tn = T if (_is_torch(T) and T.is_cuda) else _f64_colmajor(T)
    if _is_torch(Tn):
        Tc = Tn.to(torch.float64).t().contiguous()
        n, d = T.shape
        tp = C.c_void_p(Tc.data_ptr())
    else:
        n, d = Tn.shape
        Tc = Tn
        tp = _ptr(Tn)
    sh = shift.to(torch.float64).contiguous() if _is_torch(shift) else np.ascontiguousarray(
        np.asarray(shift, dtype=np.float64).reshape(-1))
    N = int(Y.shape[0])
    if int(Y.shape[1]) != d:
        raise _lib.InvalidArgument(1, "backmap_into: transformation shape mismatch with samples")
    ydt = _lib.DTYPE_F64 if str(Y.dtype) in ("float64", "torch.float64") else _lib.DTYPE_F32
    if out is None:
        out = np.empty((N, n), dtype=out_dtype)
    vdt = _lib.DTYPE_F64 if str(out.dtype) in ("float64", "torch.float64") else _lib.DTYPE_F32
    if stream is None:
        stream = _stream_of(out, Y)
    check(lib.naja_backmap(int(n), int(d), N, tp, int(n), _ptr(sh), _ptr(Y), ydt, _ptr(out), vdt,
                           _BACKMAP[mode], stream))
    del Tc
    return out


def mrg_tape(seed, nchains, count, chain_base=0, device=0):
    """cuRAND MRG32k3a uniforms of curand_init(seed, chain, 0) streams (test hook)."""
    tape = np.empty((nchains, count), dtype=np.float64)
    check(load().naja_mrg_tape(device, int(seed) & 0xFFFFFFFFFFFFFFFF, int(chain_base), int(nchains), int(count),
                               _ptr(tape)))
    return tape
