"""Sampling with the backmap and the copy to host overlapped.

`sample_backmapped` is the job of `naja sample run --backmap` as one call
(naja_chr_run_backmapped in the C ABI): CHR samples of a polytope, mapped to
reaction space (v = T y + shift) and delivered into a host buffer.  The
chains run in chunks; while the step kernel of chunk k + 1 runs on one
stream (one CTA per chain, a few SMs), the backmap of chunk k runs on the
tensor cores of the other SMs and its rows are copied to the host on a
second stream.  The library queues chunk k + 1 before chunk k's backmap, so
the step kernel never waits for the host.

A chunk boundary falls on a multiple of both the resync interval and the
thinning.  There a single run recomputes the slack from x in FP64 anyway,
and a new launch starts from the previous chunk's final x (exact, FP64) and
the same Philox step counter, so every sample is bit-identical to the one
launch of naja_chr_run (src/engine/job_sampling.cu:300-385 of
quothbonney/naja samples, then backmaps, then writes).  Without a resync
interval, or with the MRG32k3a streams, the job runs as one chunk.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import check, load
from .sampler import _BACKMAP, Polytope, _is_torch, _ptr

try:
    import torch
except Exception:  # pragma: no cover
    torch = None


def chunk_samples(nspc: int, thinning: int, resync_interval: int, rng: str = "philox",
                  target_steps: int = 1 << 16) -> int:
    """Samples per chunk the library picks: whole periods of lcm(resync,
    thinning) steps, about `target_steps` steps long; all of nspc when the
    job cannot be split."""
    if resync_interval <= 0 or rng != "philox":
        return int(nspc)
    period = math.lcm(int(resync_interval), int(thinning)) // int(thinning)
    k = max(1, int(target_steps) // (period * int(thinning)))
    return int(min(nspc, k * period))


def sample_backmapped(P: Polytope, T, shift, X0, nspc: int, thinning: int, nchains: int, out, *,
                      mode: str = "tf32x3", chunk: int | None = None, resync_interval: int = 0,
                      rng: str = "philox", samples=None, stream=None, **kw):
    """Runs `nchains` chains of `nspc` samples from X0 ((nchains, d) or (d,))
    and writes v = T y + shift for every sample into `out`, a (nspc * nchains,
    n) float32 or float64 array or tensor (pinned host memory for the copies
    to overlap), rows in the sample order of naja_chr_run.  `samples`
    (optional, (nspc * nchains, d)) also receives the samples.  Returns the
    final positions (nchains, d) as float64 (a CUDA tensor when torch is
    present).  Extra keywords go to Polytope.params (seed, pair_prob,
    precision, sparse, out_dtype, ...)."""
    if "out_nchains" in kw or "chain_base" in kw:
        raise ValueError("sample_backmapped runs whole jobs: no chain_base or out_nchains")
    d = P.d
    Tn = T if (_is_torch(T) and T.is_cuda) else np.asfortranarray(np.asarray(T, dtype=np.float64))
    n, dT = int(T.shape[0]), int(T.shape[1])
    if dT != d:
        raise _lib.InvalidArgument(1, "backmap_into: transformation shape mismatch with samples")
    # column-major T: a Fortran-ordered array, or for a CUDA tensor the row-major T^T
    Tc = Tn.to(torch.float64).t().contiguous() if _is_torch(Tn) else Tn
    sh = shift.to(torch.float64).contiguous() if _is_torch(shift) else np.ascontiguousarray(
        np.asarray(shift, dtype=np.float64).reshape(-1))
    if tuple(out.shape) != (nspc * nchains, n):
        raise ValueError(f"out must be ({nspc * nchains}, {n})")
    vdt = _lib.DTYPE_F64 if str(out.dtype) in ("float64", "torch.float64") else _lib.DTYPE_F32
    if _is_torch(X0):
        X = X0.to(torch.float64)
        if X.dim() == 1:
            X = X.expand(nchains, d)
        X = X.contiguous()
    else:
        X = np.asarray(X0, dtype=np.float64)
        if X.ndim == 1:
            X = np.broadcast_to(X, (nchains, d))
        X = np.ascontiguousarray(X)
    if torch is not None:
        dev = torch.device("cuda", P.device)
        Xf = torch.empty((nchains, d), dtype=torch.float64, device=dev)
        if stream is None:
            stream = torch.cuda.current_stream(dev).cuda_stream
    else:
        Xf = np.empty((nchains, d), dtype=np.float64)
    p, keep = P.params(nspc, thinning, nchains, resync_interval=resync_interval, rng=rng, **kw)
    check(load().naja_chr_run_backmapped(P._h, C.byref(p), _ptr(X), d, n, _ptr(Tc), n, _ptr(sh), _BACKMAP[mode],
                                         _ptr(out), vdt, _ptr(samples), _ptr(Xf), int(chunk or 0),
                                         None if stream is None else C.c_void_p(int(stream))))
    del keep
    return Xf
