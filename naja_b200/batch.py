"""Batched multi-model sampling: many polytopes of the same dimension and
their chains in one persistent launch (naja_chr_run_batched), optionally
captured once into a CUDA graph and replayed.

The reference runs such model sets one model at a time, one small launch
each (src/engine/job_bulk.cpp:115-189).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import _lib
from ._lib import BatchConfig, check, load
from .sampler import Polytope, _ptr

try:
    import torch
except Exception:  # pragma: no cover
    torch = None


@dataclass(frozen=True)
class Shape:
    """Launch shape of a batched run (see naja_batch_config)."""

    threads: int = 256
    slots: int = 3
    slack_smem: int = 1
    ctas_per_sm: int = 0
    sparse: int = 0  # 1: compressed-column kernel (threads 64 / 128 / 256)

    def c(self) -> BatchConfig:
        return BatchConfig(self.threads, self.slots, self.slack_smem, self.ctas_per_sm, self.sparse)


class Batch:
    """A set of device-resident polytopes sharing the dimension d."""

    def __init__(self, polytopes: list[Polytope]):
        if not polytopes:
            raise _lib.InvalidArgument(1, "empty batch")
        self.models = list(polytopes)
        self.d = polytopes[0].d
        self._arr = (C.c_void_p * len(self.models))(*[p._h.value for p in self.models])

    def occupancy(self, shape: Shape) -> int:
        out = C.c_int(0)
        cfg = shape.c()
        check(load().naja_batch_occupancy(len(self.models), self._arr, C.byref(cfg), C.byref(out)))
        return int(out.value)

    def _args(self, X0s, outs, nspc, thinning, nchains, kw, X_finals=None):
        p, keep = self.models[0].params(nspc, thinning, nchains, **kw)
        X = (C.c_void_p * len(self.models))(*[x.data_ptr() for x in X0s])
        O = (C.c_void_p * len(self.models))(*[o.data_ptr() for o in outs])
        F = None
        if X_finals is not None:
            F = (C.c_void_p * len(self.models))(*[(f.data_ptr() if f is not None else None) for f in X_finals])
        return p, keep, X, O, F

    def run(self, X0s, outs, nspc, thinning, nchains, shape: Shape = Shape(), seed_stride=1, stream=None,
            X_finals=None, **kw):
        """X0s[k]: (nchains, d) float64 CUDA tensor; outs[k]: (nspc*nchains, d) CUDA tensor;
        X_finals[k] (optional): (nchains, d) float64 CUDA tensor receiving model k's last states."""
        p, keep, X, O, F = self._args(X0s, outs, nspc, thinning, nchains, kw, X_finals)
        cfg = shape.c()
        if stream is None:
            stream = C.c_void_p(torch.cuda.current_stream(outs[0].device).cuda_stream)
        check(load().naja_chr_run_batched(len(self.models), self._arr, C.byref(p), X, self.d, O, F, int(seed_stride),
                                          C.byref(cfg), stream))
        del keep

    def capture(self, X0s, outs, nspc, thinning, nchains, shape: Shape = Shape(), seed_stride=1, X_finals=None,
                **kw) -> "Graph":
        p, keep, X, O, F = self._args(X0s, outs, nspc, thinning, nchains, kw, X_finals)
        cfg = shape.c()
        h = C.c_void_p()
        check(load().naja_chr_capture_batched(len(self.models), self._arr, C.byref(p), X, self.d, O, F,
                                              int(seed_stride), C.byref(cfg), C.byref(h)))
        del keep
        return Graph(h)

    def check(self):
        self.models[0].check()


class Graph:
    """A captured batched launch."""

    def __init__(self, handle):
        self._h = handle

    def launch(self, stream=None):
        if stream is None:
            stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        check(load().naja_graph_launch(self._h, stream))

    def check(self):
        check(load().naja_graph_check(self._h))

    def close(self):
        if self._h:
            load().naja_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
