"""Autotuner for the batched kernel's launch shape.

Candidates are (consumer threads, ring depth, slack store, resident chains
per SM); the occupancy calculator drops shapes that do not fit, and each
remaining shape is timed with CUDA events on a short run of the actual batch
(same models, chains and step settings, fewer samples).  The fastest shape
per (models' max rows, d, chains) is cached for the process.
"""
from __future__ import annotations

import itertools

from ._lib import NajaError
from .batch import Batch, Shape

_cache: dict = {}

THREADS = (128, 256, 512)
SLOTS = (0, 2, 3, 4)
CTAS = (0, 1, 2, 3, 4)


SPARSE_THREADS = (64, 128, 256)
SPARSE_SLOTS = (3, 4, 8)


def _shapes():
    for t, s, ss, c in itertools.product(THREADS, SLOTS, (1, 0), CTAS):
        yield Shape(t, s, ss, c)
    for t, s, c in itertools.product(SPARSE_THREADS, SPARSE_SLOTS, CTAS):
        yield Shape(t, s, 1, c, sparse=1)


def candidates(batch: Batch):
    seen = set()
    for shape in _shapes():
        t, s, ss, c = shape.threads, shape.slots, shape.slack_smem, shape.ctas_per_sm
        try:
            occ = batch.occupancy(shape)
        except NajaError:  # no instantiated capacity holds these models
            continue
        if occ == 0:
            continue
        eff = (t, s, ss, min(c, occ) if c else occ, shape.sparse)
        if eff in seen:
            continue
        seen.add(eff)
        yield shape


def tune(batch: Batch, X0s, outs, nchains, thinning, *, probe_nspc=16, reps=2, verbose=False, **kw):
    """Returns (best Shape, {shape: chain-steps per second})."""
    import torch

    key = (max(p.m for p in batch.models), batch.d, len(batch.models), nchains, thinning,
           tuple(sorted(kw.items())))
    if key in _cache:
        return _cache[key]
    results = {}
    steps = len(batch.models) * nchains * probe_nspc * thinning
    for shape in candidates(batch):
        batch.run(X0s, outs, probe_nspc, thinning, nchains, shape=shape, **kw)  # warm
        torch.cuda.synchronize()
        best = None
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            batch.run(X0s, outs, probe_nspc, thinning, nchains, shape=shape, **kw)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        results[shape] = steps / (best / 1e3)
        if verbose:
            print(shape, f"{results[shape] / 1e6:.1f} M steps/s", flush=True)
    batch.check()
    best_shape = max(results, key=results.get)
    _cache[key] = (best_shape, results)
    return best_shape, results
