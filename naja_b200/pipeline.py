"""Sampling with the backmap and the copy to host overlapped.

`sample_backmapped` is the job of `naja sample run --backmap` as one call:
CHR samples of a polytope, mapped to reaction space (v = T y + shift) and
delivered into a host buffer.  The chains run in chunks; while the step
kernel of chunk k + 1 runs on one stream (one CTA per chain, a few SMs), the
backmap of chunk k runs on the tensor cores of the other SMs and its rows
are copied to the host on a second stream.

A chunk boundary falls on a multiple of both the resync interval and the
thinning.  There a single run recomputes the slack from x in FP64 anyway,
and a new launch starts from the previous chunk's final x (exact, FP64) and
the same Philox step counter, so every sample is bit-identical to the one
launch of naja_chr_run (src/engine/job_sampling.cu:300-385 of
quothbonney/naja samples, then backmaps, then writes).  Without a resync
interval, or with the MRG32k3a streams, the job runs as one chunk.
"""
from __future__ import annotations

import math

import numpy as np

from .sampler import Polytope, backmap

try:
    import torch
except Exception:  # pragma: no cover
    torch = None


def chunk_samples(nspc: int, thinning: int, resync_interval: int, rng: str = "philox",
                  target_steps: int = 1 << 16) -> int:
    """Samples per chunk: whole periods of lcm(resync, thinning) steps, about
    `target_steps` steps long; all of nspc when the job cannot be split."""
    if resync_interval <= 0 or rng != "philox":
        return int(nspc)
    period = math.lcm(int(resync_interval), int(thinning)) // int(thinning)
    k = max(1, int(target_steps) // (period * int(thinning)))
    return int(min(nspc, k * period))


def sample_backmapped(P: Polytope, T, shift, X0, nspc: int, thinning: int, nchains: int, out, *,
                      mode: str = "tf32x3", chunk: int | None = None, resync_interval: int = 0,
                      rng: str = "philox", **kw):
    """Runs `nchains` chains of `nspc` samples from X0 ((nchains, d) or (d,))
    and writes v = T y + shift for every sample into `out`, a (nspc * nchains,
    n) float32 host tensor (pinned for the copies to overlap), rows in the
    sample order of naja_chr_run.  Returns the final positions (nchains, d)
    on the device.  Extra keywords go to Polytope.run (seed, pair_prob,
    precision, sparse, ...)."""
    if torch is None:
        raise RuntimeError("sample_backmapped needs torch")
    if "step_offset" in kw or "out_nchains" in kw or "chain_base" in kw:
        raise ValueError("sample_backmapped runs whole jobs: no step_offset, chain_base or out_nchains")
    dev = torch.device("cuda", P.device)
    d = P.d

    def on_device(v):
        t = v if torch.is_tensor(v) else torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64))
        return t.to(device=dev, dtype=torch.float64)

    T_dev, sh_dev = on_device(T), on_device(shift)
    n = T_dev.shape[0]
    if tuple(out.shape) != (nspc * nchains, n):
        raise ValueError(f"out must be ({nspc * nchains}, {n})")
    X = torch.as_tensor(X0, dtype=torch.float64).to(dev)
    if X.dim() == 1:
        X = X.expand(nchains, d)
    X = X.contiguous().clone()
    cs = int(chunk) if chunk else chunk_samples(nspc, thinning, resync_interval, rng)
    if cs < nspc and (resync_interval <= 0 or (cs * thinning) % resync_interval or rng != "philox"):
        raise ValueError("a chunk must span whole resync intervals of a Philox run")
    rows = cs * nchains
    samples = [torch.empty((rows, d), dtype=torch.float32, device=dev) for _ in range(2)]
    V = [torch.empty((rows, n), dtype=torch.float32, device=dev) for _ in range(2)]
    xs = [X, torch.empty_like(X)]
    s_chr = torch.cuda.Stream(dev)
    s_bm = torch.cuda.Stream(dev)
    s_chr.wait_stream(torch.cuda.current_stream(dev))
    s_bm.wait_stream(torch.cuda.current_stream(dev))
    freed = [None, None]  # event: chunk k - 2's backmap and copy are done with buffer k % 2
    for k, s0 in enumerate(range(0, nspc, cs)):
        ns = min(cs, nspc - s0)
        b = k % 2
        r = ns * nchains
        with torch.cuda.stream(s_chr):
            if freed[b] is not None:
                s_chr.wait_event(freed[b])
            P.run(xs[k % 2], ns, thinning, nchains, out=samples[b][:r], X_final=xs[(k + 1) % 2],
                  step_offset=s0 * thinning, resync_interval=resync_interval, rng=rng, **kw)
            done = torch.cuda.Event()
            done.record(s_chr)
        with torch.cuda.stream(s_bm):
            s_bm.wait_event(done)
            backmap(T_dev, sh_dev, samples[b][:r], mode=mode, out=V[b][:r])
            out[s0 * nchains:s0 * nchains + r].copy_(V[b][:r], non_blocking=True)
            freed[b] = torch.cuda.Event()
            freed[b].record(s_bm)
    torch.cuda.current_stream(dev).wait_stream(s_bm)
    torch.cuda.current_stream(dev).wait_stream(s_chr)
    torch.cuda.synchronize(dev)
    P.check()
    return xs[len(range(0, nspc, cs)) % 2]
