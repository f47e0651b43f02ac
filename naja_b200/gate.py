"""Sampling until the convergence gate: split-R-hat < 1.01 and no bound
violations.

The metric is min-ESS per second at that gate: the chains of one polytope
(optionally rounded, y = M z + c) run chunk after chunk, each chunk
continuing the previous one (final x and Philox step counter carried, so the
samples are those of one long run), every chunk's samples are mapped back to
y by the FP64 backmap kernel and appended on the device, and after each
chunk the chain-correct split-R-hat of all samples so far is computed on the
device (naja_validate).  The run stops when max R-hat over dimensions drops
below the target and the samples satisfy A y <= b + 1e-6 max(1, |b|), or
when the time budget is spent; the R-hat curve is returned either way.

Timing (CUDA events, plus the host time of computing the rounding): the
rounding, every chunk's sampling and back-map, and the R-hat checks -- the
whole cost of reaching the gate.  ESS (Geyer, chains de-interleaved, summed
over chains, minimum over dimensions; src/validate/mcmc.cpp:60-76 of
quothbonney/naja) is computed once at the end; series longer than the
validate kernel's on-chip limit are thinned by the smallest factor that fits,
which can only lower the estimate.  R-hat follows mcmc.cpp:126-194.
"""
from __future__ import annotations

import time

import numpy as np

from . import rounding as rnd
from .sampler import Polytope, backmap
from .validate import ess_rhat

ESS_MAX_SERIES = 48 * 1024


def make_rounding(method, A, b, start):
    """Rounding for `method`: "none", "dikin" (the reference's preconditioner)
    or "dikin_full" (whole Dikin ellipsoid); a Rounding passes through."""
    if isinstance(method, rnd.Rounding):
        return method
    if method in (None, "none", "plain"):
        return rnd.identity(A, b, start)
    if method == "dikin":
        return rnd.dikin(A, b, start)
    if method == "dikin_full":
        return rnd.dikin_full(A, b, start)
    raise ValueError(f"unknown rounding {method!r}")


def sample_to_gate(A, b, start, *, method="dikin_full", nchains=16, thinning=116, chunk_nspc=12500,
                   pair_prob=0.3, resync_interval=2048, precision="fp32", seed=0, budget_s=60.0,
                   rhat_target=1.01, max_chunks=64, device=0, check_bounds=True, keep_samples=False,
                   adapt_after=0):
    """Runs chunks of `chunk_nspc` samples per chain until the gate or the
    budget (seconds, counted as described in the module docstring).

    adapt_after > 0: after that many chunks (a warm-up), the rounding is
    replaced once by the isotropic position of the samples so far (y = Sigma^
    1/2 z + mean, from their covariance), the chains continue from their
    current positions in the new coordinates, and only the samples after it
    count for the gate and the ESS; the warm-up's time counts."""
    import torch

    dev = torch.device("cuda", device)
    A = np.asarray(A, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = A.shape[1]
    t_host = time.perf_counter()
    R = make_rounding(method, A, b, np.asarray(start, dtype=np.float64))
    rounding_s = time.perf_counter() - t_host
    label = R.info.get("method") + ("+covariance" if adapt_after else "")
    t_host = time.perf_counter()
    P = Polytope(R.A, R.b, device=device)
    identity = R.info.get("method") == "identity" and not np.any(R.c)  # then y = z
    M = torch.from_numpy(np.ascontiguousarray(R.M)).to(dev)
    c = torch.from_numpy(R.c).to(dev)
    Z = torch.from_numpy(np.broadcast_to(R.z0, (nchains, d)).copy()).to(dev)
    Zf = torch.empty_like(Z)
    rows = chunk_nspc * nchains
    Y = torch.empty((max_chunks * rows, d), dtype=torch.float32, device=dev)
    zbuf = torch.empty((rows, d), dtype=torch.float32, device=dev)
    setup_s = time.perf_counter() - t_host
    kw = dict(seed=seed, pair_prob=pair_prob, resync_interval=resync_interval, precision=precision)
    curve = []
    dev_ms = 0.0
    reached = False
    k = 0
    k0 = 0  # first chunk that counts (after an adaptation)
    viol = 0
    while k < max_chunks:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        dst = Y[k * rows:(k + 1) * rows]
        P.run(Z, chunk_nspc, thinning, nchains, out=(dst if identity else zbuf), X_final=Zf,
              step_offset=k * chunk_nspc * thinning, **kw)
        if not identity:
            backmap(M, c, zbuf, mode="fp64", out=dst)  # y = M z + c, FP64 products
        if k + 1 - k0 >= 2:
            _, rh = ess_rhat(Y[k0 * rows:(k + 1) * rows], nchains, layout=1, ess=False)
        else:
            rh = np.full(d, np.inf)
        e1.record()
        torch.cuda.synchronize()
        Z, Zf = Zf, Z
        k += 1
        dev_ms += e0.elapsed_time(e1)
        if adapt_after and k == adapt_after:
            t_host = time.perf_counter()
            Yw = Y[:k * rows].double()
            mean = Yw.mean(dim=0)
            cov = torch.cov(Yw.T)
            y_now = Z @ M.T + c  # current positions in y (FP64)
            R = rnd.from_covariance(A, b, cov.cpu().numpy(), mean.cpu().numpy(), y_now.cpu().numpy())
            P.close()
            P = Polytope(R.A, R.b, device=device)
            M = torch.from_numpy(np.ascontiguousarray(R.M)).to(dev)
            c = torch.from_numpy(R.c).to(dev)
            Z = torch.from_numpy(R.z0).to(dev).contiguous()
            identity = False
            k0 = k
            del Yw
            torch.cuda.synchronize()
            rounding_s += time.perf_counter() - t_host
        elapsed = rounding_s + setup_s + dev_ms / 1e3
        rmax = float(rh.max())
        curve.append({"seconds": elapsed, "steps_per_chain": k * chunk_nspc * thinning, "rhat_max": rmax,
                      "rhat_median": float(np.median(rh))})
        if rmax < rhat_target:
            if check_bounds:
                viol = _violations(torch, A, b, Y[k0 * rows:k * rows])
            if viol == 0:
                reached = True
                break
        if elapsed >= budget_s:
            break
    P.check()
    Yk = Y[k0 * rows:k * rows]
    spc = (k - k0) * chunk_nspc
    stride = -(-spc // ESS_MAX_SERIES)
    Ye = Yk.view(spc, nchains, d)[::stride].reshape(-1, d) if stride > 1 else Yk
    ess, rh = ess_rhat(Ye, nchains, layout=1)
    if check_bounds and not reached:
        viol = _violations(torch, A, b, Yk)
    per_dim = ess.sum(axis=1)
    total_s = curve[-1]["seconds"]
    out = {"method": label, "reached": reached, "seconds": total_s, "rounding_seconds": rounding_s,
           "chunks": k, "warmup_chunks": k0, "steps_per_chain": k * chunk_nspc * thinning,
           "samples_per_chain": spc,
           "rhat_max": curve[-1]["rhat_max"], "bounds_violations": int(viol), "min_ess": float(per_dim.min()),
           "min_ess_per_s": float(per_dim.min()) / total_s, "ess_thinning": int(stride), "curve": curve}
    if keep_samples:
        out["samples"] = Yk
    P.close()
    return out


def _violations(torch, A, b, Y):
    At = torch.from_numpy(A).to(Y.device)
    bt = torch.from_numpy(b).to(Y.device)
    tol = 1e-6 * torch.clamp(bt.abs(), min=1.0)
    v = 0
    for s0 in range(0, Y.shape[0], 50000):
        v += int(((Y[s0:s0 + 50000].double() @ At.T - bt) > tol).sum())
    return v
