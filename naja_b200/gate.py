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


def make_rounding(method, A, b, start, device=None):
    """Rounding for `method`: "none", "dikin" (the reference's preconditioner)
    or "dikin_full" (whole Dikin ellipsoid; on the GPU when `device` is
    given); a Rounding passes through."""
    if isinstance(method, rnd.Rounding):
        return method
    if method in (None, "none", "plain"):
        return rnd.identity(A, b, start)
    if method == "dikin":
        return rnd.dikin(A, b, start)
    if method == "dikin_full":
        return rnd.dikin_full(A, b, start, device=device)
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


def batch_to_gate(models, roundings, *, nchains=8, thinning=116, chunk_nspc=1000, pair_prob=0.3,
                  resync_interval=2048, seed=0, budget_s=60.0, rhat_target=1.01, device=0, max_bytes=40 << 30,
                  shape=None, extra_seconds=0.0):
    """Many polytopes (models[k] = (A, b)) sampled together in one batched
    launch per chunk (naja_chr_run_batched, chains continued through
    X_finals and the step offset), each on its rounding (roundings[k], y = M z
    + c), until every model's split-R-hat < rhat_target with no bound
    violations, or the budget.  A model's seconds are the batch's seconds
    divided by the number of models (plus `extra_seconds`, e.g. the time of
    computing its rounding).  Returns per-model min-ESS, R-hat, whether it
    passed, and the aggregate figures."""
    import torch

    from .batch import Batch, Shape

    dev = torch.device("cuda", device)
    nm = len(models)
    d = np.asarray(models[0][0]).shape[1]
    polys = [Polytope(R.A, R.b, device=device) for R in roundings]
    dense = any(R.info.get("method") != "identity" for R in roundings)
    if shape is None:
        # up to one chain per SM: the single-model shape (512 threads, slack in
        # registers); more chains share SMs with slack in shared memory
        few = nm * nchains <= _sm_count(torch, dev)
        if dense:
            shape = Shape(512, 3, 0, 1, 0) if few else Shape(256, 3, 1, 0, 0)
        else:
            shape = Shape(256, 8, 1, 1, 1) if few else Shape(128, 3, 1, 0, 1)
    B = Batch(polys)
    rows = chunk_nspc * nchains
    per_chunk = nm * rows * d * 4
    max_chunks = max(2, int(max_bytes // per_chunk))
    Ys = [torch.empty((max_chunks * rows, d), dtype=torch.float32, device=dev) for _ in range(nm)]
    Zs = [torch.empty((rows, d), dtype=torch.float32, device=dev) for _ in range(nm)]
    X = [torch.from_numpy(np.broadcast_to(R.z0, (nchains, d)).copy()).to(dev) for R in roundings]
    Xf = [torch.empty_like(x) for x in X]
    Ms = [torch.from_numpy(np.ascontiguousarray(R.M)).to(dev) for R in roundings]
    cs = [torch.from_numpy(R.c).to(dev) for R in roundings]
    passed = np.zeros(nm, dtype=bool)
    rh_last = np.full(nm, np.inf)
    dev_ms = 0.0
    k = 0
    curve = []
    while k < max_chunks:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        B.run(X, Zs, chunk_nspc, thinning, nchains, shape=shape, seed_stride=1, X_finals=Xf, seed=seed,
              pair_prob=pair_prob, resync_interval=resync_interval, step_offset=k * chunk_nspc * thinning)
        for j in range(nm):
            backmap(Ms[j], cs[j], Zs[j], mode="fp64", out=Ys[j][k * rows:(k + 1) * rows])
        k += 1
        if k >= 2:
            for j in range(nm):
                _, rh = ess_rhat(Ys[j][:k * rows], nchains, layout=1, ess=False)
                rh_last[j] = float(rh.max())
        e1.record()
        torch.cuda.synchronize()
        X, Xf = Xf, X
        dev_ms += e0.elapsed_time(e1)
        passed = rh_last < rhat_target
        curve.append([round(dev_ms / 1e3, 2), round(float(rh_last.max()), 4), int(passed.sum())])
        if passed.all() or dev_ms / 1e3 >= budget_s:
            break
    B.check()
    spc = k * chunk_nspc
    stride = -(-spc // ESS_MAX_SERIES)
    out_models = []
    for j, (A, b) in enumerate(models):
        Yk = Ys[j][:k * rows]
        Ye = Yk.view(spc, nchains, d)[::stride].reshape(-1, d) if stride > 1 else Yk
        ess, rh = ess_rhat(Ye, nchains, layout=1)
        viol = _violations(torch, np.asarray(A, dtype=np.float64), np.asarray(b, dtype=np.float64), Yk)
        out_models.append({"min_ess": float(ess.sum(axis=1).min()), "rhat_max": float(rh_last[j]),
                           "passed": bool(rh_last[j] < rhat_target and viol == 0), "bounds_violations": int(viol)})
    for p in polys:
        p.close()
    per_model_s = dev_ms / 1e3 / nm + extra_seconds
    ess_m = np.array([m["min_ess"] for m in out_models])
    return {"models": nm, "chains_per_model": nchains, "chunks": k, "steps_per_chain": k * chunk_nspc * thinning,
            "batch_seconds": dev_ms / 1e3, "seconds_per_model": per_model_s,
            "passed": int(sum(m["passed"] for m in out_models)), "rhat_max": float(rh_last.max()),
            "min_ess_median": float(np.median(ess_m)), "min_ess_per_s_median": float(np.median(ess_m) / per_model_s),
            "min_ess_per_s_min": float(ess_m.min() / per_model_s), "curve": curve, "per_model": out_models}


def _sm_count(torch, dev):
    return torch.cuda.get_device_properties(dev).multi_processor_count
