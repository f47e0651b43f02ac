"""`naja validate` metrics on the GPU (naja_validate) and their summaries.

Reference: src/validate/mcmc.cpp:91-194 and src/cli/validate_cli.cpp:138-233
of quothbonney/naja.  Two chain layouts:

* ``layout=0`` -- the reference's reading: rows [c*spc, (c+1)*spc) are
  "chain c" (mcmc.cpp:103-109).  Because the sampler writes chains
  interleaved (row r = sample r // k of chain r % k), these windows mix all
  chains round-robin.
* ``layout=1`` -- chain-correct: row r belongs to chain r % n_chains.

`summary` reproduces the reference's aggregates (per-dim ESS = min over
chains, min / p10 / median / max by linear-interpolation percentiles,
R-hat counts above 1.1 and 1.2, the OK/WARN/FAIL status rule);
`chain_ess` gives the metric's per-dim ESS = sum over chains.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, load
from .sampler import _is_torch, _ptr, _stream_of


def ess_rhat(samples, n_chains: int, layout: int = 1, ess: bool = True, rhat: bool = True):
    """Returns (ess[dim, n_chains], rhat[dim]) as float64 numpy arrays; a
    metric not asked for (ess=False or rhat=False) is returned as None and
    not computed."""
    N, dim = int(samples.shape[0]), int(samples.shape[1])
    if _is_torch(samples):
        import torch

        samples = samples.to(torch.float32).contiguous()
    else:
        samples = np.ascontiguousarray(np.asarray(samples, dtype=np.float32))
    e = np.empty((dim, n_chains), dtype=np.float64) if ess else None
    r = np.empty(dim, dtype=np.float64) if rhat else None
    check(load().naja_validate(_ptr(samples), N, dim, int(n_chains), int(layout), _ptr(e), _ptr(r),
                               _stream_of(samples)))
    return e, r


def percentile(v, q: float) -> float:
    """Linear-interpolation percentile as in mcmc.cpp:78-87 (float math)."""
    v = np.sort(np.asarray(v, dtype=np.float32))
    if v.size == 0:
        return 0.0
    pos = np.float32(q) * np.float32(v.size - 1)
    lo, hi = int(np.floor(pos)), int(np.ceil(pos))
    if lo == hi:
        return float(v[lo])
    t = np.float32(pos - np.float32(lo))
    return float(v[lo] * (np.float32(1.0) - t) + v[hi] * t)


def summary(ess, rhat) -> dict:
    """The reference's validate aggregates from per-(dim, chain) ESS and per-dim R-hat."""
    per_dim = np.min(ess, axis=1).astype(np.float32)
    rh = np.asarray(rhat, dtype=np.float32)
    dim = per_dim.size
    out = {
        "ess": {"min": float(per_dim.min()), "p10": percentile(per_dim, 0.10),
                "median": percentile(per_dim, 0.50), "max": float(per_dim.max())},
        "rhat": {"median": percentile(rh, 0.50), "max": float(rh.max()),
                 "above_1_1": int(np.sum(rh > 1.1)), "above_1_2": int(np.sum(rh > 1.2))},
        "per_dim_ess": per_dim,
        "per_dim_rhat": rh,
    }
    status = "OK"
    if out["rhat"]["above_1_2"] > dim // 4:
        status = "FAIL"
    elif out["rhat"]["above_1_1"] > dim // 4 or out["ess"]["min"] < 10:
        status = "WARN"
    out["status"] = status
    return out


def chain_ess(ess) -> np.ndarray:
    """Per-dim ESS summed over (de-interleaved) chains."""
    return np.sum(ess, axis=1)
