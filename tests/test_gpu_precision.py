"""FP32 tier against the FP64 tier (GPU): the stated tolerance.

Same polytope, same Philox streams.  The FP32 tier keeps the slack in FP32
and recomputes it as b - A x in FP64 every K steps (the reference's resync
hook, src/gpu/chr.cu:384-395 of quothbonney/naja).  Checked here:

* slack drift: after the last K steps of a run, |slack32 - (b - A x)| in
  FP64 at the final state is at most 1e-5 max(1, |b|) for K = 64 and grows
  with K (K = 1024 no smaller than K = 64);
* positions: for the first 128 steps of every chain, every coordinate of the
  FP32-tier chain is within 1e-3 of that coordinate's range (over the FP64
  run) of the FP64-tier chain; after that the chains may separate (a
  rounding difference changes which constraint bounds a chord), both
  remaining samplers of the same uniform target;
* the FP32 samples satisfy A y <= b + 1e-6 max(1, |b|).
"""
import numpy as np
import pytest

from naja_b200 import Polytope, synth

pytestmark = pytest.mark.gpu


def _run(P, g, precision, K, nspc, thin, nch):
    import torch

    dev = torch.device("cuda", 0)
    m, d = g["A"].shape
    out = torch.empty((nspc * nch, d), dtype=torch.float64, device=dev)
    xf = torch.empty((nch, d), dtype=torch.float64, device=dev)
    sf = torch.empty((nch, m), dtype=torch.float64 if precision == "fp64" else torch.float32, device=dev)
    P.run(np.zeros((nch, d)), nspc, thin, nch, seed=17, pair_prob=0.3, precision=precision, resync_interval=K,
          out=out, out_dtype="f64", X_final=xf, slack_final=sf)
    P.check()
    A = torch.from_numpy(g["A"]).to(dev)
    b = torch.from_numpy(g["b"]).to(dev)
    drift = ((sf.double() - (b - xf @ A.T)).abs() / b.abs().clamp(min=1.0)).max().item()
    return out.cpu().numpy(), drift


def test_fp32_tier_tolerance(cuda):
    g = synth.genome_shaped(n=1200, d=300, density=0.08, seed_T=31, seed_u=32)
    P = Polytope(g["A"], g["b"])
    nspc, thin, nch = 64, 64, 8  # 4,096 steps: a multiple of every K
    y64, d64 = _run(P, g, "fp64", 0, nspc, thin, nch)
    assert d64 < 1e-9
    drift = {}
    for K in (64, 1024):
        y32, drift[K] = _run(P, g, "fp32", K, nspc, thin, nch)
        viol = y32 @ g["A"].T - g["b"]
        assert (viol <= 1e-6 * np.maximum(1.0, np.abs(g["b"]))).all()
        span = np.maximum(y64.max(axis=0) - y64.min(axis=0), 1e-12)
        rel = (np.abs(y32 - y64) / span).reshape(nspc, nch, -1).max(axis=2)  # (saved sample, chain)
        for c in range(nch):
            off = np.nonzero(rel[:, c] > 1e-3)[0]
            # saved sample s follows step s * thin + 1: the chains agree through the step of the
            # last saved sample before the first one that differs
            agreed = (off[0] - 1) * thin + 1 if off.size else nspc * thin
            assert agreed >= 128, (K, c, agreed)
    assert drift[64] <= 1e-5, drift
    assert drift[1024] >= drift[64], drift
