"""FP64 slack recompute between step-kernel segments (GPU).

A dense single-CTA run whose recompute interval K is shorter than the run,
on a polytope whose A has at least 2^19 entries, runs as segments of K
steps; before each segment one kernel over the whole GPU recomputes every
chain's slack b - A x in FP64, and the segment starts from it.  Its samples,
final positions and final slack must be those of the single launch (the
wait-cycle instrumentation keeps a run in one launch) and the oracle's, bit
for bit: at the rounded headline shape (16 chains, thinning 116, pair 0.3,
K = 2048) in the FP32 tier, against the reference's own kernel in the FP64
tier with its MRG32k3a streams, with a run length that is not a multiple of
K and a thinning that does not divide K, and continued through step_offset.
"""
import numpy as np
import pytest

import oracle.oracle as O
from naja_b200 import Polytope, synth
from naja_b200 import gate

pytestmark = pytest.mark.gpu


def _single_launch(P, *args, nchains, **kw):
    """The same run kept in one launch (instrumented runs are not segmented)."""
    import torch

    wc = torch.zeros(4 * nchains, dtype=torch.int64, device="cuda")
    return P.run(*args, nchains, wait_cycles=wc, **kw)


@pytest.fixture(scope="module")
def rounded():
    g = synth.genome_shaped(n=2600, d=700, density=0.08, seed_T=0, seed_u=1)
    return gate.make_rounding("dikin_full", g["A"], g["b"], g["start"])


def test_rounded_headline_shape_fp32_matches_oracle(cuda, rounded):
    R = rounded
    P = Polytope(R.A, R.b)
    kw = dict(seed=0, pair_prob=0.3, resync_interval=2048, precision="fp32")
    nspc, thin, nch = 20, 116, 16  # 2,320 steps: segments of 2,048 and 272 steps
    choice = P.kernel_choice(12500, thin, nch, **kw)
    assert choice["kernel"] == "dense" and choice["threads"] == 448, choice
    xf = np.empty((nch, R.A.shape[1]))
    got = P.run(R.z0, nspc, thin, nch, out_dtype="f64", X_final=xf, **kw)
    P.check()
    ref, ref_xf = O.chr_run(R.A, R.b, R.z0, nspc, thin, nch, x_final=True, **kw)
    assert np.array_equal(got, ref), np.abs(got - ref).max()
    assert np.array_equal(xf, ref_xf)
    xf1 = np.empty_like(xf)
    one = _single_launch(P, R.z0, nspc, thin, nchains=nch, out_dtype="f64", X_final=xf1, **kw)
    assert np.array_equal(one, got) and np.array_equal(xf1, xf)


@pytest.mark.skipif(not O.reference_available(), reason="reference build (oracle/_ref) not present")
def test_rounded_headline_shape_fp64_mrg_matches_reference_kernel(cuda, rounded):
    R = rounded
    P = Polytope(R.A, R.b)
    nspc, thin, nch = 20, 116, 16
    S_ref, _, _ = O.reference_chr_run(R.A, R.b, R.z0, nspc, thin, nch, tpb=128, seed=3, pair_prob=0.3,
                                      resync_interval=1024)
    kw = dict(seed=3, pair_prob=0.3, resync_interval=1024, precision="fp64", rng="mrg", out_dtype="f64")
    got = P.run(R.z0, nspc, thin, nch, **kw)
    P.check()
    assert np.array_equal(got, S_ref), np.abs(got - S_ref).max()
    assert np.array_equal(_single_launch(P, R.z0, nspc, thin, nchains=nch, **kw), got)


@pytest.mark.parametrize("sparse", ["dense", "columns"])
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_ragged_segments_and_final_slack(cuda, precision, sparse):
    """K = 100 with thinning 7 over 350 steps: segments of 100, 100, 100 and
    50 steps, samples saved inside segments; the final slack too; for the
    dense and the compressed-column step kernel."""
    import torch

    g = synth.genome_shaped(n=1300, d=420, density=0.1, seed_T=4, seed_u=5)  # m d = 1,092,000
    P = Polytope(g["A"], g["b"])
    nch, nspc, thin, K = 4, 50, 7, 100
    kw = dict(seed=11, pair_prob=0.3, resync_interval=K, precision=precision, sparse=sparse, out_dtype="f64")
    dt = torch.float64 if precision == "fp64" else torch.float32
    sf = torch.empty((nch, P.m), dtype=dt, device="cuda")
    got = P.run(g["start"], nspc, thin, nch, slack_final=sf, **kw)
    P.check()
    ref = O.chr_run(g["A"], g["b"], g["start"], nspc, thin, nch, seed=11, pair_prob=0.3, resync_interval=K,
                    precision=precision)
    assert np.array_equal(got, ref), np.abs(got - ref).max()
    sf1 = torch.empty_like(sf)
    one = _single_launch(P, g["start"], nspc, thin, nchains=nch, slack_final=sf1, **kw)
    assert np.array_equal(one, got)
    assert torch.equal(sf, sf1)


def test_continuation_through_step_offset(cuda):
    """Two calls of whole recompute intervals (the overlapped pipeline's
    chunks) continue the chains of one call."""
    g = synth.genome_shaped(n=1300, d=420, density=0.1, seed_T=4, seed_u=5)
    P = Polytope(g["A"], g["b"])
    nch, thin, K = 4, 5, 100
    kw = dict(seed=2, pair_prob=0.3, resync_interval=K, sparse="dense", out_dtype="f64")
    whole = P.run(g["start"], 100, thin, nch, **kw)
    xf = np.empty((nch, P.d))
    a = P.run(g["start"], 40, thin, nch, X_final=xf, **kw)  # 200 steps = 2 K
    b = P.run(xf, 60, thin, nch, step_offset=200, **kw)
    P.check()
    assert np.array_equal(np.vstack([a, b]), whole)
