"""Parity at the shapes the benchmark runs (GPU).

* Genome-shaped polytope at full size (n 2600, d 700, m 5200, 16 chains,
  thinning 116, pair-prob 0.3, resync 2048): the automatic kernel choice is
  the compressed-column kernel with 256 consumer threads, and its samples are
  the oracle's bit for bit (FP32 tier); in the FP64 tier with the MRG32k3a
  streams they are the reference kernel's own (src/gpu/chr.cu:232-490 of
  quothbonney/naja) bit for bit.
* The 64-model conditioned batch (m 5,202-5,400) in the compressed and dense
  batched kernels: every model equals its standalone run, and one model the
  oracle.
* The unit cube [0,1]^50 (4 chains x 2000 samples, thinning 8, seed 0): the
  oracle's samples bit for bit, and the analytic mean 1/2 and variance 1/12.
Runs are shortened (fewer samples per chain) where the CPU oracle has to
follow them.
"""
import numpy as np
import pytest

import oracle.oracle as O
from naja_b200 import Polytope, synth
from naja_b200 import validate as V
from naja_b200.batch import Batch, Shape

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def genome():
    return synth.genome_shaped(n=2600, d=700, density=0.08, seed_T=0, seed_u=1)


def test_genome_full_shape_fp32_matches_oracle(cuda, genome):
    g = genome
    P = Polytope(g["A"], g["b"])
    kw = dict(seed=0, pair_prob=0.3, resync_interval=2048, precision="fp32")
    nspc, thin, nch = 20, 116, 16  # 2,320 steps per chain: one FP64 recompute at step 2048
    choice = P.kernel_choice(12500, thin, nch, **kw)
    assert choice["kernel"] == "columns" and choice["threads"] == 256, choice
    got = P.run(g["start"], nspc, thin, nch, out_dtype="f64", **kw)
    P.check()
    ref = O.chr_run(g["A"], g["b"], g["start"], nspc, thin, nch, **kw)
    assert np.array_equal(got, ref), np.abs(got - ref).max()
    # the float samples are the FP64 ones rounded once
    got32 = P.run(g["start"], nspc, thin, nch, **kw)
    assert np.array_equal(got32, ref.astype(np.float32))


@pytest.mark.skipif(not O.reference_available(), reason="reference build (oracle/_ref) not present")
def test_genome_full_shape_fp64_matches_reference_kernel(cuda, genome):
    g = genome
    P = Polytope(g["A"], g["b"])
    nspc, thin, nch = 12, 116, 16
    S_ref, _, _ = O.reference_chr_run(g["A"], g["b"], np.zeros(700), nspc, thin, nch, tpb=128, seed=0,
                                      pair_prob=0.3)
    got = P.run(np.zeros(700), nspc, thin, nch, seed=0, pair_prob=0.3, precision="fp64", rng="mrg",
                out_dtype="f64")
    P.check()
    assert np.array_equal(got, S_ref), np.abs(got - S_ref).max()


@pytest.fixture(scope="module")
def batch64(genome):
    import torch

    base = genome
    variants = synth.conditioned_variants(base, 64, max_reactions=100, seed=2)
    polys = [Polytope(np.vstack([base["A"], v["extra_A"]]), np.concatenate([base["b"], v["extra_b"]]))
             for v in variants]
    ms = [p.m for p in polys]
    assert min(ms) >= 5200 and max(ms) <= 5400 and max(ms) > 5300
    dev = torch.device("cuda", 0)
    yield polys, dev
    for p in polys:
        p.close()


@pytest.mark.parametrize("shape", [Shape(256, 8, 1, 0, 1), Shape(128, 4, 1, 0, 1), Shape(256, 3, 1, 0, 0)],
                         ids=["columns256x8", "columns128x4", "dense256x3"])
def test_conditioned_batch_of_64_equals_standalone(cuda, batch64, shape):
    import torch

    polys, dev = batch64
    nch, nspc, thin = 8, 3, 116
    kw = dict(seed=5, pair_prob=0.3, resync_interval=2048)
    d = polys[0].d
    X = [torch.zeros((nch, d), dtype=torch.float64, device=dev) for _ in polys]
    outs = [torch.empty((nspc * nch, d), dtype=torch.float32, device=dev) for _ in polys]
    B = Batch(polys)
    B.run(X, outs, nspc, thin, nch, shape=shape, seed_stride=7, **kw)
    torch.cuda.synchronize()
    polys[0].check()
    for k, P in enumerate(polys):
        ref = P.run(np.zeros(d), nspc, thin, nch, seed=5 + 7 * k, pair_prob=0.3, resync_interval=2048)
        assert np.array_equal(outs[k].cpu().numpy(), ref), f"model {k} (m={P.m}) differs from its standalone run"


def test_conditioned_batch_model_matches_oracle(cuda, genome, batch64):
    import torch

    polys, dev = batch64
    base = genome
    variants = synth.conditioned_variants(base, 64, max_reactions=100, seed=2)
    k = 37
    A = np.vstack([base["A"], variants[k]["extra_A"]])
    b = np.concatenate([base["b"], variants[k]["extra_b"]])
    nch, nspc, thin = 8, 3, 116
    d = A.shape[1]
    X = [torch.zeros((nch, d), dtype=torch.float64, device=dev) for _ in polys]
    outs = [torch.empty((nspc * nch, d), dtype=torch.float64, device=dev) for _ in polys]
    Batch(polys).run(X, outs, nspc, thin, nch, shape=Shape(256, 8, 1, 0, 1), seed_stride=7, seed=5, pair_prob=0.3,
                     resync_interval=2048, out_dtype="f64")
    torch.cuda.synchronize()
    ref = O.chr_run(A, b, np.zeros(d), nspc, thin, nch, seed=5 + 7 * k, pair_prob=0.3, resync_interval=2048,
                    precision="fp32")
    assert np.array_equal(outs[k].cpu().numpy(), ref)


def test_unit_cube_d50_matches_oracle_and_moments(cuda):
    A, b, x0 = synth.unit_cube_stacked(50)
    P = Polytope(A, b)
    nspc, thin, nch = 2000, 8, 4
    got = P.run(x0, nspc, thin, nch, seed=0, pair_prob=0.0, precision="fp32", out_dtype="f64")
    P.check()
    ref = O.chr_run(A, b, x0, nspc, thin, nch, seed=0, pair_prob=0.0, precision="fp32")
    assert np.array_equal(got, ref)
    assert got.min() >= 0.0 and got.max() <= 1.0
    ess = V.chain_ess(V.ess_rhat(got.astype(np.float32), nch, layout=1)[0])  # per dim, summed over chains
    mean = got.mean(axis=0)
    var = got.var(axis=0, ddof=1)
    # per coordinate: 5 standard errors of the mean and of the variance at that dimension's ESS
    se_mean = np.sqrt((1.0 / 12.0) / ess)
    se_var = np.sqrt((1.0 / 80.0 - 1.0 / 144.0) / ess)  # Var((x - 1/2)^2) = mu4 - sigma^4 for U(0, 1)
    assert np.all(np.abs(mean - 0.5) < 5 * se_mean), np.abs(mean - 0.5).max()
    assert np.all(np.abs(var - 1.0 / 12.0) < 5 * se_var), np.abs(var - 1 / 12).max()
    # over all 50 coordinates the averages are much tighter
    assert abs(mean.mean() - 0.5) < 5 * se_mean.mean() / np.sqrt(50)
    assert abs(var.mean() - 1.0 / 12.0) < 5 * se_var.mean() / np.sqrt(50)
