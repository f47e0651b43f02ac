"""Parity with the reference's own kernel (GPU).

The reference's src/gpu/{chr,dmatrix,dvector,backmap}.cu are compiled
unmodified for sm_100a into oracle/_ref/ (oracle/refharness/Makefile) and
driven through their own API (naja::gpu::CoordinateHitAndRun).  With the
cuRAND MRG32k3a stream mode, the FP64 tier of this project's kernel and the
oracle fed with the recorded cuRAND tape must reproduce the reference's
samples bit for bit.  The reference initialises slack with cublasDgemm,
whose summation order is its own, so the start points here make A x0 exact
(x0 = 0), or a resync at t = 0 recomputes slack with the reference's own
sequential formula.
"""
import numpy as np
import pytest

import oracle.oracle as O
from naja_b200 import Polytope, mrg_tape, synth

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.reference_available(), reason="reference build (oracle/_ref) absent")]


def _cases():
    g = synth.genome_shaped(n=260, d=70, density=0.08, seed_T=3, seed_u=4)
    return {
        "cube8": synth.cube(8),
        "dense15x60": synth.random_dense(15, 60, 999),
        "slab6": synth.thin_slab(6, 1e-4),
        "genome260x70": (g["A"], g["b"], g["start"]),
    }


CASES = _cases()


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("pair_prob", [0.0, 0.3])
def test_kernel_and_oracle_reproduce_reference(cuda, name, pair_prob):
    A, b, x0 = CASES[name]
    nspc, thin, k, seed = 40, 5, 4, 77
    ref, _, _ = O.reference_chr_run(A, b, x0, nspc, thin, k, tpb=128, seed=seed, pair_prob=pair_prob)
    P = Polytope(A, b)
    ours = P.run(x0, nspc, thin, k, seed=seed, pair_prob=pair_prob, precision="fp64", rng="mrg", out_dtype="f64")
    tape = mrg_tape(seed, k, 4 * nspc * thin + 8)
    orc = O.chr_run(A, b, x0, nspc, thin, k, pair_prob=pair_prob, precision="fp64", tape=tape)
    assert np.array_equal(orc, ref), np.abs(orc - ref).max()
    assert np.array_equal(ours, ref), np.abs(ours - ref).max()


def test_resync_formula_matches_reference(cuda):
    """Non-trivial start: the t = 0 resync replaces cuBLAS's slack init on both sides."""
    A, b, x0 = synth.simplex(6)
    nspc, thin, k, seed, K = 60, 7, 3, 5, 10 ** 6
    ref, _, _ = O.reference_chr_run(A, b, x0, nspc, thin, k, tpb=64, seed=seed, pair_prob=0.3, resync_interval=K)
    P = Polytope(A, b)
    ours = P.run(x0, nspc, thin, k, seed=seed, pair_prob=0.3, precision="fp64", rng="mrg", out_dtype="f64",
                 resync_interval=K)
    assert np.array_equal(ours, ref), np.abs(ours - ref).max()


def test_reference_pair_mode2_and_ksparse(cuda):
    A, b, x0 = CASES["genome260x70"]
    d = A.shape[1]
    rng = np.random.default_rng(8)
    perm = rng.permutation(d)
    th = rng.uniform(-np.pi, np.pi, d // 2)
    pairs = (perm[0::2][: d // 2], perm[1::2][: d // 2], np.cos(th), np.sin(th))
    kw = dict(pair_prob=0.3, pair_mode=2, pairs=pairs, ksparse_prob=0.1, ksparse_k=6)
    ref, _, _ = O.reference_chr_run(A, b, x0, 30, 4, 3, tpb=256, seed=3, **kw)
    P = Polytope(A, b)
    ours = P.run(x0, 30, 4, 3, seed=3, precision="fp64", rng="mrg", out_dtype="f64", **kw)
    assert np.array_equal(ours, ref), np.abs(ours - ref).max()


def test_reference_backmap_close(cuda):
    from naja_b200 import backmap

    g = synth.genome_shaped(n=260, d=70, density=0.08, seed_T=3, seed_u=4)
    ref_s, ref_v, _ = O.reference_chr_run(g["A"], g["b"], g["start"], 50, 3, 4, seed=1, T=g["T"],
                                          shift=np.linspace(-1, 1, 260))
    V = backmap(g["T"], np.linspace(-1, 1, 260), ref_s, mode="fp64", out_dtype=np.float64)
    assert np.allclose(V, ref_v, rtol=1e-12, atol=1e-12 * np.abs(ref_v).max())
