"""Sparse-column CHR kernel vs the CPU oracle and vs the dense kernel (GPU).

The compressed-column kernel walks only the rows where the step's column(s)
of A are nonzero; its samples must equal the oracle's (and so the dense
kernel's) bit for bit in both tiers, for coordinate, random-pair and Jacobi
pair directions, with the FP64 recompute, with the reference's MRG32k3a
streams, for every consumer thread count, and on degenerate chords, where it
repeats the pass over all rows.
"""
import numpy as np
import pytest

import oracle.oracle as O
from naja_b200 import Polytope, mrg_tape, synth
from naja_b200._lib import NajaError

pytestmark = pytest.mark.gpu


def _genome(n=260, d=70, seed=3):
    g = synth.genome_shaped(n=n, d=d, density=0.08, seed_T=seed, seed_u=seed + 1)
    return g["A"], g["b"], g["start"]


CASES = {
    "genome260x70": _genome(),
    "genome600x150": _genome(600, 150, 7),
    "cube8": synth.cube(8),
    "dense15x60": synth.random_dense(15, 60, 999),
    "simplex6": synth.simplex(6),
}


def _oracle(A, b, x0, nspc, thin, nchains, **kw):
    keep = {k: v for k, v in kw.items() if k in ("seed", "pair_prob", "resync_interval", "precision", "pairs",
                                                  "pair_mode", "tape")}
    return O.chr_run(A, b, x0, nspc, thin, nchains, **keep)


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("pair_prob", [0.0, 0.3, 1.0])
def test_columns_bit_exact(cuda, name, precision, pair_prob):
    A, b, x0 = CASES[name]
    kw = dict(seed=11, pair_prob=pair_prob, resync_interval=13 if precision == "fp32" else 0, precision=precision)
    P = Polytope(A, b)
    got = P.run(x0, 40, 5, 5, out_dtype="f64", sparse="columns", **kw)
    P.check()
    ref = _oracle(A, b, x0, 40, 5, 5, **kw)
    assert np.array_equal(got, ref), np.abs(got - ref).max()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_columns_long_run_matches_dense(cuda, precision):
    A, b, x0 = CASES["genome600x150"]
    P = Polytope(A, b)
    kw = dict(seed=5, pair_prob=0.3, resync_interval=64, precision=precision, out_dtype="f64")
    sp = P.run(x0, 200, 29, 6, sparse="columns", **kw)
    de = P.run(x0, 200, 29, 6, sparse="dense", **kw)
    auto = P.run(x0, 200, 29, 6, **kw)
    assert np.array_equal(sp, de) and np.array_equal(sp, auto)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_columns_jacobi_pairs(cuda, precision):
    A, b, x0 = CASES["genome260x70"]
    d = A.shape[1]
    rng = np.random.default_rng(5)
    perm = rng.permutation(d)
    th = rng.uniform(-np.pi, np.pi, d // 2)
    pairs = (perm[0::2][: d // 2], perm[1::2][: d // 2], np.cos(th), np.sin(th))
    kw = dict(seed=2, pair_prob=0.6, pair_mode=2, pairs=pairs, resync_interval=9, precision=precision)
    P = Polytope(A, b)
    got = P.run(x0, 50, 6, 4, out_dtype="f64", sparse="columns", **kw)
    ref = _oracle(A, b, x0, 50, 6, 4, **kw)
    assert np.array_equal(got, ref)


def test_columns_pair_of_a_column_with_itself(cuda):
    """A Jacobi pair (i, i): every row of column j is shared with column i."""
    A, b, x0 = CASES["genome260x70"]
    pairs = (np.array([3, 5]), np.array([3, 5]), np.array([0.6, 0.8]), np.array([0.8, 0.6]))
    for precision in ("fp64", "fp32"):
        kw = dict(seed=8, pair_prob=1.0, pair_mode=2, pairs=pairs, precision=precision)
        P = Polytope(A, b)
        got = P.run(x0, 20, 3, 3, out_dtype="f64", sparse="columns", **kw)
        de = P.run(x0, 20, 3, 3, out_dtype="f64", sparse="dense", **kw)
        assert np.array_equal(got, de, equal_nan=True)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_columns_mrg_matches_tape(cuda, precision):
    A, b, x0 = CASES["genome260x70"]
    nspc, thin, nchains, seed = 30, 4, 3, 2024
    P = Polytope(A, b)
    got = P.run(x0, nspc, thin, nchains, seed=seed, pair_prob=0.3, precision=precision, rng="mrg",
                out_dtype="f64", sparse="columns")
    tape = mrg_tape(seed, nchains, 4 * nspc * thin + 8)
    ref = O.chr_run(A, b, x0, nspc, thin, nchains, pair_prob=0.3, precision=precision, tape=tape)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("max_slots", [3, 4, 8])
def test_columns_ring_depth_invariance(cuda, max_slots):
    A, b, x0 = CASES["genome260x70"]
    P = Polytope(A, b)
    kw = dict(seed=4, pair_prob=0.5, precision="fp32", resync_interval=31, out_dtype="f64")
    got = P.run(x0, 60, 5, 3, sparse="columns", max_slots=max_slots, **kw)
    ref = _oracle(A, b, x0, 60, 5, 3, **kw)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("tpb", [32, 64, 128, 256, 512])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_columns_thread_count_invariance(cuda, tpb, precision):
    A, b, x0 = CASES["genome600x150"]
    kw = dict(seed=6, pair_prob=0.4, resync_interval=23, precision=precision)
    P = Polytope(A, b)
    got = P.run(x0, 30, 7, 4, out_dtype="f64", sparse="columns", tpb=tpb, **kw)
    ref = _oracle(A, b, x0, 30, 7, 4, **kw)
    assert np.array_equal(got, ref)


def test_columns_chain_slices_and_final_state(cuda):
    A, b, x0 = CASES["genome260x70"]
    P = Polytope(A, b)
    xf_w = np.zeros((5, A.shape[1]))
    whole = P.run(x0, 20, 3, 5, seed=9, out_dtype="f64", sparse="columns", X_final=xf_w)
    xf_d = np.zeros((5, A.shape[1]))
    dense = P.run(x0, 20, 3, 5, seed=9, out_dtype="f64", sparse="dense", X_final=xf_d)
    assert np.array_equal(whole, dense) and np.array_equal(xf_w, xf_d)
    out = np.zeros_like(whole)
    P.run(np.broadcast_to(x0, (3, len(x0))), 20, 3, 3, seed=9, out_dtype="f64", out=out, chain_base=0,
          out_nchains=5, sparse="columns")
    P.run(np.broadcast_to(x0, (2, len(x0))), 20, 3, 2, seed=9, out_dtype="f64", out=out, chain_base=3,
          out_nchains=5, sparse="columns")
    assert np.array_equal(out, whole)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_degenerate_chord_repeats_dense_pass(cuda, precision):
    """x1 is unbounded below: on a step along e1 the nonzero rows give no
    negative ratio, the kernel falls back to all rows, and the first step of
    every chain equals the dense kernel's (an infinite or NaN move included)."""
    A = np.array([[1.0, 0.0], [0.0, 1.0], [0.0, -1.0], [0.0, 0.0]])
    b = np.array([1.0, 1.0, 1.0, 1.0])
    x0 = np.zeros(2)
    P = Polytope(A, b)
    kw = dict(seed=3, precision=precision, out_dtype="f64")
    got = P.run(x0, 1, 1, 64, sparse="columns", **kw)
    de = P.run(x0, 1, 1, 64, sparse="dense", **kw)
    assert np.array_equal(got, de, equal_nan=True)
    moved_x1 = got[:, 1] == 0.0
    assert moved_x1.any() and (~moved_x1).any()
    assert not np.isfinite(got[moved_x1, 0]).all()
    # the other steps stay inside the bounded coordinate
    assert (np.abs(got[~moved_x1, 1]) <= 1.0).all()


def test_columns_rejects_what_it_cannot_run(cuda):
    A, b, x0 = CASES["genome260x70"]
    P = Polytope(A, b)
    with pytest.raises(NajaError, match="compressed columns"):
        P.run(x0, 10, 1, 2, sparse="columns", ksparse_prob=0.1)
    with pytest.raises(NajaError, match="compressed columns"):
        P.run(x0, 10, 1, 2, sparse="columns", tpb=1024)
    with pytest.raises(NajaError, match="compressed columns"):
        P.run(x0, 10, 1, 2, sparse="columns", cluster=2)
    # automatic falls back to the dense kernel for those and agrees
    a = P.run(x0, 10, 1, 2, ksparse_prob=0.1, seed=1, out_dtype="f64")
    d = P.run(x0, 10, 1, 2, ksparse_prob=0.1, seed=1, out_dtype="f64", sparse="dense")
    assert np.array_equal(a, d)


def test_automatic_choice(cuda):
    A, b, x0 = CASES["genome600x150"]
    P = Polytope(A, b)
    assert P.kernel_choice(10, 1, 4)["kernel"] == "columns"
    assert P.kernel_choice(10, 1, 4, precision="fp64")["kernel"] == "columns"
    assert P.kernel_choice(10, 1, 4, tpb=128)["kernel"] == "dense"
    assert P.kernel_choice(10, 1, 4, ksparse_prob=0.1)["kernel"] == "dense"
    assert P.kernel_choice(10, 1, 4, sparse="dense")["kernel"] == "dense"
    Ad, bd, xd = CASES["dense15x60"]
    assert Polytope(Ad, bd).kernel_choice(10, 1, 4)["kernel"] == "dense"
    ch = P.kernel_choice(10, 1, 4, sparse="columns")
    assert ch["threads"] == 64 and ch["slots"] >= 3 and ch["smem"] > 0
    assert P.kernel_choice(10, 1, 4, sparse="columns", tpb=256)["threads"] == 256


@pytest.mark.parametrize("pair_mode", [1, 2])
def test_columns_pair_steps_by_search_when_scratch_does_not_fit(cuda, pair_mode):
    """m = 12,000 rows in the FP64 tier: slack and a scratch column of 12,001
    doubles each leave no room for three staged columns, so pair steps
    combine the columns by binary search; the samples stay the oracle's."""
    A, b, x0 = _genome(6000, 100, 21)
    assert A.shape[0] == 12000
    P = Polytope(A, b)
    assert P.kernel_choice(10, 5, 3, precision="fp64", pair_prob=0.5)["kernel"] == "columns"
    d = A.shape[1]
    rng = np.random.default_rng(2)
    perm = rng.permutation(d)
    th = rng.uniform(-np.pi, np.pi, d // 2)
    pairs = (perm[0::2], perm[1::2], np.cos(th), np.sin(th)) if pair_mode == 2 else None
    kw = dict(seed=9, pair_prob=0.5, precision="fp64", pair_mode=pair_mode, pairs=pairs)
    got = P.run(x0, 30, 5, 3, out_dtype="f64", sparse="columns", **kw)
    P.check()
    ref = _oracle(A, b, x0, 30, 5, 3, **kw)
    assert np.array_equal(got, ref), np.abs(got - ref).max()
