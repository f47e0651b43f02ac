"""CHR step kernel vs the CPU oracle, through the C ABI (GPU).

Both tiers are compared bit for bit: the kernel and the oracle perform the
same IEEE operations in the same order (explicit fma, exact max/min), so
the FP64 samples must be identical, and the FP32 tier's FP64 positions too.
The MRG32k3a mode is checked against the oracle fed with the cuRAND uniform
tape of the same (seed, chain) streams.
"""
import numpy as np
import pytest

import oracle.oracle as O
from naja_b200 import Polytope, mrg_tape, synth
from naja_b200._lib import InvalidArgument

pytestmark = pytest.mark.gpu


def _cases():
    g = synth.genome_shaped(n=260, d=70, density=0.08, seed_T=3, seed_u=4)
    return {
        "cube8": synth.cube(8),
        "simplex6": synth.simplex(6),
        "slab6": synth.thin_slab(6, 1e-4),
        "dense15x60": synth.random_dense(15, 60, 999),
        "genome260x70": (g["A"], g["b"], g["start"]),
    }


CASES = _cases()


def _run_both(name, precision, pair_prob=0.0, resync=0, nspc=40, thin=5, nchains=5, seed=11, **kw):
    A, b, x0 = CASES[name]
    P = Polytope(A, b)
    got = P.run(x0, nspc, thin, nchains, seed=seed, pair_prob=pair_prob, resync_interval=resync,
                precision=precision, out_dtype="f64", **kw)
    P.check()
    ref = O.chr_run(A, b, x0, nspc, thin, nchains, seed=seed, pair_prob=pair_prob, resync_interval=resync,
                    precision=precision, **{k: v for k, v in kw.items() if k in ("pairs", "ksparse_prob",
                                                                                  "ksparse_k", "pair_mode")})
    return got, ref


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("pair_prob", [0.0, 0.3])
def test_philox_bit_exact(cuda, name, precision, pair_prob):
    got, ref = _run_both(name, precision, pair_prob=pair_prob, resync=13 if precision == "fp32" else 0)
    assert np.array_equal(got, ref), np.abs(got - ref).max()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_resync_and_long_run(cuda, precision):
    got, ref = _run_both("genome260x70", precision, pair_prob=0.3, resync=64, nspc=200, thin=29, nchains=3)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("tpb", [32, 64, 128, 256, 512, 1024])
def test_thread_count_invariance(cuda, tpb):
    got, ref = _run_both("genome260x70", "fp32", pair_prob=0.3, resync=17, tpb=tpb)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("max_slots", [3, 4, 5, 8])
def test_ring_depth_invariance(cuda, max_slots):
    got, ref = _run_both("genome260x70", "fp64", pair_prob=0.5, max_slots=max_slots, nspc=60)
    assert np.array_equal(got, ref)


def test_pair_mode2_and_ksparse(cuda):
    A, b, x0 = CASES["genome260x70"]
    d = A.shape[1]
    rng = np.random.default_rng(5)
    perm = rng.permutation(d)
    th = rng.uniform(-np.pi, np.pi, d // 2)
    pairs = (perm[0::2][: d // 2], perm[1::2][: d // 2], np.cos(th), np.sin(th))
    for kw in ({"pair_mode": 2, "pairs": pairs}, {"ksparse_prob": 0.2, "ksparse_k": 5},
               {"ksparse_prob": 0.1, "ksparse_k": 40, "pair_mode": 2, "pairs": pairs}):
        for precision in ("fp64", "fp32"):
            got, ref = _run_both("genome260x70", precision, pair_prob=0.4, resync=9, **kw)
            assert np.array_equal(got, ref), (kw.keys(), precision)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_mrg_stream_matches_tape(cuda, precision):
    A, b, x0 = CASES["genome260x70"]
    nspc, thin, nchains, seed = 30, 4, 3, 2024
    P = Polytope(A, b)
    got = P.run(x0, nspc, thin, nchains, seed=seed, pair_prob=0.3, precision=precision, rng="mrg", out_dtype="f64")
    tape = mrg_tape(seed, nchains, 4 * nspc * thin + 8)
    ref = O.chr_run(A, b, x0, nspc, thin, nchains, pair_prob=0.3, precision=precision, tape=tape)
    assert np.array_equal(got, ref)


def test_float_output_is_rounded_fp64(cuda):
    A, b, x0 = CASES["dense15x60"]
    P = Polytope(A, b)
    g64 = P.run(x0, 50, 3, 4, seed=3, out_dtype="f64")
    g32 = P.run(x0, 50, 3, 4, seed=3, out_dtype="f32")
    assert g32.dtype == np.float32
    assert np.array_equal(g32, g64.astype(np.float32))


def test_chain_slices_compose(cuda):
    """Two launches over chain ranges [0,3) and [3,5) fill the same rows as one launch."""
    A, b, x0 = CASES["genome260x70"]
    P = Polytope(A, b)
    whole = P.run(x0, 20, 3, 5, seed=9, out_dtype="f64")
    out = np.zeros_like(whole)
    P.run(np.broadcast_to(x0, (3, len(x0))), 20, 3, 3, seed=9, out_dtype="f64", out=out, chain_base=0,
          out_nchains=5)
    P.run(np.broadcast_to(x0, (2, len(x0))), 20, 3, 2, seed=9, out_dtype="f64", out=out, chain_base=3,
          out_nchains=5)
    assert np.array_equal(out, whole)


def test_continuation_matches_one_run(cuda):
    """Philox chains continue exactly from X_final with step_offset."""
    A, b, x0 = CASES["dense15x60"]
    P = Polytope(A, b)
    whole = P.run(x0, 40, 5, 2, seed=1, out_dtype="f64", precision="fp64")
    xf = np.zeros((2, A.shape[1]))
    first = P.run(x0, 20, 5, 2, seed=1, out_dtype="f64", precision="fp64", X_final=xf)
    # slack is rebuilt from x at the start of the second call: identical when A x is exact
    second = P.run(xf, 20, 5, 2, seed=1, out_dtype="f64", precision="fp64", step_offset=100)
    assert np.array_equal(first, whole[:40])
    assert np.allclose(second, whole[40:], rtol=0, atol=1e-9)


def test_invalid_arguments(cuda):
    A, b, x0 = CASES["cube8"]
    P = Polytope(A, b)
    with pytest.raises(InvalidArgument, match="Invalid threads per block"):
        P.run(x0, 10, 1, 2, tpb=100)
    with pytest.raises(InvalidArgument):
        P.run(x0, 0, 1, 2)
    with pytest.raises(InvalidArgument):
        P.run(x0, 10, 0, 2)
    with pytest.raises(InvalidArgument):
        P.run(np.zeros(7), 10, 1, 2)


def test_bad_pair_index_reports_device_error(cuda):
    from naja_b200._lib import NajaError

    A, b, x0 = CASES["cube8"]
    P = Polytope(A, b)
    pairs = (np.array([0, 99]), np.array([1, 2]), np.array([1.0, 1.0]), np.array([0.0, 0.0]))
    with pytest.raises(NajaError, match="pair schedule index"):
        P.run(x0, 200, 1, 2, pair_prob=1.0, pair_mode=2, pairs=pairs)
    # the context stays usable
    out = P.run(x0, 10, 1, 2)
    assert np.isfinite(out).all()


@pytest.mark.parametrize("cluster", [2, 3, 4, 8])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_cluster_split_bit_exact(cuda, cluster, precision):
    """A chain's rows split over a thread-block cluster give the oracle's samples."""
    got, ref = _run_both("genome260x70", precision, pair_prob=0.3, resync=37 if precision == "fp32" else 0,
                         nspc=60, thin=7, nchains=3, cluster=cluster)
    assert np.array_equal(got, ref), np.abs(got - ref).max()


def test_cluster_split_large_model(cuda):
    """A genome-shaped model with few chains: one CTA per chain, the automatic
    choice and an 8-CTA cluster per chain agree, in both tiers and with
    k-sparse moves."""
    g = synth.genome_shaped(n=1300, d=300, density=0.08, seed_T=5, seed_u=6)
    P = Polytope(g["A"], g["b"])
    for precision in ("fp32", "fp64"):
        kw = dict(seed=4, pair_prob=0.3, ksparse_prob=0.05, ksparse_k=4, resync_interval=100,
                  precision=precision, out_dtype="f64")
        one = P.run(g["start"], 30, 11, 4, cluster=1, **kw)
        auto = P.run(g["start"], 30, 11, 4, cluster=0, **kw)
        eight = P.run(g["start"], 30, 11, 4, cluster=8, **kw)
        assert np.array_equal(one, auto) and np.array_equal(one, eight)


def test_cluster_mrg_matches_reference_tape(cuda):
    A, b, x0 = CASES["genome260x70"]
    nspc, thin, nchains, seed = 30, 4, 3, 2024
    P = Polytope(A, b)
    got = P.run(x0, nspc, thin, nchains, seed=seed, pair_prob=0.3, precision="fp64", rng="mrg", out_dtype="f64",
                cluster=4)
    tape = mrg_tape(seed, nchains, 4 * nspc * thin + 8)
    ref = O.chr_run(A, b, x0, nspc, thin, nchains, pair_prob=0.3, precision="fp64", tape=tape)
    assert np.array_equal(got, ref)


def test_cluster_rejects_bad_size(cuda):
    A, b, x0 = CASES["cube8"]
    P = Polytope(A, b)
    with pytest.raises(InvalidArgument, match="cluster"):
        P.run(x0, 10, 1, 2, cluster=9)


@pytest.mark.parametrize("extra_rows", [0, 1, 2, 3])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_dense_kernel_row_counts(cuda, extra_rows, precision):
    """The dense kernel at m % 4 = 0..3 and several thread counts: uniform
    chunks (every warp the same straight-line row pass, the rows past m
    repeating the last ones; m a multiple of the rows per lane) and the
    row-count-tested chunks give the oracle's samples and final slack."""
    import torch

    g = synth.genome_shaped(n=600, d=90, density=0.1, seed_T=8, seed_u=9)
    A = np.vstack([g["A"], g["A"][:extra_rows] * 0.5])
    b = np.concatenate([g["b"], g["b"][:extra_rows] * 0.5 + 1.0])
    P = Polytope(A, b)
    kw = dict(seed=4, pair_prob=0.3, resync_interval=40, ksparse_prob=0.1, ksparse_k=3)
    ref = O.chr_run(A, b, g["start"], 30, 6, 3, precision=precision, **kw)
    sfs = []
    for tpb in (64, 256, 512):
        sf = torch.empty((3, P.m), dtype=torch.float64 if precision == "fp64" else torch.float32, device="cuda")
        xf = np.empty((3, P.d))
        got = P.run(g["start"], 30, 6, 3, precision=precision, out_dtype="f64", sparse="dense", tpb=tpb,
                    X_final=xf, slack_final=sf, **kw)
        P.check()
        assert np.array_equal(got, ref), (tpb, np.abs(got - ref).max())
        sfs.append(sf)
    # columns read straight from global memory (a ring of fewer than 3 slots)
    direct = P.run(g["start"], 30, 6, 3, precision=precision, out_dtype="f64", sparse="dense", max_slots=2, **kw)
    assert np.array_equal(direct, ref)
    # every thread count leaves the same final slack, close to b - A x_final
    assert all(torch.equal(sfs[0], s) for s in sfs[1:])
    exact = b - xf @ A.T
    tol = 1e-9 if precision == "fp64" else 1e-3
    assert np.abs(sfs[0].cpu().numpy() - exact).max() <= tol * max(1.0, np.abs(b).max())
