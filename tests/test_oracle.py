"""The CPU oracle pinned against the reference's known answers (CPU only).

Pins:
* Philox4x32-10 known-answer vectors of the Random123 distribution
  (the generator of Salmon et al., SC'11).
* The analytic moments the reference's GPU tests assert:
  cube [-1,1]^8 (tests/test_gpu_sampling_cube_moments.cu:60-111),
  6-D simplex (tests/test_gpu_sampling_simplex_moments.cu:61-70),
  feasibility <= 1e-7 on four polytopes (tests/test_gpu_sampling_feasibility.cu:144-185),
  the thin slab (tests/test_gpu_thin_polytope.cu:51-125), and the 2-D
  pair-step escape (tests/test_chr_pair_steps.cpp:103-162).
* The unit-cube workload's analytic answer: mean 0.5, variance 1/12.
* ESS / split-R-hat on series with known answers.
"""
import numpy as np
import pytest

import oracle.oracle as O
from naja_b200 import synth


def test_philox_known_answers():
    assert list(O.philox([0, 0, 0, 0], [0, 0])) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert list(O.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF, 0xFFFFFFFF])) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6,
                                                                          0x6D5451FD]
    assert list(O.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0])) == [
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_cube_moments(precision):
    A, b, x0 = synth.cube(8)
    S = O.chr_run(A, b, np.zeros(8), 20000, 20, 8, seed=42, precision=precision)
    assert S.shape == (160000, 8)
    mean, var = S.mean(0), S.var(0)
    assert np.all(np.abs(mean) < 0.05)
    assert np.all(np.abs(var - 1 / 3) / (1 / 3) < 0.15)
    corr = np.corrcoef(S.T)
    assert np.max(np.abs(corr - np.eye(8))) < 0.05


def test_simplex_moments():
    n = 6
    A, b, x0 = synth.simplex(n)
    S = O.chr_run(A, b, x0, 30000, 20, 8, seed=314, precision="fp64")
    mean = S.mean(0)
    cov = np.cov(S.T)
    e_mean = 1 / (n + 1)
    e_var = n / ((n + 1) ** 2 * (n + 2))
    e_cov = -1 / ((n + 1) ** 2 * (n + 2))
    assert np.all(np.abs(mean - e_mean) < 0.01)
    assert np.all(np.abs(np.diag(cov) - e_var) / e_var < 0.15)
    off = cov[~np.eye(n, dtype=bool)]
    assert np.all(np.abs(off - e_cov) < 0.005)
    assert (S @ A.T - b).max() <= 1e-7


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_feasibility(precision):
    cases = [(synth.cube(10), 42), (synth.simplex(8), 123), (synth.thin_slab(6, 1e-4), 777),
             (synth.random_dense(15, 60, 999), 555)]
    for (A, b, x0), seed in cases:
        S = O.chr_run(A, b, x0, 5000, 10, 4, seed=seed, precision=precision)
        tol = 1e-7 if precision == "fp64" else 1e-6 * np.maximum(1.0, np.abs(b))
        assert np.all(S @ A.T - b <= tol)


def test_thin_slab_pairs():
    d, eps = 10, 1e-4
    A = np.zeros((2 * d + 2, d))
    b = np.zeros(2 * d + 2)
    for i in range(d):
        A[2 * i, i], A[2 * i + 1, i] = 1.0, -1.0
        b[2 * i] = b[2 * i + 1] = 1.0
    A[2 * d, :3], A[2 * d + 1, :3] = 1.0, -1.0
    b[2 * d] = b[2 * d + 1] = eps
    Sc = O.chr_run(A, b, np.zeros(d), 10000, 5, 4, seed=42, pair_prob=0.0, precision="fp64")
    Sp = O.chr_run(A, b, np.zeros(d), 10000, 5, 4, seed=42, pair_prob=0.3, precision="fp64")
    for S in (Sc, Sp):
        assert (S @ A.T - b).max() <= 1e-7
    assert np.abs(Sc[:, :3].sum(1)).max() <= eps + 1e-7
    assert np.all(Sp[:, 3:].var(0) > 0.1)


def test_pair_steps_escape_slab():
    # |x| <= 1, |y| <= 1, |x + y| <= eps: coordinate moves stay on x == y,
    # pair moves (e0 - e1)/sqrt 2 travel along the slab.
    eps = 1e-4
    A = np.array([[1, 0], [-1, 0], [0, 1], [0, -1], [1, 1], [-1, -1]], dtype=float)
    b = np.array([1, 1, 1, 1, eps, eps])
    Sc = O.chr_run(A, b, np.zeros(2), 200, 1, 1, seed=123, pair_prob=0.0, precision="fp64")
    Sp = O.chr_run(A, b, np.zeros(2), 200, 1, 1, seed=123, pair_prob=1.0, precision="fp64")
    assert np.abs(Sc[:, 0] - Sc[:, 1]).max() < 1e-2
    assert np.abs(Sp[:, 0] - Sp[:, 1]).max() > 1e-1


def test_unit_cube_workload_analytic():
    A, b, x0 = synth.unit_cube_stacked(50)
    S = O.chr_run(A, b, x0, 2000, 8, 4, seed=0, precision="fp32")
    assert abs(S.mean() - 0.5) < 0.01
    assert abs(S.var(0).mean() - 1 / 12) / (1 / 12) < 0.05
    assert np.all((S >= 0) & (S <= 1))


def test_tiers_share_picks():
    g = synth.genome_shaped(n=120, d=30, density=0.2)
    _, t64 = O.chr_run(g["A"], g["b"], g["start"], 50, 3, 3, seed=7, pair_prob=0.3, precision="fp64", trace=True)
    S32, t32 = O.chr_run(g["A"], g["b"], g["start"], 50, 3, 3, seed=7, pair_prob=0.3, precision="fp32",
                         trace=True, resync_interval=16)
    S64 = O.chr_run(g["A"], g["b"], g["start"], 50, 3, 3, seed=7, pair_prob=0.3, precision="fp64")
    assert np.array_equal(t64, t32)
    scale = np.abs(S64).max()
    assert np.abs(S32 - S64).max() <= 1e-3 * scale


def test_ess_ar1():
    rng = np.random.default_rng(0)
    n, rho = 20000, 0.6
    x = np.empty(n)
    x[0] = rng.standard_normal()
    for t in range(1, n):
        x[t] = rho * x[t - 1] + np.sqrt(1 - rho ** 2) * rng.standard_normal()
    expected = n * (1 - rho) / (1 + rho)
    got = O.ess_series(x)
    # the estimator's own spread around n(1-rho)/(1+rho) is ~15-20% at this n
    assert abs(got - expected) / expected < 0.3
    # independent restatement: FFT autocovariance (numpy) + Geyer's rule
    y = x - x.mean()
    f = np.fft.rfft(y, 2 * n)
    acov = np.fft.irfft(f * np.conj(f), 2 * n)[:n] / n
    tau = 1.0
    for k in range(1, n // 2):
        pair = acov[2 * k - 1] / acov[0] + acov[2 * k] / acov[0]
        if pair < 0:
            break
        tau += 2 * pair
    assert abs(got - n / max(tau, 1.0)) < 1e-6 * n
    assert O.ess_series(np.ones(100)) == 1.0
    assert O.ess_series(np.arange(3.0)) == 3.0


def test_split_rhat_known():
    rng = np.random.default_rng(1)
    same = rng.standard_normal((4000, 3)).astype(np.float32)
    r = O.split_rhat(same, 4, layout=1)
    assert np.all(np.abs(r - 1.0) < 0.01)
    shifted = same.copy()
    shifted[0::4] += 3.0  # chain 0 of the interleaved layout sits elsewhere
    assert np.all(O.split_rhat(shifted, 4, layout=1) > 1.2)
    # the reference's windows see every chain in every window: no signal
    assert np.all(O.split_rhat(shifted, 4, layout=0) < 1.01)


def test_fft_ess_matches_direct_oracle():
    rng = np.random.default_rng(0)
    S = (np.cumsum(rng.standard_normal((4000, 5)), axis=0) * 0.05 + rng.standard_normal((4000, 5))).astype(np.float32)
    for layout in (0, 1):
        a, b = O.ess(S, 4, layout=layout), O.ess_fft(S, 4, layout=layout)
        assert np.abs(a - b).max() <= 1e-9 * np.abs(a).max()
