"""Affine roundings on the host (CPU): the reference's Dikin preconditioner
(src/rounding/dikin_precondition.cpp:36-183 of quothbonney/naja) on
polytopes with a known answer, the whole-ellipsoid Dikin rounding and the
covariance rounding."""
import numpy as np
import pytest
import scipy.linalg

from naja_b200 import rounding, synth


def _thin_box(d, k, eps):
    """[-1, 1]^d with coordinate k limited to [-eps, eps]."""
    A = np.vstack([np.eye(d), -np.eye(d)])
    b = np.ones(2 * d)
    b[k] = b[d + k] = eps
    return A, b


@pytest.mark.parametrize("eps,alpha", [(0.005, 200.0), (0.002, 500.0), (1e-4, 1000.0)])
def test_dikin_thin_box_known_answer(eps, alpha):
    d, k = 6, 2
    A, b = _thin_box(d, k, eps)
    r = rounding.dikin(A, b, np.zeros(d))
    # tight set: the two facets of the thin side (distance eps <= 100 * eps); the
    # other facets are at distance 1 > 100 eps
    assert r.info["tight_rows"] == 2 and r.info["n_corrected"] == 1
    # target chord: median chord along the coordinate axes = 2; alpha = clip(2 / (2 eps), 1, 1000)
    assert r.info["target_chord"] == pytest.approx(2.0)
    assert r.info["alphas"][0] == pytest.approx(alpha)
    expect = np.eye(d)
    expect[k, k] = 1.0 / alpha
    assert np.allclose(r.M, expect, atol=1e-12)
    assert np.allclose(r.A, A @ expect) and np.allclose(r.b, b) and np.allclose(r.c, 0.0)
    # in z the thin side is 2 eps alpha wide: the box is a cube when alpha is not clipped
    chord = rounding.chord_along(r.A, r.b, np.zeros(d), np.eye(d)[k])
    assert chord == pytest.approx(2 * eps * alpha)


def test_dikin_not_tight_when_all_facets_equal():
    A, b, _ = synth.cube(5)
    r = rounding.dikin(A, b, np.zeros(5))
    # every facet is tight, H = 2 I, no eigenvalue exceeds 10 x median: one direction kept, alpha 1
    assert r.info["tight_rows"] == 10 and r.info["n_corrected"] == 1
    assert np.allclose(r.info["alphas"], 1.0) and np.allclose(r.M, np.eye(5))


def test_dikin_eigen_selection_matches_scipy():
    rng = np.random.default_rng(3)
    d = 12
    # a random polytope around 0 with a few very close facets along random normals
    A = rng.standard_normal((60, d))
    b = np.ones(60)
    b[:5] = 1e-3
    r = rounding.dikin(A, b, np.zeros(d), k_directions=4)
    s = b
    norms = np.linalg.norm(A, axis=1)
    delta = s / norms
    tight = delta <= 100 * delta.min()
    Nn = A[tight] / norms[tight, None]
    H = (Nn / delta[tight, None] ** 2).T @ Nn
    ev, V = scipy.linalg.eigh(H)
    med = ev[d // 2]
    want = [j for j in range(d - 1, -1, -1) if ev[j] > 10 * max(med, 1e-10)][:4]
    assert r.info["n_corrected"] == max(1, len(want))
    # P^-1 acts as 1/alpha_j on each selected eigenvector and as 1 on their complement
    for q, j in enumerate(want):
        v = V[:, j]
        assert np.allclose(r.M @ v, v / r.info["alphas"][q], atol=1e-9)
    comp = V[:, [j for j in range(d) if j not in want]]
    assert np.allclose(r.M @ comp, comp, atol=1e-9)


def test_compose_backmap():
    g = synth.genome_shaped(n=80, d=20, density=0.3, seed_T=1, seed_u=2)
    r = rounding.dikin(g["A"], g["b"], g["start"])
    T2, sh2 = r.compose_backmap(g["T"], g["shift"])
    z = np.random.default_rng(0).standard_normal((7, 20)) * 0.01
    assert np.allclose(z @ T2.T + sh2, r.to_y(z) @ g["T"].T + g["shift"])


def test_analytic_centre_and_dikin_full():
    A, b, _ = synth.simplex(6)
    x, s, _ = rounding.analytic_center(A, b, np.array([0.01, 0.3, 0.02, 0.05, 0.1, 0.2]))
    assert np.allclose(x, 1.0 / 7.0, atol=1e-9)
    assert np.allclose(A.T @ (1.0 / s), 0.0, atol=1e-6)  # gradient of the barrier vanishes
    g = synth.genome_shaped(n=300, d=60, density=0.1, seed_T=5, seed_u=6)
    r = rounding.dikin_full(g["A"], g["b"], g["start"])
    w = 1.0 / (g["b"] - g["A"] @ r.c)
    H = (g["A"] * (w * w)[:, None]).T @ g["A"]
    assert np.allclose(r.M.T @ H @ r.M, np.eye(60), atol=1e-8)  # the Dikin ellipsoid is the unit ball in z
    # the unit ball in z lies inside the rounded polytope
    rng = np.random.default_rng(1)
    u = rng.standard_normal((500, 60))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    assert np.all(u @ r.A.T <= r.b + 1e-9)
    with pytest.raises(ValueError):
        rounding.analytic_center(A, b, np.full(6, 0.5))  # outside: sum > 1


def test_covariance_rounding_carries_positions():
    g = synth.genome_shaped(n=100, d=10, density=0.3, seed_T=2, seed_u=3)
    rng = np.random.default_rng(4)
    C = np.cov(rng.standard_normal((200, 10)) * np.arange(1, 11), rowvar=False)
    c = np.full(10, 0.01)
    y0 = rng.standard_normal((3, 10)) * 1e-3
    r = rounding.from_covariance(g["A"], g["b"], C, c, y0)
    assert np.allclose(r.M @ r.M.T, C)
    assert np.allclose(r.to_y(r.z0), y0)
    assert np.allclose(r.z0 @ r.A.T - r.b, y0 @ g["A"].T - g["b"])
