"""Seeded synthetic polytopes: the shapes the sampler is measured and tested on.

Genome-scale-shaped polytope (`genome_shaped`): T (n x d) with each entry
nonzero independently with probability `density`, values N(0, 1); bounds
u = 10^U(0, 3) (log-uniform on [1, 1000]) and l = -u; A = [T; -T],
b = [u; u]; start y = 0, shift = 0.  This stands in for a real rounded
genome-scale model (n reactions, d = reduced dimension) such as the
n = 2583 model behind the example verdict line in the reference README;
no model data is shipped with the reference.

Conditioned variants (`conditioned_variants`): extra rows tightening
randomly chosen reaction bounds by a factor f ~ U[0.05, 0.5], with the
reference's extra-row rule (src/cli/prepare/cmd_prepare.cpp:111-156 of
quothbonney/naja): for ub_new < ub - 1e-9 a row T_i with rhs ub_new - shift_i,
for lb_new > lb + 1e-9 a row -T_i with rhs -lb_new + shift_i.

Small polytopes from the reference's GPU tests (tests/test_gpu_*.cu):
cube, simplex, thin slab, random dense.
"""
from __future__ import annotations

import numpy as np


def cube(d: int, lo: float = -1.0, hi: float = 1.0):
    """[lo, hi]^d as A = [I; -I] interleaved per coordinate (test_gpu_sampling_cube_moments.cu:32-37)."""
    A = np.zeros((2 * d, d))
    b = np.zeros(2 * d)
    for i in range(d):
        A[2 * i, i] = 1.0
        A[2 * i + 1, i] = -1.0
        b[2 * i] = hi
        b[2 * i + 1] = -lo
    return A, b, np.full(d, 0.5 * (lo + hi))


def unit_cube_stacked(d: int):
    """[0,1]^d as A = [I; -I], b = [1; 0], start at the centre."""
    A = np.vstack([np.eye(d), -np.eye(d)])
    b = np.concatenate([np.ones(d), np.zeros(d)])
    return A, b, np.full(d, 0.5)


def simplex(d: int):
    """{x >= 0, sum x <= 1} (test_gpu_sampling_feasibility.cu:195-205)."""
    A = np.zeros((d + 1, d))
    b = np.zeros(d + 1)
    for i in range(d):
        A[i, i] = -1.0
    A[d, :] = 1.0
    b[d] = 1.0
    return A, b, np.full(d, 1.0 / (d + 1))


def thin_slab(d: int, eps: float):
    """[-1,1]^d with |sum x| <= eps (test_gpu_sampling_feasibility.cu:207-222)."""
    A = np.zeros((2 * d + 2, d))
    b = np.zeros(2 * d + 2)
    for i in range(d):
        A[2 * i, i] = 1.0
        A[2 * i + 1, i] = -1.0
        b[2 * i] = b[2 * i + 1] = 1.0
    A[2 * d, :] = 1.0
    A[2 * d + 1, :] = -1.0
    b[2 * d] = b[2 * d + 1] = eps
    return A, b, np.zeros(d)


def random_dense(d: int, m: int, seed: int):
    """Gaussian rows with slack 1 at the origin (test_gpu_sampling_feasibility.cu:225-236)."""
    rng = np.random.default_rng(seed)
    return rng.standard_normal((m, d)), np.ones(m), np.zeros(d)


def genome_shaped(n: int = 2600, d: int = 700, density: float = 0.08, seed_T: int = 0, seed_u: int = 1):
    """Returns dict(A, b, T, shift, u, start) of the genome-shaped polytope."""
    rT = np.random.default_rng(seed_T)
    mask = rT.random((n, d)) < density
    T = np.where(mask, rT.standard_normal((n, d)), 0.0)
    # every column must touch at least one row, or the polytope is unbounded
    empty = np.where(~mask.any(axis=0))[0]
    for j in empty:
        T[rT.integers(n), j] = rT.standard_normal()
    ru = np.random.default_rng(seed_u)
    u = 10.0 ** ru.uniform(0.0, 3.0, size=n)
    A = np.vstack([T, -T])
    b = np.concatenate([u, u])
    return {"A": A, "b": b, "T": T, "shift": np.zeros(n), "u": u, "l": -u, "start": np.zeros(d)}


def conditioned_variants(base: dict, n_models: int, max_reactions: int = 100, fmin: float = 0.05,
                         fmax: float = 0.5, seed: int = 2):
    """Extra-row variants of `base`; returns a list of dicts with extra_A, extra_b, u_new, l_new."""
    rng = np.random.default_rng(seed)
    T, shift, u, l = base["T"], base["shift"], base["u"], base["l"]
    n = T.shape[0]
    out = []
    for _ in range(n_models):
        r = int(rng.integers(0, max_reactions + 1))
        idx = rng.choice(n, size=r, replace=False) if r else np.zeros(0, dtype=int)
        f = rng.uniform(fmin, fmax, size=r)
        u_new, l_new = u.copy(), l.copy()
        u_new[idx] = u[idx] * f
        l_new[idx] = l[idx] * f
        rows, rhs = [], []
        for i in range(n):
            if u_new[i] < u[i] - 1e-9:
                rows.append(T[i])
                rhs.append(u_new[i] - shift[i])
            if l_new[i] > l[i] + 1e-9:
                rows.append(-T[i])
                rhs.append(-l_new[i] + shift[i])
        eA = np.array(rows).reshape(-1, T.shape[1])
        out.append({"extra_A": eA, "extra_b": np.array(rhs), "u_new": u_new, "l_new": l_new,
                    "tightened": idx})
    return out
