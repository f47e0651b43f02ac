"""Affine roundings of a polytope {y : A y <= b} for CHR.

A rounding is an invertible affine map y = M z + c.  CHR then samples z in
{z : (A M) z <= b - A c}, which is uniform exactly when y is uniform on the
original polytope (the Jacobian of an affine map is constant), and the
samples are mapped back with the same backmap kernel: y = M z + c, or
directly to flux space with T' = T M, shift' = T c + shift.

`dikin` restates the Dikin-ellipsoid preconditioner of quothbonney/naja
(src/rounding/dikin_precondition.cpp:36-183, defaults .h:35-42), which the
reference never wires into sampling:
  1. facet distances delta_i = (b_i - a_i x_c) / ||a_i||, unit normals n_i
  2. tight set: 0 < delta_i <= tight_factor * min positive delta
  3. barrier Hessian H = sum_tight n_i n_i^T / delta_i^2
  4. the top eigenvectors of H (at most k) whose eigenvalue exceeds
     10 * max(median eigenvalue, 1e-10); at least one
  5. target chord = median positive chord along the first min(d, 50)
     coordinate axes (when not given); alpha_j = clip(target / chord_j, 1,
     alpha_max), or min(alpha_max, 10) for a dead direction (chord < 1e-15)
  6. P = I + V (diag(alpha) - I) V^T, P^-1 = I + V (diag(1/alpha) - I) V^T
  7. A_new = A P^-1, b_new = b - A x_c, z0 = 0
so y = P^-1 z + x_c (M = P^-1, c = x_c).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Rounding:
    """y = M z + c, with the transformed polytope and start point."""

    M: np.ndarray          # d x d
    c: np.ndarray          # d
    A: np.ndarray          # A M
    b: np.ndarray          # b - A c
    z0: np.ndarray         # start point in z
    info: dict

    def compose_backmap(self, T, shift):
        """T' = T M, shift' = T c + shift: flux space straight from z."""
        return T @ self.M, T @ self.c + shift

    def to_y(self, Z):
        """Rows z -> rows y (host helper; the GPU path uses the backmap kernel)."""
        return Z @ self.M.T + self.c


def identity(A, b, x0) -> Rounding:
    d = A.shape[1]
    return Rounding(np.eye(d), np.asarray(x0, float).copy(), np.asarray(A, float), np.asarray(b, float) - A @ x0,
                    np.zeros(d), {"method": "identity"})


def chord_along(A, b, x, v) -> float:
    """Length of the chord through x along v in {A y <= b} (dikin_precondition.cpp:13-32)."""
    slack = b - A @ x
    Av = A @ v
    t_min, t_max = -np.inf, np.inf
    nz = np.abs(Av) >= 1e-15
    pos = nz & (Av > 0)
    neg = nz & (Av < 0)
    if pos.any():
        t_max = float(np.min(slack[pos] / Av[pos]))
    if neg.any():
        t_min = float(np.max(slack[neg] / Av[neg]))
    if t_max <= t_min:
        return 0.0
    return t_max - t_min


def dikin(A, b, x_c, k_directions: int = 64, tight_factor: float = 100.0, target_chord: float = 0.0,
          alpha_max: float = 1000.0) -> Rounding:
    A = np.asarray(A, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    x_c = np.asarray(x_c, dtype=np.float64)
    m, d = A.shape
    if m == 0 or d == 0:
        raise ValueError("dikin_precondition: empty polytope")
    slack = b - A @ x_c
    norms = np.linalg.norm(A, axis=1)
    ok = norms >= 1e-15
    deltas = np.full(m, np.inf)
    deltas[ok] = slack[ok] / norms[ok]
    N = np.zeros_like(A)
    N[ok] = A[ok] / norms[ok, None]
    finite_pos = (deltas > 0) & np.isfinite(deltas)
    if not finite_pos.any():
        r = identity(A, b, x_c)
        r.info.update(method="dikin", n_corrected=0)
        return r
    min_delta = float(deltas[finite_pos].min())
    tight = np.where((deltas > 0) & (deltas <= tight_factor * min_delta))[0]
    if tight.size == 0:
        r = identity(A, b, x_c)
        r.info.update(method="dikin", n_corrected=0)
        return r
    w = 1.0 / deltas[tight] ** 2
    Nt = N[tight]
    H = (Nt * w[:, None]).T @ Nt
    evals, evecs = np.linalg.eigh(H)  # ascending
    k = min(k_directions, d)
    median = evals[d // 2]
    actual = 0
    for j in range(d - 1, -1, -1):
        if actual >= k:
            break
        if evals[j] > 10.0 * max(median, 1e-10):
            actual += 1
        else:
            break
    actual = max(actual, 1)
    V = evecs[:, ::-1][:, :actual]
    if target_chord <= 0.0:
        chords = []
        for j in range(min(d, 50)):
            e = np.zeros(d)
            e[j] = 1.0
            ch = chord_along(A, b, x_c, e)
            if ch > 0:
                chords.append(ch)
        target_chord = float(np.sort(chords)[len(chords) // 2]) if chords else 1.0
    alphas = np.empty(actual)
    for j in range(actual):
        ch = chord_along(A, b, x_c, V[:, j])
        alphas[j] = min(alpha_max, 10.0) if ch < 1e-15 else min(max(target_chord / ch, 1.0), alpha_max)
    P_inv = np.eye(d) + (V * (1.0 / alphas - 1.0)) @ V.T
    return Rounding(P_inv, x_c.copy(), A @ P_inv, slack.copy(), np.zeros(d),
                    {"method": "dikin", "n_corrected": int(actual), "tight_rows": int(tight.size),
                     "target_chord": target_chord, "alphas": alphas})


def diag_lowrank(log_diag, U, c, A, b) -> Rounding:
    """Rounding from a diagonal-plus-low-rank factor L = diag(exp(log_diag)) + U U^T-free form.

    M = diag(exp(log_diag)) (I + U V^T)-style factors are not needed: the
    factor is taken as L = diag(exp(log_diag)) + U W with W = U^T (so L is
    symmetric positive definite when exp(log_diag) > 0), y = L z + c."""
    D = np.exp(np.asarray(log_diag, dtype=np.float64))
    U = np.asarray(U, dtype=np.float64)
    M = np.diag(D) + U @ U.T
    c = np.asarray(c, dtype=np.float64)
    return Rounding(M, c.copy(), A @ M, b - A @ c, np.zeros(A.shape[1]), {"method": "diag+lowrank",
                                                                           "rank": int(U.shape[1])})


def analytic_center(A, b, x0=None, tol: float = 1e-9, max_iter: int = 200):
    """Analytic centre of {y : A y <= b}: argmin of -sum log(b - A y), by
    damped Newton from a strictly feasible x0 (default 0).  Returns (x_c,
    slack at x_c, Newton iterations)."""
    A = np.asarray(A, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    x = np.zeros(A.shape[1]) if x0 is None else np.asarray(x0, dtype=np.float64).copy()
    s = b - A @ x
    if not np.all(s > 0):
        raise ValueError("analytic_center: the start point is not strictly feasible")
    it = 0
    for it in range(1, max_iter + 1):
        w = 1.0 / s
        g = A.T @ w
        H = (A * (w * w)[:, None]).T @ A
        L = np.linalg.cholesky(H)
        dx = -np.linalg.solve(L.T, np.linalg.solve(L, g))
        lam2 = float(-g @ dx)  # Newton decrement squared
        if lam2 <= tol * tol:
            break
        Adx = A @ dx
        t = 1.0 / (1.0 + np.sqrt(lam2))  # damped step, stays inside the Dikin ellipsoid
        pos = Adx > 0
        if pos.any():
            t = min(t, 0.99 * float(np.min(s[pos] / Adx[pos])))
        x = x + t * dx
        s = b - A @ x
    return x, s, it


def _sym_sqrt(S, inverse=False):
    ev, V = np.linalg.eigh(S)
    ev = np.maximum(ev, ev.max() * 1e-14)
    return (V * (ev ** (-0.5 if inverse else 0.5))) @ V.T


def dikin_full(A, b, x0=None, device=None) -> Rounding:
    """Whole-ellipsoid Dikin rounding: y = H^{-1/2} z + x_c with x_c the
    analytic centre and H = A^T S^-2 A its barrier Hessian (S = diag(b - A
    x_c)).  The Dikin ellipsoid {(y - x_c)^T H (y - x_c) <= 1}, which lies
    inside the polytope, becomes the unit ball in z, along every direction at
    once -- where dikin() stretches at most k_directions eigen-directions by a
    clipped factor (the reference's preconditioner).

    device: a CUDA device (index or torch.device) computes the same steps in
    FP64 on the GPU (cuBLAS / cuSOLVER through torch): the same rounding up
    to rounding differences in the last digits, in a fraction of the host's
    time for genome-scale A."""
    if device is not None:
        return _dikin_full_gpu(A, b, x0, device)
    A = np.asarray(A, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    t0 = _now()
    x_c, s, iters = analytic_center(A, b, x0)
    w = 1.0 / s
    H = (A * (w * w)[:, None]).T @ A
    M = _sym_sqrt(H, inverse=True)
    return Rounding(M, x_c, A @ M, s.copy(), np.zeros(A.shape[1]),
                    {"method": "dikin_full", "newton_iterations": iters, "seconds": _now() - t0})


def _dikin_full_gpu(A, b, x0, device, tol: float = 1e-9, max_iter: int = 200) -> Rounding:
    """dikin_full's steps (analytic_center's damped Newton, the Hessian, its
    inverse square root by eigendecomposition, A M) in FP64 on `device`."""
    import torch

    dev = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
    t0 = _now()
    At = torch.as_tensor(np.asarray(A, dtype=np.float64), device=dev)
    bt = torch.as_tensor(np.asarray(b, dtype=np.float64).reshape(-1), device=dev)
    d = At.shape[1]
    x = torch.zeros(d, dtype=torch.float64, device=dev) if x0 is None else \
        torch.as_tensor(np.asarray(x0, dtype=np.float64).reshape(-1), device=dev).clone()
    s = bt - At @ x
    if not bool((s > 0).all()):
        raise ValueError("analytic_center: the start point is not strictly feasible")
    it = 0
    for it in range(1, max_iter + 1):
        w = 1.0 / s
        g = At.T @ w
        Aw = At * w[:, None]
        L = torch.linalg.cholesky(Aw.T @ Aw)
        dx = -torch.cholesky_solve(g[:, None], L)[:, 0]
        lam2 = float(-(g @ dx))
        if lam2 <= tol * tol:
            break
        Adx = At @ dx
        t = 1.0 / (1.0 + lam2 ** 0.5)
        pos = Adx > 0
        if bool(pos.any()):
            t = min(t, 0.99 * float((s[pos] / Adx[pos]).min()))
        x = x + t * dx
        s = bt - At @ x
    Aw = At * (1.0 / s)[:, None]
    ev, V = torch.linalg.eigh(Aw.T @ Aw)
    ev = torch.clamp(ev, min=float(ev.max()) * 1e-14)
    M = (V * ev.rsqrt()) @ V.T
    AM = At @ M
    # the device copies stay in info["dev"] for callers that keep working on the GPU
    out = Rounding(M.cpu().numpy(), x.cpu().numpy(), AM.cpu().numpy(), s.cpu().numpy(), np.zeros(d),
                   {"method": "dikin_full", "newton_iterations": it, "device": str(dev),
                    "dev": {"M": M, "c": x, "A": AM, "b": s}})
    out.info["seconds"] = _now() - t0
    return out


def from_covariance(A, b, cov, c, y0=None) -> Rounding:
    """Rounding to the isotropic position of a sample: y = Sigma^{1/2} z + c,
    with Sigma a sample covariance of the uniform distribution on the
    polytope (or a factor's estimate of it).  y0 (rows of current positions,
    optional) are carried into z so that running chains continue."""
    A = np.asarray(A, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    M = _sym_sqrt(np.asarray(cov, dtype=np.float64))
    c = np.asarray(c, dtype=np.float64)
    z0 = np.zeros(A.shape[1]) if y0 is None else np.linalg.solve(M, (np.atleast_2d(y0) - c).T).T
    return Rounding(M, c.copy(), A @ M, b - A @ c, z0, {"method": "covariance"})


def _now():
    import time

    return time.perf_counter()
