"""Learned rounding: a small MLP from bound ratios to an affine rounding.

A conditioned model (the base polytope with some reactions' bounds
tightened, the extra-row rule of src/cli/prepare/cmd_prepare.cpp:111-156 in
quothbonney/naja) is described by x = log(u_new / u_base) over the base
model's reactions.  The network maps x to a diagonal-plus-low-rank factor

    M = diag(exp(d)) + U U^T        (d in R^dim, U in R^(dim x rank))

and CHR samples z in {z : (A M) z <= b - A c}; y = M z + c is uniform on
the original polytope because the map is affine (naja_b200.rounding).  The
targets are factors of sample covariances that plain CHR itself produced
(`factor_targets`), and the Dikin preconditioner (rounding.dikin) remains
the fallback and the comparison.

Every step of training and inference runs on the project's kernels
(include/naja_mlp.h): BF16 operands with FP32 accumulation on the tensor
cores for the nine GEMMs of a training step, fused bias + GELU epilogues
that also emit the transposed activations the weight gradients need, the
GELU backward, the weighted MSE gradient, bias gradients and Adam on FP32
master weights.  PyTorch only provides device memory and the stream.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from ._lib import GemmEpilogue, check, load


def _pad8(n: int) -> int:
    return (n + 7) // 8 * 8


def _p(t) -> int:
    return 0 if t is None else int(t.data_ptr())


@dataclass
class _Layer:
    n_in: int
    n_out: int
    W: object          # FP32 master (n_out, pad8(n_in))
    b: object          # FP32 (n_out,)
    mW: object
    vW: object
    mb: object
    vb: object
    W_bf: object       # BF16 (n_out, pad8(n_in))
    W_bf_t: object     # BF16 (n_in, pad8(n_out))
    gW: object = None
    gb: object = None


@dataclass
class _Buffers:
    B: int
    X: object = None
    X_bf: object = None
    X_bf_t: object = None
    pre: list = field(default_factory=list)      # FP32 (B, pad8(out)) per hidden layer
    act: list = field(default_factory=list)      # BF16 (B, pad8(out))
    act_t: list = field(default_factory=list)    # BF16 (out, pad8(B))
    out: object = None
    target: object = None
    g: list = field(default_factory=list)        # FP32 gradient w.r.t. each layer's pre-activation
    g_bf: list = field(default_factory=list)
    g_bf_t: list = field(default_factory=list)
    dact: list = field(default_factory=list)
    loss: object = None


class RoundingNet:
    """dims = (n_in, hidden..., n_out); GELU between layers, linear output."""

    def __init__(self, dims, *, seed=0, device="cuda", lr=1e-3, betas=(0.9, 0.999), eps=1e-8):
        import torch

        self.torch = torch
        self.dims = tuple(int(v) for v in dims)
        self.device = torch.device(device)
        self.stream = 0
        self.lr, self.betas, self.eps = lr, betas, eps
        self.step_count = 0
        self.lib = load()
        g = np.random.default_rng(seed)
        self.layers = []
        for li, (a, b) in enumerate(zip(self.dims[:-1], self.dims[1:])):
            scale = np.sqrt(2.0 / a) if li < len(self.dims) - 2 else np.sqrt(0.1 / a)
            w = np.zeros((b, _pad8(a)), np.float32)
            w[:, :a] = g.standard_normal((b, a)) * scale
            self.layers.append(self._make_layer(a, b, w, np.zeros(b, np.float32)))
        self._bufs = {}

    # ------------------------------------------------------------ memory
    def _make_layer(self, a, b, w, bias):
        t = self.torch
        dev = self.device
        W = t.from_numpy(w).to(dev)
        L = _Layer(a, b, W, t.from_numpy(bias).to(dev), t.zeros_like(W), t.zeros_like(W),
                   t.zeros(b, device=dev), t.zeros(b, device=dev),
                   t.zeros((b, _pad8(a)), dtype=t.bfloat16, device=dev),
                   t.zeros((a, _pad8(b)), dtype=t.bfloat16, device=dev))
        check(self.lib.naja_cast_bf16(b, a, _p(W), W.shape[1], _p(L.W_bf), L.W_bf.shape[1], _p(L.W_bf_t),
                                      L.W_bf_t.shape[1], self.stream))
        return L

    def _buffers(self, B):
        if B in self._bufs:
            return self._bufs[B]
        t, dev = self.torch, self.device
        bf = t.bfloat16
        z = _Buffers(B)
        n_in = self.dims[0]
        z.X = t.zeros((B, _pad8(n_in)), device=dev)
        z.X_bf = t.zeros((B, _pad8(n_in)), dtype=bf, device=dev)
        z.X_bf_t = t.zeros((n_in, _pad8(B)), dtype=bf, device=dev)
        for L in self.layers:
            o = L.n_out
            z.pre.append(t.zeros((B, _pad8(o)), device=dev))
            z.act.append(t.zeros((B, _pad8(o)), dtype=bf, device=dev))
            z.act_t.append(t.zeros((o, _pad8(B)), dtype=bf, device=dev))
            z.g.append(t.zeros((B, _pad8(o)), device=dev))
            z.g_bf.append(t.zeros((B, _pad8(o)), dtype=bf, device=dev))
            z.g_bf_t.append(t.zeros((o, _pad8(B)), dtype=bf, device=dev))
            z.dact.append(t.zeros((B, _pad8(o)), device=dev))
            if L.gW is None:
                L.gW = t.zeros_like(L.W)
                L.gb = t.zeros(o, device=dev)
        z.out = z.pre[-1]
        z.target = t.zeros_like(z.out)
        z.loss = t.zeros(1, dtype=t.float64, device=dev)
        self._bufs[B] = z
        return z

    # ------------------------------------------------------------ kernels
    def _gemm(self, M, N, K, A, lda, Bm, ldb, *, bias=None, c=None, ldc=0, acc=0, act=None, ld_act=0,
              act_t=None, ld_act_t=0, gelu=0):
        e = GemmEpilogue(_p(bias), _p(c), ldc, acc, _p(act), ld_act, _p(act_t), ld_act_t, gelu)
        check(self.lib.naja_gemm_bf16(M, N, K, _p(A), lda, _p(Bm), ldb, C.byref(e), self.stream))

    def _forward(self, z):
        nl = len(self.layers)
        A, lda = z.X_bf, z.X_bf.shape[1]
        for li, L in enumerate(self.layers):
            last = li == nl - 1
            self._gemm(z.B, L.n_out, L.n_in, A, lda, L.W_bf, L.W_bf.shape[1], bias=L.b, c=z.pre[li],
                       ldc=z.pre[li].shape[1], act=None if last else z.act[li], ld_act=z.act[li].shape[1],
                       act_t=None if last else z.act_t[li], ld_act_t=z.act_t[li].shape[1], gelu=0 if last else 1)
            A, lda = z.act[li], z.act[li].shape[1]

    def _load_inputs(self, z, X):
        t = self.torch
        n_in = self.dims[0]
        z.X[:, :n_in].copy_(t.as_tensor(X, dtype=t.float32, device=self.device))
        check(self.lib.naja_cast_bf16(z.B, n_in, _p(z.X), z.X.shape[1], _p(z.X_bf), z.X_bf.shape[1], _p(z.X_bf_t),
                                      z.X_bf_t.shape[1], self.stream))

    def predict(self, X):
        """X (B, n_in) -> outputs (B, n_out) as a float32 CUDA tensor."""
        X = np.asarray(X, np.float32) if not hasattr(X, "data_ptr") else X
        z = self._buffers(int(X.shape[0]))
        self._load_inputs(z, X)
        self._forward(z)
        check(self.lib.naja_mlp_check(self.stream))
        return z.out[:, : self.dims[-1]].clone()

    def gradients(self, X, T, w=None):
        """Forward + backward; returns loss and leaves gradients in the layers (no update)."""
        t = self.torch
        B = int(X.shape[0])
        z = self._buffers(B)
        self._load_inputs(z, X)
        n_out = self.dims[-1]
        z.target[:, :n_out].copy_(t.as_tensor(T, dtype=t.float32, device=self.device))
        self._forward(z)
        z.loss.zero_()
        nl = len(self.layers)
        wt = None if w is None else t.as_tensor(w, dtype=t.float32, device=self.device).contiguous()
        ld = z.out.shape[1]
        check(self.lib.naja_mse_grad(B, n_out, _p(z.out), _p(z.target), ld, _p(wt), _p(z.loss), _p(z.g[-1]),
                                     _p(z.g_bf[-1]), z.g_bf[-1].shape[1], _p(z.g_bf_t[-1]), z.g_bf_t[-1].shape[1],
                                     self.stream))
        for li in range(nl - 1, -1, -1):
            L = self.layers[li]
            check(self.lib.naja_col_sum(B, L.n_out, _p(z.g[li]), z.g[li].shape[1], _p(L.gb), self.stream))
            # dW = g^T act_prev: A = g^T (n_out x B), B-operand = act_prev^T (n_in x B)
            prev_t = z.X_bf_t if li == 0 else z.act_t[li - 1]
            self._gemm(L.n_out, L.n_in, B, z.g_bf_t[li], z.g_bf_t[li].shape[1], prev_t, prev_t.shape[1], c=L.gW,
                       ldc=L.gW.shape[1])
            if li > 0:
                # dact_prev = g W: A = g (B x n_out), B-operand = W^T (n_in x n_out)
                P = self.layers[li - 1]
                self._gemm(B, L.n_in, L.n_out, z.g_bf[li], z.g_bf[li].shape[1], L.W_bf_t, L.W_bf_t.shape[1],
                           c=z.dact[li - 1], ldc=z.dact[li - 1].shape[1])
                check(self.lib.naja_gelu_backward(B, P.n_out, _p(z.dact[li - 1]), _p(z.pre[li - 1]),
                                                  z.pre[li - 1].shape[1], _p(z.g[li - 1]), _p(z.g_bf[li - 1]),
                                                  z.g_bf[li - 1].shape[1], _p(z.g_bf_t[li - 1]),
                                                  z.g_bf_t[li - 1].shape[1], self.stream))
        check(self.lib.naja_mlp_check(self.stream))
        return float(z.loss.item())

    def apply_gradients(self):
        self.step_count += 1
        b1, b2 = self.betas
        for L in self.layers:
            check(self.lib.naja_adam(L.n_out, L.n_in, _p(L.W), _p(L.gW), _p(L.mW), _p(L.vW), L.W.shape[1], self.lr, b1,
                                     b2, self.eps, self.step_count, _p(L.W_bf), L.W_bf.shape[1], _p(L.W_bf_t),
                                     L.W_bf_t.shape[1], self.stream))
            check(self.lib.naja_adam(1, L.n_out, _p(L.b), _p(L.gb), _p(L.mb), _p(L.vb), L.n_out, self.lr, b1, b2,
                                     self.eps, self.step_count, None, 0, None, 0, self.stream))

    def train_step(self, X, T, w=None) -> float:
        loss = self.gradients(X, T, w)
        self.apply_gradients()
        return loss

    # ------------------------------------------------------------ state
    def snapshot(self):
        """Copies of the FP32 master weights and biases (device tensors)."""
        return [(L.W.clone(), L.b.clone()) for L in self.layers]

    def restore(self, snap):
        """Loads a snapshot and refreshes the BF16 copies the kernels read."""
        for L, (W, b) in zip(self.layers, snap):
            L.W.copy_(W)
            L.b.copy_(b)
            check(self.lib.naja_cast_bf16(L.n_out, L.n_in, _p(L.W), L.W.shape[1], _p(L.W_bf), L.W_bf.shape[1],
                                          _p(L.W_bf_t), L.W_bf_t.shape[1], self.stream))

    def weights(self):
        """[(W (n_out, n_in) float32, b (n_out,))] as numpy arrays."""
        return [(L.W[:, : L.n_in].cpu().numpy(), L.b.cpu().numpy()) for L in self.layers]

    def weight_grads(self):
        return [(L.gW[:, : L.n_in].cpu().numpy(), L.gb.cpu().numpy()) for L in self.layers]


# ---------------------------------------------------------------- targets
def factor_target(cov, rank):
    """(log d, U) of M = diag(exp(d)) + U U^T approximating the symmetric
    square root S = cov^(1/2): U spans S's top `rank` eigen-directions with
    weights sqrt(s_i - s_floor) (s_floor = the largest remaining eigenvalue
    of S), d is the log of S - U U^T's diagonal.  Each column of U is signed
    so that its largest-magnitude entry is positive."""
    w, V = np.linalg.eigh(np.asarray(cov, np.float64))
    w = np.clip(w, 1e-18, None)
    s = np.sqrt(w)[::-1]
    V = V[:, ::-1]
    floor = s[rank] if rank < len(s) else 0.0
    U = V[:, :rank] * np.sqrt(np.clip(s[:rank] - floor, 0.0, None))
    idx = np.argmax(np.abs(U), axis=0)
    U = U * np.where(U[idx, np.arange(U.shape[1])] < 0, -1.0, 1.0)
    S = (V * s) @ V.T
    diag = np.clip(np.diag(S) - np.sum(U * U, axis=1), 1e-12, None)
    return np.log(diag), U


def pack(logd, U):
    return np.concatenate([logd, U.reshape(-1)])


def unpack(vec, dim, rank):
    v = np.asarray(vec, np.float64)
    return v[:dim], v[dim:].reshape(dim, rank)


# ------------------------------------------------------------ experiment
def features(variant, base):
    """log(u_new / u_base) over the base model's reactions."""
    return np.log(np.asarray(variant["u_new"], np.float64) / np.asarray(base["u"], np.float64))


def factor_targets(samples, rank, torch, inverse=False):
    """Batched factor_target on the GPU: samples (V, N, dim) -> (V, dim + dim*rank) float64 numpy.

    inverse=True factors G = Sigma^-1/2 instead of Sigma^1/2, with G's
    eigenvalues raised to at least their median: the rank-r part then holds
    the directions in which the samples are thinnest (the ones a rounding
    must stretch), and no direction is shrunk below the median scale (a
    short run underestimates the spread of slowly mixing directions, which
    must not be mistaken for thin ones)."""
    Y = samples.to(torch.float64)
    Y = Y - Y.mean(dim=1, keepdim=True)
    cov = Y.transpose(1, 2) @ Y / (Y.shape[1] - 1)
    w, V = torch.linalg.eigh(cov)
    if inverse:
        g = w.clamp_min(1e-18).rsqrt()
        g = torch.maximum(g, g.median(dim=-1, keepdim=True).values)
        w = g * g  # so that s = sqrt(w) = g below
    w = w.clamp_min(1e-18)
    order = torch.argsort(w, dim=-1, descending=True)
    w = torch.gather(w, -1, order)
    V = torch.gather(V, -1, order[:, None, :].expand_as(V))
    s = w.sqrt()
    floor = s[:, rank:rank + 1] if rank < s.shape[1] else torch.zeros_like(s[:, :1])
    U = V[:, :, :rank] * (s[:, :rank] - floor).clamp_min(0.0).sqrt()[:, None, :]
    idx = U.abs().argmax(dim=1, keepdim=True)
    sign = torch.where(torch.gather(U, 1, idx) < 0, -1.0, 1.0)
    U = U * sign
    S_diag = (V * V * s[:, None, :]).sum(-1)
    diag = (S_diag - (U * U).sum(-1)).clamp_min(1e-12)
    return torch.cat([diag.log(), U.reshape(U.shape[0], -1)], dim=1).cpu().numpy()


def _rounded_rows(A0M, extra_A, M0, torch):
    """[A_base M0; extra_A M0] on the device (FP64)."""
    if extra_A.shape[0] == 0:
        return A0M
    E = torch.from_numpy(np.ascontiguousarray(extra_A)).to(A0M.device) @ M0
    return torch.cat([A0M, E], dim=0)


def _targets(base, variants, idx, R0, nchains, nspc, thinning, kw, rank, group, torch, say):
    """Plain CHR (no per-variant rounding) of each variant in the base
    model's rounded coordinates w (y = M0 w + c0), batched `group` variants
    per launch; targets are diag + rank-r factors of the w-sample
    covariances."""
    from .batch import Batch, Shape
    from .sampler import Polytope

    dev = torch.device("cuda")
    M0 = torch.from_numpy(R0.M).to(dev)
    A0M = torch.from_numpy(base["A"]).to(dev) @ M0
    d = M0.shape[0]
    out, t_samp = [], 0.0
    for g0 in range(0, len(idx), group):
        ks = idx[g0:g0 + group]
        polys = []
        for k in ks:
            v = variants[k]
            A = np.vstack([base["A"], v["extra_A"]])
            b = np.concatenate([base["b"], v["extra_b"]])
            polys.append(Polytope(_rounded_rows(A0M, v["extra_A"], M0, torch), b - A @ R0.c))
        B = Batch(polys)
        X = [torch.zeros((nchains, d), dtype=torch.float64, device=dev) for _ in polys]
        W = [torch.empty((nspc * nchains, d), dtype=torch.float32, device=dev) for _ in polys]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        B.run(X, W, nspc, thinning, nchains, shape=Shape(256, 3, 1, 0, 0), **kw)
        e1.record()
        torch.cuda.synchronize()
        B.check()
        t_samp += e0.elapsed_time(e1) / 1e3
        out.append(factor_targets(torch.stack(W), rank, torch, inverse=True))
        del W, polys, B
        say(f"targets: {min(g0 + group, len(idx))}/{len(idx)} variants")
    return np.concatenate(out), t_samp


def run_experiment(*, n=2600, d=700, n_train=1024, n_test=16, nchains=8, nspc_train=1500, thinning=116,
                   pair_prob=0.3, rank=32, hidden=(512, 512), epochs=60, batch=64, lr=1e-3, resync=2048, seed=0,
                   gate_budget_s=45.0, chunk_nspc=4000, group=256, log=None):
    """Learned rounding on conditioned variants of the genome-shaped polytope.

    The base model is rounded once by its whole Dikin ellipsoid, y = M0 w +
    c0.  A conditioned variant tightens some reactions, which squeezes its
    polytope along their rows; the network predicts, from the variant's
    bound ratios, a diagonal-plus-low-rank stretch G = diag(exp(d)) + U U^T
    in the base coordinates (U: the variant's thinnest directions), and the
    variant is sampled in z with y = M0 G^-1 z + c0 -- affine, so the uniform
    target is unchanged.  Targets: factors of the inverse square root of the
    w-space sample covariances that plain CHR (no per-variant rounding)
    produces for the training variants (factor_targets, inverse=True).  Held-out variants are then
    sampled until split-R-hat < 1.01 (batched, one launch per chunk) with:
    plain CHR, the reference's Dikin preconditioner per variant, the
    whole-ellipsoid Dikin rounding per variant, the base rounding alone, and
    the learned rounding; each method's seconds per variant include
    computing its rounding (network inference for the learned one), and
    training time is reported separately."""
    import time

    import torch

    from . import gate, rounding, synth

    say = log or (lambda *a: None)
    base = synth.genome_shaped(n=n, d=d, density=0.08, seed_T=0, seed_u=1)
    variants = synth.conditioned_variants(base, n_train + n_test, max_reactions=100, seed=seed + 11)
    F = np.stack([features(v, base) for v in variants]).astype(np.float32)
    kw = dict(seed=seed, pair_prob=pair_prob, resync_interval=resync)
    t0 = time.perf_counter()
    R0 = rounding.dikin_full(base["A"], base["b"], base["start"])
    t_base = time.perf_counter() - t0

    # 1. targets from plain CHR in the base coordinates
    t0 = time.perf_counter()
    T, t_train_samp = _targets(base, variants, list(range(n_train)), R0, nchains, nspc_train, thinning, kw, rank,
                               group, torch, say)
    t_targets = time.perf_counter() - t0
    mu, sd = T.mean(axis=0), T.std(axis=0) + 1e-6
    Tn = ((T - mu) / sd).astype(np.float32)
    # log ratios lie in [log fmin, 0] (most are 0): one global scale
    Fn = (F / 3.0).astype(np.float32)

    # 2. train on the project's kernels; 90 / 10 split, early stopping on validation
    net = RoundingNet((n, *hidden, d + d * rank), seed=seed, lr=lr)
    rng = np.random.default_rng(seed)
    n_val = max(1, n_train // 10)
    fit_idx, val_idx = np.arange(n_train - n_val), np.arange(n_train - n_val, n_train)
    t0 = time.perf_counter()
    first = loss = None
    best = (float(np.mean(Tn[val_idx] ** 2)), -1, net.snapshot())  # the mean predictor (zero output)
    for ep in range(epochs):
        perm = rng.permutation(fit_idx)
        for i in range(0, len(perm), batch):
            loss = net.train_step(Fn[perm[i:i + batch]], Tn[perm[i:i + batch]])
            first = loss if first is None else first
        val = float(np.mean((net.predict(Fn[val_idx]).cpu().numpy() - Tn[val_idx]) ** 2))
        if val < best[0]:
            best = (val, ep, net.snapshot())
    net.restore(best[2])
    torch.cuda.synchronize()
    t_fit = time.perf_counter() - t0
    say(f"training: {epochs} epochs in {t_fit:.2f} s, best validation {best[0]:.4f} at epoch {best[1]}")

    # 3. held-out variants
    test = list(range(n_train, n_train + n_test))
    models = [(np.vstack([base["A"], variants[k]["extra_A"]]), np.concatenate([base["b"], variants[k]["extra_b"]]))
              for k in test]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pred = net.predict(Fn[test]).cpu().numpy() * sd + mu
    t_inf = (time.perf_counter() - t0) / n_test
    T_test, _ = _targets(base, variants, test, R0, nchains, nspc_train, thinning, kw, rank, group, torch, say)
    out = {"train": {"variants": n_train, "epochs": epochs, "seconds": t_fit, "first_loss": first, "last_loss": loss,
                     "best_epoch": best[1], "validation_mse_std_units": best[0],
                     "target_sampling_seconds": t_train_samp, "targets_seconds": t_targets,
                     "base_rounding_seconds": t_base},
           "test_variants": n_test,
           "test_mse_std_units": float(np.mean(((pred - T_test) / sd) ** 2)),
           "test_mse_mean_predictor": float(np.mean(((mu - T_test) / sd) ** 2)),
           "methods": {}}

    def compose(A, b, Fm):
        """Rounding y = M0 Fm z + c0 of (A, b)."""
        M = R0.M @ Fm
        return rounding.Rounding(M, R0.c.copy(), A @ M, b - A @ R0.c, np.zeros(d), {"method": "composed"})

    for name in ("plain", "dikin", "dikin_full", "base", "learned"):
        rs, t_round = [], 0.0
        for j, (A, b) in enumerate(models):
            t1 = time.perf_counter()
            if name == "plain":
                r = rounding.identity(A, b, np.zeros(d))
            elif name == "dikin":
                r = rounding.dikin(A, b, np.zeros(d))
            elif name == "dikin_full":
                r = rounding.dikin_full(A, b, np.zeros(d))
            elif name == "base":
                r = compose(A, b, np.eye(d))
            else:
                logd, U = unpack(pred[j], d, rank)
                r = compose(A, b, np.linalg.inv(np.diag(np.exp(logd)) + U @ U.T))
            t_round += time.perf_counter() - t1
            rs.append(r)
        extra = t_round / n_test + (t_inf if name == "learned" else 0.0)
        res = gate.batch_to_gate(models, rs, nchains=nchains, thinning=thinning, chunk_nspc=chunk_nspc,
                                 pair_prob=pair_prob, resync_interval=resync, seed=seed, budget_s=gate_budget_s,
                                 extra_seconds=extra)
        res["rounding_seconds_per_variant"] = extra
        out["methods"][name] = res
        say(f"{name}: {res['passed']}/{n_test} passed, median min-ESS/s {res['min_ess_per_s_median']:.2f}")
    m = out["methods"]
    for other in ("plain", "dikin", "dikin_full", "base"):
        out[f"learned_vs_{other}"] = m["learned"]["min_ess_per_s_median"] / max(m[other]["min_ess_per_s_median"],
                                                                               1e-12)
    return out
