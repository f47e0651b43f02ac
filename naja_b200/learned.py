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


def factor_targets(samples, rank, torch):
    """Batched factor_target on the GPU: samples (V, N, dim) -> (V, dim + dim*rank) float64 numpy."""
    Y = samples.to(torch.float64)
    Y = Y - Y.mean(dim=1, keepdim=True)
    cov = Y.transpose(1, 2) @ Y / (Y.shape[1] - 1)
    w, V = torch.linalg.eigh(cov)
    w = w.clamp_min(1e-18).flip(-1)
    V = V.flip(-1)
    s = w.sqrt()
    floor = s[:, rank:rank + 1] if rank < s.shape[1] else torch.zeros_like(s[:, :1])
    U = V[:, :, :rank] * (s[:, :rank] - floor).clamp_min(0.0).sqrt()[:, None, :]
    idx = U.abs().argmax(dim=1, keepdim=True)
    sign = torch.where(torch.gather(U, 1, idx) < 0, -1.0, 1.0)
    U = U * sign
    S_diag = (V * V * s[:, None, :]).sum(-1)
    diag = (S_diag - (U * U).sum(-1)).clamp_min(1e-12)
    return torch.cat([diag.log(), U.reshape(U.shape[0], -1)], dim=1).cpu().numpy()


def _sample(polys, Ms, cs, nchains, nspc, thinning, kw, torch, shape=None):
    """Batched CHR over polytopes given in the rounded space; returns (y samples per model as
    float32 CUDA tensors, seconds of sampling + map back)."""
    from .batch import Batch, Shape
    from .sampler import backmap

    d = polys[0].d
    dev = torch.device("cuda")
    B = Batch(polys)
    X = [torch.zeros((nchains, d), dtype=torch.float64, device=dev) for _ in polys]
    outs = [torch.empty((nspc * nchains, d), dtype=torch.float32, device=dev) for _ in polys]
    ys = [torch.empty_like(o) for o in outs]
    shape = shape or Shape(512, 3, 1, 0)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    B.run(X, outs, nspc, thinning, nchains, shape=shape, **kw)
    for k, o in enumerate(outs):
        if Ms[k] is None:
            ys[k] = o
        else:
            backmap(Ms[k], cs[k], o, mode="fp64", out=ys[k])
    e1.record()
    torch.cuda.synchronize()
    B.check()
    return ys, e0.elapsed_time(e1) / 1e3


def _diagnose(ys, nchains):
    from . import validate as V

    res = []
    for y in ys:
        ess, rh = V.ess_rhat(y, nchains, layout=1)
        res.append((float(V.chain_ess(ess).min()), float(rh.max())))
    return res


def run_experiment(*, n=2600, d=700, n_train=256, n_test=16, nchains=8, nspc_train=500, nspc_test=1000,
                   thinning=116, pair_prob=0.3, rank=32, hidden=(512, 512), epochs=60, batch=64, lr=1e-3,
                   resync=2048, seed=0, train_chains=None, log=None):
    """Plain vs Dikin-rounded vs learned-rounded CHR on held-out conditioned
    variants of the genome-shaped polytope.  Returns a dict of results."""
    import time

    import torch

    from . import rounding, synth
    from .sampler import Polytope

    say = log or (lambda *a: None)
    base = synth.genome_shaped(n=n, d=d, density=0.08, seed_T=0, seed_u=1)
    variants = synth.conditioned_variants(base, n_train + n_test, max_reactions=100, seed=seed + 11)
    A_list = [np.vstack([base["A"], v["extra_A"]]) for v in variants]
    b_list = [np.concatenate([base["b"], v["extra_b"]]) for v in variants]
    F = np.stack([features(v, base) for v in variants]).astype(np.float32)
    kw = dict(seed=seed, pair_prob=pair_prob, resync_interval=resync)

    # 1. plain CHR on the training variants -> covariance factor targets
    t0 = time.perf_counter()
    polys = [Polytope(A_list[k], b_list[k]) for k in range(n_train)]
    ys, t_train_samp = _sample(polys, [None] * n_train, [None] * n_train, train_chains or nchains, nspc_train,
                               thinning, kw, torch)
    T = factor_targets(torch.stack(ys), rank, torch)
    del ys, polys
    mu, sd = T.mean(axis=0), T.std(axis=0) + 1e-6
    Tn = ((T - mu) / sd).astype(np.float32)
    # log ratios lie in [log fmin, 0] (most are 0): one global scale, no
    # per-feature standardisation, which would blow up reactions that are
    # rarely tightened in the training set
    Fn = (F / 3.0).astype(np.float32)
    t_targets = time.perf_counter() - t0
    say(f"targets: {n_train} variants, {t_train_samp:.2f} s sampling, {t_targets:.2f} s total")

    # 2. train on the project's kernels
    # 90 / 10 split of the training variants; the weights of the epoch with
    # the lowest validation error are kept (early stopping)
    net = RoundingNet((n, *hidden, d + d * rank), seed=seed, lr=lr)
    rng = np.random.default_rng(seed)
    n_val = max(1, n_train // 10)
    fit_idx, val_idx = np.arange(n_train - n_val), np.arange(n_train - n_val, n_train)
    t0 = time.perf_counter()
    first = None
    best = (float(np.mean(Tn[val_idx] ** 2)), -1, net.snapshot())  # the mean predictor (zero output)
    curve = []
    for ep in range(epochs):
        perm = rng.permutation(fit_idx)
        for i in range(0, len(perm), batch):
            idx = perm[i:i + batch]
            loss = net.train_step(Fn[idx], Tn[idx])
            first = loss if first is None else first
        val = float(np.mean((net.predict(Fn[val_idx]).cpu().numpy() - Tn[val_idx]) ** 2))
        curve.append(val)
        if val < best[0]:
            best = (val, ep, net.snapshot())
    net.restore(best[2])
    torch.cuda.synchronize()
    t_fit = time.perf_counter() - t0
    pred_train = net.predict(Fn[fit_idx]).cpu().numpy()
    train_mse = float(np.mean((pred_train - Tn[fit_idx]) ** 2))
    say(f"training: {epochs} epochs in {t_fit:.2f} s, loss {first:.4f} -> {loss:.4f}, best validation "
        f"{best[0]:.4f} at epoch {best[1]}")

    # 3. held-out variants: plain, Dikin, learned
    test = list(range(n_train, n_train + n_test))
    out = {"train": {"variants": n_train, "epochs": epochs, "seconds": t_fit, "first_loss": first,
                     "last_loss": loss, "train_mse_std_units": train_mse, "best_epoch": best[1],
                     "validation_mse_std_units": best[0], "validation_curve": curve,
                     "target_sampling_seconds": t_train_samp},
           "test_variants": n_test, "methods": {}}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pred = net.predict(Fn[test]).cpu().numpy() * sd + mu
    t_inf = time.perf_counter() - t0
    # the held-out variants' own covariance factors (for the regression error only)
    polys = [Polytope(A_list[k], b_list[k]) for k in test]
    ys, t_plain = _sample(polys, [None] * n_test, [None] * n_test, nchains, nspc_test, thinning, kw, torch)
    diag_plain = _diagnose(ys, nchains)
    T_test = factor_targets(torch.stack(ys), rank, torch)
    out["test_mse_std_units"] = float(np.mean(((pred - T_test) / sd) ** 2))
    out["test_mse_mean_predictor"] = float(np.mean(((mu - T_test) / sd) ** 2))
    del ys
    methods = {"plain": (None, t_plain, diag_plain)}
    for name in ("dikin", "learned"):
        Ms, cs, zp = [], [], []
        t_round = 0.0
        for j, k in enumerate(test):
            t1 = time.perf_counter()
            if name == "dikin":
                r = rounding.dikin(A_list[k], b_list[k], np.zeros(d))
            else:
                logd, U = unpack(pred[j], d, rank)
                r = rounding.diag_lowrank(logd, U, np.zeros(d), A_list[k], b_list[k])
            t_round += time.perf_counter() - t1
            Ms.append(r.M)
            cs.append(r.c)
            zp.append(Polytope(r.A, r.b))
        ys, t_s = _sample(zp, Ms, cs, nchains, nspc_test, thinning, kw, torch)
        methods[name] = (t_round + (t_inf if name == "learned" else 0.0), t_s, _diagnose(ys, nchains))
        del ys, zp
    for name, (t_round, t_s, diag) in methods.items():
        per = t_s / n_test  # sampling seconds per variant in the batched run
        ess = np.array([e for e, _ in diag])
        rh = np.array([r for _, r in diag])
        out["methods"][name] = {"sampling_seconds": t_s, "rounding_seconds": t_round or 0.0,
                                "min_ess_per_variant": ess.tolist(), "rhat_max": float(rh.max()),
                                "rhat_gate_1_01": bool(rh.max() < 1.01),
                                "min_ess_per_s_median": float(np.median(ess) / per),
                                "min_ess_per_s_min": float(ess.min() / per)}
    m = out["methods"]
    out["learned_vs_plain"] = m["learned"]["min_ess_per_s_median"] / m["plain"]["min_ess_per_s_median"]
    out["learned_vs_dikin"] = m["learned"]["min_ess_per_s_median"] / m["dikin"]["min_ess_per_s_median"]
    return out
