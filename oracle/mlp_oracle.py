"""TEST INFRASTRUCTURE ONLY -- CPU oracle of the rounding network's kernels.

Only tests/ may import it.  A numpy restatement of what the GPU kernels of
include/naja_mlp.h compute for one training step of the MLP in
naja_b200/learned.py (the network has no counterpart in quothbonney/naja):

  forward   pre_l = bf16(a_{l-1}) bf16(W_l)^T + b_l, a_l = bf16(GELU(pre_l))
            for hidden layers (GELU in the erf form), out = pre_L;
  loss      sum_n w_n (out - t)^2 / B;
  backward  g_L = 2 w (out - t) / B; db_l = colsum(g_l);
            dW_l = bf16(g_l)^T bf16(a_{l-1});
            g_{l-1} = (bf16(g_l) bf16(W_l)) * GELU'(pre_{l-1});
  adam      m = b1 m + (1-b1) g; v = b2 v + (1-b2) g^2;
            W -= lr (m / (1 - b1^t)) / (sqrt(v / (1 - b2^t)) + eps).

Products of BF16 values are exact in FP64, so the oracle's GEMMs differ from
the tensor cores' FP32 accumulation only by accumulation rounding.  With
`bf16=False` every rounding is dropped and the functions are plain FP64
(used for the finite-difference check of the backward pass itself).
"""
from __future__ import annotations

import math

import numpy as np


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


_erf = np.vectorize(math.erf)


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + _erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def _r(x, on):
    return bf16(x) if on else np.asarray(x, np.float64)


def forward(layers, X, *, bf16_on=True):
    """layers: [(W (out, in), b (out,))]; returns (out, pres, acts)."""
    a = _r(X, bf16_on)
    pres, acts = [], [a]
    for li, (W, b) in enumerate(layers):
        pre = a @ _r(W, bf16_on).T + np.asarray(b, np.float64)
        pres.append(pre)
        if li < len(layers) - 1:
            a = _r(gelu(pre), bf16_on)
            acts.append(a)
    return pres[-1], pres, acts


def loss_and_grads(layers, X, T, w=None, *, bf16_on=True):
    out, pres, acts = forward(layers, X, bf16_on=bf16_on)
    B = out.shape[0]
    wv = np.ones(out.shape[1]) if w is None else np.asarray(w, np.float64)
    diff = out - np.asarray(T, np.float64)
    loss = float(np.sum(wv * diff * diff) / B)
    g = 2.0 * wv * diff / B
    grads = [None] * len(layers)
    for li in range(len(layers) - 1, -1, -1):
        W, _ = layers[li]
        gb = _r(g, bf16_on)
        grads[li] = (gb.T @ acts[li], g.sum(axis=0))
        if li > 0:
            g = (gb @ _r(W, bf16_on)) * gelu_grad(pres[li - 1])
    return loss, grads


def adam(W, g, m, v, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    W = W - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return W, m, v
