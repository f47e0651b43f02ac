"""The rounding network's CPU oracle checked on its own (CPU).

The backward pass of oracle/mlp_oracle.py is checked against central finite
differences of its FP64 forward (no BF16 rounding), and the BF16 rounding
against exactly representable values and ties.  tests/test_gpu_mlp.py then
holds the GPU kernels to this oracle.
"""
import numpy as np

from oracle import mlp_oracle as MO


def _net(rng, dims):
    return [(rng.standard_normal((b, a)) / np.sqrt(a), rng.standard_normal(b) * 0.1) for a, b in zip(dims[:-1], dims[1:])]


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(3)
    dims = (7, 9, 6, 5)
    layers = _net(rng, dims)
    X = rng.standard_normal((4, dims[0]))
    T = rng.standard_normal((4, dims[-1]))
    w = rng.uniform(0.5, 2.0, dims[-1])
    _, grads = MO.loss_and_grads(layers, X, T, w, bf16_on=False)
    h = 1e-6
    for li, (W, b) in enumerate(layers):
        for (i, j) in [(0, 0), (W.shape[0] - 1, W.shape[1] - 1), (1, 2)]:
            Wp, Wm = W.copy(), W.copy()
            Wp[i, j] += h
            Wm[i, j] -= h
            lp = MO.loss_and_grads([(Wp, b) if k == li else layers[k] for k in range(len(layers))], X, T, w,
                                   bf16_on=False)[0]
            lm = MO.loss_and_grads([(Wm, b) if k == li else layers[k] for k in range(len(layers))], X, T, w,
                                   bf16_on=False)[0]
            assert abs((lp - lm) / (2 * h) - grads[li][0][i, j]) < 1e-6 * max(1.0, abs(grads[li][0][i, j]))
        bp, bm = b.copy(), b.copy()
        bp[0] += h
        bm[0] -= h
        lp = MO.loss_and_grads([(W, bp) if k == li else layers[k] for k in range(len(layers))], X, T, w, bf16_on=False)[0]
        lm = MO.loss_and_grads([(W, bm) if k == li else layers[k] for k in range(len(layers))], X, T, w, bf16_on=False)[0]
        assert abs((lp - lm) / (2 * h) - grads[li][1][0]) < 1e-6 * max(1.0, abs(grads[li][1][0]))


def test_bf16_rounding():
    assert MO.bf16(1.0) == 1.0 and MO.bf16(-3.5) == -3.5
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: ties to even -> 1
    assert MO.bf16(1.0 + 2.0 ** -8) == 1.0
    assert MO.bf16(1.0 + 3 * 2.0 ** -8) == 1.0 + 2.0 ** -6
    x = np.random.default_rng(0).standard_normal(1000)
    assert np.all(np.abs(MO.bf16(x) - x) <= np.abs(x) * 2.0 ** -8)
