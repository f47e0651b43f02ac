"""Backmap V = T y + shift against an FP64 numpy reference (GPU).

FP64 mode: the reference's arithmetic up to summation order (1e-12).
Tensor-core modes, error normalised by sum_k |T_ik y_k| + |shift_i| per
element (the scale an FP32 product can resolve):
  BF16X3 (bf16 hi + lo, three products): <= 2^-15
  TF32X3 (tf32 hi + lo, three products): <= 2^-17
(at K = 700 the FP32 accumulation itself reaches a few 2^-24 * sqrt(K)).
"""
import numpy as np
import pytest

from naja_b200 import backmap, synth

pytestmark = pytest.mark.gpu

TOL = {"bf16x3": 2.0 ** -15, "tf32x3": 2.0 ** -17}


def _case(N, n, d, seed):
    rng = np.random.default_rng(seed)
    T = np.where(rng.random((n, d)) < 0.3, rng.standard_normal((n, d)), 0.0)
    Y = (rng.standard_normal((N, d)) * 10 ** rng.uniform(-2, 2, (1, d))).astype(np.float32)
    shift = rng.standard_normal(n)
    ref = Y.astype(np.float64) @ T.T + shift
    scale = np.abs(Y.astype(np.float64)) @ np.abs(T).T + np.abs(shift)
    return T, Y, shift, ref, scale


@pytest.mark.parametrize("shape", [(1000, 300, 70), (777, 260, 70), (129, 257, 65), (128, 256, 64), (5, 3, 2)])
def test_fp64_mode(cuda, shape):
    T, Y, shift, ref, scale = _case(*shape, seed=1)
    V = backmap(T, shift, Y, mode="fp64", out_dtype=np.float64)
    assert np.max(np.abs(V - ref) / scale) < 1e-12


@pytest.mark.parametrize("mode", ["bf16x3", "tf32x3"])
@pytest.mark.parametrize("shape", [(1000, 300, 70), (777, 260, 70), (129, 257, 65), (128, 256, 64), (5, 3, 2),
                                   (3000, 2600, 700)])
def test_tensor_core_modes(cuda, mode, shape):
    T, Y, shift, ref, scale = _case(*shape, seed=2)
    V = backmap(T, shift, Y, mode=mode, out_dtype=np.float64)
    err = np.abs(V - ref) / scale
    assert np.max(err) <= TOL[mode], (mode, shape, float(np.max(err)))
    V32 = backmap(T, shift, Y, mode=mode, out_dtype=np.float32)
    assert np.array_equal(V32, V.astype(np.float32))


def test_tensor_core_genome_shaped(cuda):
    g = synth.genome_shaped(n=2600, d=700)
    rng = np.random.default_rng(3)
    Y = (rng.standard_normal((4096, 700)) * 50).astype(np.float32)
    ref = Y.astype(np.float64) @ g["T"].T
    scale = np.abs(Y.astype(np.float64)) @ np.abs(g["T"]).T + 1e-300
    for mode in ("bf16x3", "tf32x3"):
        V = backmap(g["T"], g["shift"], Y, mode=mode, out_dtype=np.float64)
        assert np.max(np.abs(V - ref) / scale) <= TOL[mode]
