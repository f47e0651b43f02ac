"""The rounding network's kernels against the CPU oracle (GPU).

* naja_gemm_bf16 against an FP64 product of the same BF16 operands, on
  shapes that are not multiples of the 128 x 128 tile or the 64-value K
  slice, with every epilogue output (tolerance: FP32 accumulation, rtol
  1e-5 of the row's absolute sum);
* one training step of a small network (forward outputs, loss, every
  weight and bias gradient) against oracle/mlp_oracle.py with the same BF16
  rounding points: relative Frobenius error below 2e-2 (a BF16 rounding that
  tips the other way on either side moves single terms by 2^-8);
* the Adam update against the oracle (rtol 1e-5);
* training on a fixed regression task lowers the loss.
"""
import numpy as np
import pytest

from oracle import mlp_oracle as MO

pytestmark = pytest.mark.gpu


def _bf(t, shape, torch, pad=True):
    rows, cols = shape
    ld = (cols + 7) // 8 * 8
    buf = torch.zeros((rows, ld), dtype=torch.bfloat16, device="cuda")
    buf[:, :cols] = torch.as_tensor(np.asarray(t, np.float32)).to("cuda").to(torch.bfloat16)
    return buf, ld


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (200, 70, 150), (37, 300, 520), (256, 23, 8)])
def test_gemm_matches_fp64(cuda, M, N, K):
    import torch

    from naja_b200._lib import GemmEpilogue, check, load
    import ctypes as C

    rng = np.random.default_rng(M + N + K)
    A = MO.bf16(rng.standard_normal((M, K)))
    B = MO.bf16(rng.standard_normal((N, K)))
    bias = rng.standard_normal(N).astype(np.float32)
    Ab, lda = _bf(A, (M, K), torch)
    Bb, ldb = _bf(B, (N, K), torch)
    Cf = torch.full((M, N + 3), 0.25, device="cuda")
    act = torch.zeros((M, (N + 7) // 8 * 8), dtype=torch.bfloat16, device="cuda")
    act_t = torch.zeros((N, (M + 7) // 8 * 8), dtype=torch.bfloat16, device="cuda")
    bt = torch.as_tensor(bias, device="cuda")
    lib = load()
    e = GemmEpilogue(bt.data_ptr(), Cf.data_ptr(), N + 3, 1, act.data_ptr(), act.shape[1], act_t.data_ptr(),
                     act_t.shape[1], 1)
    check(lib.naja_gemm_bf16(M, N, K, Ab.data_ptr(), lda, Bb.data_ptr(), ldb, C.byref(e), None))
    check(lib.naja_mlp_check(None))
    ref = A @ B.T + bias
    tol = 1e-5 * (np.abs(A) @ np.abs(B).T + 1.0)
    got = Cf[:, :N].cpu().numpy().astype(np.float64) - 0.25
    assert np.all(np.abs(got - ref) <= tol)
    assert np.all(Cf[:, N:].cpu().numpy() == 0.25)  # nothing written past N
    g = MO.gelu(got)
    a_got = act[:, :N].float().cpu().numpy()
    assert np.allclose(a_got, MO.bf16(g), rtol=2 ** -7, atol=1e-6)
    assert np.array_equal(act_t[:, :M].float().cpu().numpy(), a_got.T)


def _small_problem(seed=0):
    rng = np.random.default_rng(seed)
    dims = (40, 64, 48, 36)
    X = rng.standard_normal((20, dims[0])).astype(np.float32)
    T = rng.standard_normal((20, dims[-1])).astype(np.float32)
    w = rng.uniform(0.5, 2.0, dims[-1]).astype(np.float32)
    return dims, X, T, w


def _rel(a, b):
    return np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30)


def test_training_step_matches_oracle(cuda):
    from naja_b200.learned import RoundingNet

    dims, X, T, w = _small_problem()
    net = RoundingNet(dims, seed=4)
    layers = [(W.astype(np.float64), b.astype(np.float64)) for W, b in net.weights()]
    out = net.predict(X).cpu().numpy()
    ref_out, _, _ = MO.forward(layers, X)
    assert _rel(out, ref_out) < 2e-2
    loss = net.gradients(X, T, w)
    ref_loss, ref_grads = MO.loss_and_grads(layers, X, T, w)
    assert abs(loss - ref_loss) <= 2e-2 * ref_loss
    for (gW, gb), (rW, rb) in zip(net.weight_grads(), ref_grads):
        assert _rel(gW, rW) < 2e-2
        assert _rel(gb, rb) < 2e-2


def test_adam_matches_oracle(cuda):
    from naja_b200.learned import RoundingNet

    dims, X, T, w = _small_problem(1)
    net = RoundingNet(dims, seed=5, lr=1e-2)
    before = [W.astype(np.float64) for W, _ in net.weights()]
    net.gradients(X, T, w)
    grads = [gW.astype(np.float64) for gW, _ in net.weight_grads()]
    net.apply_gradients()
    after = [W.astype(np.float64) for W, _ in net.weights()]
    for W0, g, W1 in zip(before, grads, after):
        ref, _, _ = MO.adam(W0, g, np.zeros_like(W0), np.zeros_like(W0), 1, lr=1e-2)
        assert np.allclose(W1, ref, rtol=1e-5, atol=1e-7)


def test_training_lowers_the_loss(cuda):
    from naja_b200.learned import RoundingNet

    rng = np.random.default_rng(2)
    dims = (30, 64, 64, 20)
    X = rng.standard_normal((128, dims[0])).astype(np.float32)
    M = rng.standard_normal((dims[0], dims[-1])) / np.sqrt(dims[0])
    T = np.tanh(X @ M).astype(np.float32)
    net = RoundingNet(dims, seed=1, lr=3e-3)
    first = net.train_step(X, T)
    for _ in range(200):
        last = net.train_step(X, T)
    assert last < 0.2 * first
