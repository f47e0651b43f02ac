"""Batched multi-model kernel (GPU): every model of a batch reproduces its
standalone naja_chr_run bit for bit, for every launch shape of the dense and
the compressed-column batch kernels; a captured CUDA graph replays the same
result."""
import numpy as np
import pytest

from naja_b200 import Polytope, synth
from naja_b200.batch import Batch, Shape

pytestmark = pytest.mark.gpu


def _models(nmodels=5, n=260, d=70):
    base = synth.genome_shaped(n=n, d=d, density=0.08, seed_T=3, seed_u=4)
    out = [(base["A"], base["b"])]
    for v in synth.conditioned_variants(base, nmodels - 1, max_reactions=25, seed=9):
        out.append((np.vstack([base["A"], v["extra_A"]]), np.concatenate([base["b"], v["extra_b"]])))
    return out, base["start"]


SHAPES = [Shape(256, 3, 1, 0), Shape(128, 2, 1, 2), Shape(512, 0, 1, 1), Shape(256, 4, 0, 1), Shape(512, 8, 0, 0),
          Shape(128, 0, 1, 3),
          # compressed-column kernel
          Shape(64, 3, 1, 0, sparse=1), Shape(128, 4, 1, 2, sparse=1), Shape(256, 8, 1, 0, sparse=1)]


@pytest.mark.parametrize("shape", SHAPES, ids=str)
def test_batched_equals_standalone(cuda, shape):
    import torch

    polys, start = _models()
    ms = {A.shape[0] for A, _ in polys}
    assert len(ms) > 1  # uneven row counts
    P = [Polytope(A, b) for A, b in polys]
    B = Batch(P)
    if B.occupancy(shape) == 0:
        pytest.skip("shape does not fit")
    nspc, thin, nch, seed = 25, 7, 3, 42
    X = [torch.from_numpy(np.broadcast_to(start, (nch, len(start))).copy()).cuda() for _ in P]
    outs = [torch.empty((nspc * nch, len(start)), dtype=torch.float64, device=cuda) for _ in P]
    B.run(X, outs, nspc, thin, nch, shape=shape, seed=seed, seed_stride=5, pair_prob=0.3, resync_interval=16,
          out_dtype="f64")
    B.check()
    for k, p in enumerate(P):
        ref = p.run(start, nspc, thin, nch, seed=42 + 5 * k, pair_prob=0.3, resync_interval=16, out_dtype="f64")
        assert np.array_equal(outs[k].cpu().numpy(), ref), k


def test_graph_replay(cuda):
    import torch

    polys, start = _models(4)
    P = [Polytope(A, b) for A, b in polys]
    B = Batch(P)
    nspc, thin, nch = 20, 5, 2
    X = [torch.from_numpy(np.broadcast_to(start, (nch, len(start))).copy()).cuda() for _ in P]
    outs = [torch.empty((nspc * nch, len(start)), dtype=torch.float32, device=cuda) for _ in P]
    B.run(X, outs, nspc, thin, nch, shape=Shape(256, 3, 1, 0), seed=3, pair_prob=0.3)
    direct = [o.clone() for o in outs]
    for o in outs:
        o.zero_()
    g = B.capture(X, outs, nspc, thin, nch, shape=Shape(128, 4, 1, 0, sparse=1), seed=3, pair_prob=0.3)
    for _ in range(2):
        g.launch()
    g.check()
    for a, b in zip(direct, outs):
        assert torch.equal(a, b)
    g.close()


def test_batch_rejects_mixed_dimensions(cuda):
    import torch

    from naja_b200._lib import InvalidArgument

    A1, b1, x1 = synth.cube(5)
    A2, b2, x2 = synth.cube(6)
    B = Batch([Polytope(A1, b1), Polytope(A2, b2)])
    X = [torch.zeros((2, 5), dtype=torch.float64, device=cuda), torch.zeros((2, 6), dtype=torch.float64, device=cuda)]
    outs = [torch.empty((20, 5), device=cuda), torch.empty((20, 6), device=cuda)]
    with pytest.raises(InvalidArgument):
        B.run(X, outs, 10, 1, 2)


@pytest.mark.parametrize("shape", [Shape(256, 3, 1, 0), Shape(128, 4, 1, 0, sparse=1)], ids=str)
def test_batched_continuation_with_final_states(cuda, shape):
    """Two batched launches, the second continuing from the first's X_finals
    at the step offset where it stopped, give the samples of one launch of
    twice the length (the chunk spans whole resync periods)."""
    import torch

    polys, start = _models()
    P = [Polytope(A, b) for A, b in polys]
    B = Batch(P)
    nspc, thin, nch, K = 16, 6, 3, 32  # 96 steps per chunk = 3 resync periods
    d = len(start)
    kw = dict(seed=7, seed_stride=3, pair_prob=0.3, resync_interval=K, out_dtype="f64")
    X = [torch.from_numpy(np.broadcast_to(start, (nch, d)).copy()).cuda() for _ in P]
    whole = [torch.empty((2 * nspc * nch, d), dtype=torch.float64, device=cuda) for _ in P]
    B.run(X, whole, 2 * nspc, thin, nch, shape=shape, **kw)
    Xf = [torch.empty_like(x) for x in X]
    first = [torch.empty((nspc * nch, d), dtype=torch.float64, device=cuda) for _ in P]
    second = [torch.empty_like(f) for f in first]
    B.run(X, first, nspc, thin, nch, shape=shape, X_finals=Xf, **kw)
    B.run(Xf, second, nspc, thin, nch, shape=shape, step_offset=nspc * thin, **kw)
    B.check()
    for k in range(len(P)):
        assert torch.equal(torch.cat([first[k], second[k]]), whole[k]), k
