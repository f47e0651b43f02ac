"""What the trained rounding network gains over sampling without it (GPU).

A family of conditioned models where rounding matters and the map from
bound ratios to rounding is learnable: rotated boxes {y : |R^T y| <= s} in
d = 8 with half-widths s = (30, 15, 8, 4, 2, 1, 1, 1) * f, f in [0.6, 1] per
axis drawn per variant (the features are log f).  CHR along coordinate
axes mixes slowly in such an elongated, rotated box.  The network
(8 -> 64 -> 64 -> 8 + 8*5, trained on the project's kernels) is fitted to
diagonal-plus-rank-5 factors of plain-CHR sample covariances of 48 training
variants, then predicts the rounding of 8 held-out variants.  At the same
number of CHR steps, learned-rounded CHR must give at least twice the
min-ESS of plain CHR and at least 1.5 times that of CHR rounded by the
reference's Dikin preconditioner (median over held-out variants; the
rounded polytopes have the same rows and columns, so a step costs the same
and the min-ESS ratio is the min-ESS/s ratio), every sample must satisfy
the original constraints, and the network must predict the held-out
targets better than their training mean.
"""
import numpy as np
import pytest

from naja_b200 import Polytope, rounding
from naja_b200 import validate as V
from naja_b200.learned import RoundingNet, factor_target, pack, unpack

pytestmark = pytest.mark.gpu

D, RANK = 8, 5
S_BASE = np.array([30.0, 15.0, 8.0, 4.0, 2.0, 1.0, 1.0, 1.0])


def _family(n, seed):
    rng = np.random.default_rng(seed)
    R, _ = np.linalg.qr(np.random.default_rng(99).standard_normal((D, D)))
    out = []
    for _ in range(n):
        f = rng.uniform(0.6, 1.0, D)
        s = S_BASE * f
        A = np.vstack([R.T, -R.T])
        b = np.concatenate([s, s])
        out.append((np.log(f), A, b))
    return out


def _min_ess(y, nchains):
    ess, _ = V.ess_rhat(np.ascontiguousarray(y, dtype=np.float32), nchains, layout=1)
    return float(V.chain_ess(ess).min())


def test_learned_rounding_beats_plain_and_dikin(cuda):
    train, test = _family(48, 1), _family(8, 2)
    # targets: factors of plain-CHR sample covariances
    T = []
    for k, (_, A, b) in enumerate(train):
        Y = Polytope(A, b).run(np.zeros(D), 1500, 40, 16, seed=k, pair_prob=0.0, out_dtype="f64")
        logd, U = factor_target(np.cov(Y.T), RANK)
        T.append(pack(logd, U))
    T = np.array(T)
    mu, sd = T.mean(axis=0), T.std(axis=0) + 1e-6
    F = np.array([f for f, _, _ in train], np.float32)
    Tn = ((T - mu) / sd).astype(np.float32)
    net = RoundingNet((D, 64, 64, D + D * RANK), seed=3, lr=3e-3)
    for _ in range(400):
        net.train_step(F, Tn)
    Ft = np.array([f for f, _, _ in test], np.float32)
    pred = net.predict(Ft).cpu().numpy() * sd + mu

    gains, gains_dikin, err_net, err_mean = [], [], [], []
    for j, (_, A, b) in enumerate(test):
        P = Polytope(A, b)
        Y0 = P.run(np.zeros(D), 400, 8, 8, seed=100 + j, out_dtype="f64")
        logd, U = unpack(pred[j], D, RANK)
        r = rounding.diag_lowrank(logd, U, np.zeros(D), A, b)
        Z = Polytope(r.A, r.b).run(r.z0, 400, 8, 8, seed=100 + j, out_dtype="f64")
        Y1 = r.to_y(Z)
        assert (Y1 @ A.T - b).max() <= 1e-6 * np.abs(b).max()
        gains.append(_min_ess(Y1, 8) / _min_ess(Y0, 8))
        rd = rounding.dikin(A, b, np.zeros(D))
        Y2 = rd.to_y(Polytope(rd.A, rd.b).run(rd.z0, 400, 8, 8, seed=100 + j, out_dtype="f64"))
        assert (Y2 @ A.T - b).max() <= 1e-6 * np.abs(b).max()
        gains_dikin.append(_min_ess(Y1, 8) / _min_ess(Y2, 8))
        # how well the held-out rounding is predicted, against the long-run target
        Yl = P.run(np.zeros(D), 1500, 40, 16, seed=200 + j, out_dtype="f64")
        tgt = pack(*factor_target(np.cov(Yl.T), RANK))
        err_net.append(np.mean(((pred[j] - tgt) / sd) ** 2))
        err_mean.append(np.mean(((mu - tgt) / sd) ** 2))
    print(f"learned / plain min-ESS per held-out variant: {np.round(gains, 2).tolist()}; "
          f"learned / Dikin: {np.round(gains_dikin, 2).tolist()}; "
          f"prediction MSE {np.mean(err_net):.3f} vs mean predictor {np.mean(err_mean):.3f}")
    assert np.median(gains) >= 2.0, gains
    assert np.median(gains_dikin) >= 1.5, gains_dikin
    assert np.mean(err_net) < np.mean(err_mean), (np.mean(err_net), np.mean(err_mean))
