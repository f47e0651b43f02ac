"""Device-side ESS / split-R-hat (naja_validate) against the CPU oracle (GPU).

Tolerances: ESS per (dim, chain) within 1e-4 relative of the oracle's exact
FP64 autocovariance (the kernel multiplies in FP32 and sums in FP64; Geyer's
stopping lag is the same unless a pair sum sits within round-off of zero,
which the cases here avoid by construction); R-hat within 1e-9.
"""
import numpy as np
import pytest

import oracle.oracle as O
from naja_b200 import validate as nv

pytestmark = pytest.mark.gpu


def _series(N, dim, seed, rho):
    rng = np.random.default_rng(seed)
    x = np.empty((N, dim))
    x[0] = rng.standard_normal(dim)
    e = rng.standard_normal((N, dim))
    for t in range(1, N):
        x[t] = rho * x[t - 1] + np.sqrt(1 - rho ** 2) * e[t]
    return (x * rng.uniform(0.1, 10, dim) + rng.standard_normal(dim)).astype(np.float32)


@pytest.mark.parametrize("layout", [0, 1])
@pytest.mark.parametrize("nchains", [1, 4, 7])
def test_ess_rhat_match_oracle(cuda, layout, nchains):
    S = _series(700 * nchains, 9, seed=nchains, rho=0.7)
    ess, rhat = nv.ess_rhat(S, nchains, layout=layout)
    ess_o = O.ess(S, nchains, layout=layout)
    rhat_o = O.split_rhat(S, nchains, layout=layout)
    assert np.allclose(ess, ess_o, rtol=1e-4, atol=0)
    assert np.allclose(rhat, rhat_o, rtol=1e-9, atol=0)


def test_constant_and_short_series(cuda):
    S = np.ones((40, 3), dtype=np.float32)
    ess, rhat = nv.ess_rhat(S, 4, layout=1)
    assert np.all(ess == 1.0) and np.all(rhat == 1.0)


def test_reference_summary_rules(cuda):
    S = _series(2000, 12, seed=3, rho=0.5)
    ess, rhat = nv.ess_rhat(S, 4, layout=0)
    s = nv.summary(ess, rhat)
    per_dim = np.min(ess, axis=1)
    assert s["ess"]["min"] == pytest.approx(float(per_dim.min()), rel=1e-6)
    assert s["status"] in ("OK", "WARN", "FAIL")
    assert s["rhat"]["above_1_1"] == int(np.sum(rhat > 1.1))
    assert np.allclose(nv.chain_ess(ess), ess.sum(axis=1))


def test_rejects_bad_shapes(cuda):
    from naja_b200._lib import NajaError

    with pytest.raises(NajaError):
        nv.ess_rhat(np.zeros((10, 2), np.float32), 3)
