"""The GPU kernels against golden vectors recorded from the reference (GPU).

See tests/test_golden.py for how the fixtures were made.  naja_validate is
held to the reference's validate outputs (float-FFT autocovariance there,
FP64 here: rtol 1e-6), and the step kernel's FP64 tier in cuRAND MRG32k3a
mode to the reference kernel's samples bit for bit.  No reference code runs
here: only the committed fixtures are read.
"""
from pathlib import Path

import numpy as np
import pytest

from naja_b200 import Polytope
from naja_b200 import validate as V

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def _cases(z):
    return sorted({k.split("/")[0] for k in z.files})


def test_validate_kernel_matches_reference(cuda):
    z = np.load(GOLDEN / "validate_ref.npz")
    for name in _cases(z):
        S, k = z[f"{name}/samples"], int(z[f"{name}/n_chains"])
        ess, rh = V.ess_rhat(S, k, layout=0)
        np.testing.assert_allclose(ess.min(axis=1), z[f"{name}/ess"], rtol=1e-6, err_msg=name)
        np.testing.assert_allclose(rh, z[f"{name}/rhat"], rtol=1e-6, err_msg=name)


def test_step_kernel_reproduces_reference_kernel(cuda):
    path = GOLDEN / "chr_ref.npz"
    if not path.exists():
        pytest.skip("chr_ref.npz not recorded")
    z = np.load(path)
    for name in _cases(z):
        nspc, thin, k, resync = (int(v) for v in z[f"{name}/config"])
        P = Polytope(z[f"{name}/A"], z[f"{name}/b"])
        seed = int(z[f"{name}/seed"])
        got = P.run(z[f"{name}/x0"], nspc, thin, k, seed=seed, pair_prob=float(z[f"{name}/pair_prob"]),
                    resync_interval=resync, precision="fp64", rng="mrg", out_dtype="f64")
        assert np.array_equal(got, z[f"{name}/samples"]), (name, np.abs(got - z[f"{name}/samples"]).max())
