"""The CPU oracle against golden vectors recorded from the reference itself.

tests/golden/make_golden.py records them:
  validate_ref.npz -- the reference's compute_ess / compute_split_rhat
      (src/validate/mcmc.cpp with its vendored float kissfft, compiled
      unmodified on the CPU) on seeded sample matrices;
  chr_ref.npz      -- the reference's CoordinateHitAndRun kernel
      (src/gpu/chr.cu, compiled unmodified for sm_100a) on small polytopes,
      with the cuRAND MRG32k3a uniform tape its chains consumed.
The validate oracle evaluates autocovariances as exact FP64 sums where the
reference uses a float FFT, so ESS agrees to float rounding (rtol 1e-6);
split-R-hat sums in FP64 on both sides (rtol 1e-6).  CHR samples must be
identical: the FP64 oracle replays the same uniforms through the same IEEE
operations.  The GPU kernels are held to the same fixtures in
tests/test_gpu_golden.py.
"""
from pathlib import Path

import numpy as np
import pytest

import oracle.oracle as O
from naja_b200 import validate as V

GOLDEN = Path(__file__).resolve().parent / "golden"


def _cases(z):
    return sorted({k.split("/")[0] for k in z.files})


@pytest.fixture(scope="module")
def vz():
    return np.load(GOLDEN / "validate_ref.npz")


def test_validate_oracle_matches_reference(vz):
    for name in _cases(vz):
        S, k = vz[f"{name}/samples"], int(vz[f"{name}/n_chains"])
        ess = O.ess(S, k, layout=0)
        rh = O.split_rhat(S, k, layout=0)
        np.testing.assert_allclose(ess.min(axis=1), vz[f"{name}/ess"], rtol=1e-6, err_msg=name)
        np.testing.assert_allclose(rh, vz[f"{name}/rhat"], rtol=1e-6, err_msg=name)
        s = V.summary(ess, rh)
        es, rs = vz[f"{name}/ess_summary"], vz[f"{name}/rhat_summary"]
        np.testing.assert_allclose([s["ess"][q] for q in ("min", "p10", "median", "max")], es, rtol=1e-6,
                                   err_msg=name)
        np.testing.assert_allclose([s["rhat"]["median"], s["rhat"]["max"]], rs[:2], rtol=1e-6, err_msg=name)
        assert (s["rhat"]["above_1_1"], s["rhat"]["above_1_2"]) == (int(rs[2]), int(rs[3])), name


def test_chr_oracle_reproduces_reference_kernel():
    path = GOLDEN / "chr_ref.npz"
    if not path.exists():
        pytest.skip("chr_ref.npz not recorded")
    z = np.load(path)
    for name in _cases(z):
        nspc, thin, k, resync = (int(v) for v in z[f"{name}/config"])
        tape = z[f"{name}/tape"]
        got = O.chr_run(z[f"{name}/A"], z[f"{name}/b"], z[f"{name}/x0"], nspc, thin, k,
                        pair_prob=float(z[f"{name}/pair_prob"]), resync_interval=resync, precision="fp64",
                        tape=tape)
        assert np.array_equal(got, z[f"{name}/samples"]), (name, np.abs(got - z[f"{name}/samples"]).max())
