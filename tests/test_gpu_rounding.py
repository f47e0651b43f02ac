"""Rounded sampling and the run-to-gate loop (GPU).

Samples of a rounded polytope {z : A M z <= b - A c}, mapped back with
y = M z + c by the FP64 backmap kernel, must lie in the original polytope
A y <= b (the reference's Dikin preconditioner, src/rounding/
dikin_precondition.cpp:36-183 of quothbonney/naja, and the whole-ellipsoid
rounding).  sample_to_gate stops at split-R-hat < 1.01 with no bound
violations and its R-hat curve and ESS agree with the validate kernel on the
same samples.
"""
import numpy as np
import pytest

from naja_b200 import Polytope, backmap, gate, rounding, synth
from naja_b200 import validate as V

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method", ["dikin", "dikin_full"])
def test_rounded_samples_map_back_inside(cuda, method):
    g = synth.genome_shaped(n=600, d=120, density=0.08, seed_T=21, seed_u=22)
    A, b = g["A"], g["b"]
    r = gate.make_rounding(method, A, b, g["start"])
    P = Polytope(r.A, r.b)
    Z = P.run(r.z0, 200, 20, 8, seed=3, pair_prob=0.3, resync_interval=400, out_dtype="f64")
    P.check()
    assert np.all(Z @ r.A.T <= r.b + 1e-6 * np.maximum(1.0, np.abs(r.b)))
    Y = backmap(r.M, r.c, Z, mode="fp64", out_dtype=np.float64)
    assert np.allclose(Y, r.to_y(Z), rtol=0, atol=1e-10 * np.abs(Y).max())
    assert np.all(Y @ A.T - b <= 1e-6 * np.maximum(1.0, np.abs(b)))


def test_sample_to_gate_reaches_gate_on_a_box(cuda):
    # a thin box: after whole-ellipsoid rounding it is a cube, mixing in a few sweeps
    d = 10
    A = np.vstack([np.eye(d), -np.eye(d)])
    b = np.concatenate([np.linspace(0.01, 1.0, d), np.linspace(0.01, 1.0, d)])
    out = gate.sample_to_gate(A, b, np.zeros(d), method="dikin_full", nchains=8, thinning=10, chunk_nspc=2000,
                              resync_interval=100, budget_s=30.0, keep_samples=True)
    assert out["reached"] and out["rhat_max"] < 1.01 and out["bounds_violations"] == 0
    Y = out["samples"]
    _, rh = V.ess_rhat(Y, 8, layout=1)
    assert rh.max() == pytest.approx(out["rhat_max"])
    # uniform on the box: mean 0, variance h^2 / 3 per coordinate (h the half-width)
    y = Y.double().cpu().numpy()
    assert np.allclose(y.var(axis=0), b[:d] ** 2 / 3.0, rtol=0.1)
    assert out["min_ess"] > 0 and out["min_ess_per_s"] > 0
    assert [c["steps_per_chain"] for c in out["curve"]] == [2000 * 10 * (k + 1) for k in range(out["chunks"])]


def test_sample_to_gate_stops_at_budget(cuda):
    g = synth.genome_shaped(n=600, d=120, density=0.08, seed_T=21, seed_u=22)
    out = gate.sample_to_gate(g["A"], g["b"], g["start"], method="none", nchains=4, thinning=50, chunk_nspc=200,
                              resync_interval=200, budget_s=0.5, max_chunks=3)
    assert out["chunks"] <= 3 and len(out["curve"]) == out["chunks"]
    assert out["bounds_violations"] == 0


def test_dikin_full_on_the_gpu_matches_the_host(cuda):
    """dikin_full(device=0) takes the host's steps in FP64 on the GPU: the same
    centre, M and rounded polytope up to rounding in the last digits."""
    from naja_b200 import rounding, synth

    g = synth.genome_shaped(n=900, d=240, density=0.08, seed_T=6, seed_u=7)
    start = g["start"] + 1e-3  # off the centre, so Newton takes several steps
    cpu = rounding.dikin_full(g["A"], g["b"], start)
    gpu = rounding.dikin_full(g["A"], g["b"], start, device=0)
    assert gpu.info["newton_iterations"] == cpu.info["newton_iterations"] > 1
    for name in ("M", "c", "A", "b"):
        x, y = getattr(cpu, name), getattr(gpu, name)
        assert np.abs(x - y).max() <= 1e-9 * max(1.0, np.abs(x).max()), name
    dv = gpu.info["dev"]
    assert np.array_equal(dv["A"].cpu().numpy(), gpu.A)
