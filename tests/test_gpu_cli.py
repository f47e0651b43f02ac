"""`naja sample run` and `naja validate` end to end on the GPU.

A genome-shaped model directory (rounding/ A, b, start, T, shift, extra
rows; gem/ bounds) is sampled with backmap and the bounds filter; the
samples.npy layout and header are the reference's (n_samples, dim) float32
C order, the samples satisfy A y <= b (checked through the unrounded run),
and `naja validate` reports the same ESS / split-R-hat as naja_validate in
the reference's chain-window reading.
"""
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from naja_b200 import synth
from naja_b200 import validate as V

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent
EXE = ROOT / "naja_b200" / "bin" / "naja"


def _write(path, M):
    M = np.atleast_2d(np.asarray(M, np.float64))
    if M.shape[0] == 1 and M.ndim == 2 and M.shape[1] > 1:
        M = M.T
    np.savetxt(path, M, delimiter=",", fmt="%.17g")


def _model_dir(tmp):
    g = synth.genome_shaped(n=130, d=40, density=0.1, seed_T=7, seed_u=8)
    v = synth.conditioned_variants(g, 1, max_reactions=10, seed=3)[0]
    md = tmp / "models" / "G130"
    (md / "rounding").mkdir(parents=True)
    (md / "gem").mkdir()
    r = md / "rounding"
    _write(r / "G130_rounding_A.csv", g["A"])
    _write(r / "G130_rounding_b.csv", g["b"].reshape(-1, 1))
    _write(r / "G130_rounding_start.csv", g["start"].reshape(-1, 1))
    _write(r / "G130_rounding_T.csv", g["T"])
    _write(r / "G130_rounding_shift.csv", g["shift"].reshape(-1, 1))
    _write(r / "G130_rounding_extra_A.csv", v["extra_A"])
    _write(r / "G130_rounding_extra_b.csv", v["extra_b"].reshape(-1, 1))
    _write(md / "gem" / "l_bounds.csv", v["l_new"].reshape(-1, 1))
    _write(md / "gem" / "u_bounds.csv", v["u_new"].reshape(-1, 1))
    A = np.vstack([g["A"], v["extra_A"]])
    b = np.concatenate([g["b"], v["extra_b"]])
    return md, A, b


def _run(*args):
    return subprocess.run([str(EXE), *map(str, args)], capture_output=True, text=True)


def test_sample_run_and_validate(cuda, tmp_path):
    md, A, b = _model_dir(tmp_path)
    out = tmp_path / "out"
    r = _run("sample", "run", "--model-dir", md, "--out-root", out, "--n-chains", 4, "--n-samples", 200,
             "--pair-prob", 0.3, "--resync-interval", 512, "--write-npy")
    assert r.returncode == 0, r.stderr + r.stdout
    assert "> gpu sampling" in r.stdout.splitlines()
    run = next(out.iterdir())
    raw = (run / "samples.npy").read_bytes()
    hlen = int.from_bytes(raw[8:10], "little")
    assert raw[:8] == b"\x93NUMPY\x01\x00" and raw[10 + hlen - 1:10 + hlen] == b"\n"
    Y = np.load(run / "samples.npy")
    assert Y.dtype == np.float32 and Y.shape == (800, 40) and Y.flags["C_CONTIGUOUS"]
    viol = (Y.astype(np.float64) @ A.T - b).max()
    assert viol <= 1e-4 * np.abs(b).max()
    prof = json.loads((run / "profile.json").read_text())
    assert prof["config"]["thinning"] == 40 // 6 and prof["config"]["constraints"] == A.shape[0]
    assert (run / "config_used.txt").exists()

    r = _run("validate", "--samples", run / "samples.npy", "--n-chains", 4)
    assert r.returncode == 0, r.stderr
    rep = json.loads(r.stdout)
    ess, rh = V.ess_rhat(Y, 4, layout=0)
    s = V.summary(ess, rh)
    assert rep["shape"] == [800, 40] and rep["status"] == s["status"]
    assert abs(rep["ess"]["min"] - s["ess"]["min"]) <= 0.05 + 1e-4 * s["ess"]["min"]
    assert abs(rep["rhat"]["max"] - s["rhat"]["max"]) <= 1e-4
    assert rep["rhat"]["above_1_1"] == s["rhat"]["above_1_1"]


def test_backmap_bounds_filter(cuda, tmp_path):
    md, A, b = _model_dir(tmp_path)
    out = tmp_path / "out"
    r = _run("sample", "run", "--model-dir", md, "--out-root", out, "--n-chains", 2, "--n-samples", 100, "--backmap",
             "--write-npy", "--bounds-policy", "filter", "--write-samples-valid", "--resync-interval", 256)
    assert r.returncode == 0, r.stderr + r.stdout
    run = next(out.iterdir())
    V_ = np.load(run / "samples.npy")
    assert V_.shape == (200, 130)
    valid = np.load(run / "samples_valid.npy")
    assert valid.shape[1] == 130 and valid.shape[0] <= 200
    r = _run("validate", "--samples", run / "samples.npy", "--n-chains", 2, "--model-dir", md)
    assert r.returncode == 0, r.stderr
    rep = json.loads(r.stdout)
    # reaction-space samples are checked against the GEM bounds directly
    assert rep["bounds"]["n_checked"] == 200 * 130
    # the same rule as the filter: no violating pair exactly when every sample was kept
    assert (rep["bounds"]["n_violations"] == 0) == (valid.shape[0] == 200)
