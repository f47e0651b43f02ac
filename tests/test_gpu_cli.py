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


def _model_dir(tmp, name="G130", seed=3):
    g = synth.genome_shaped(n=130, d=40, density=0.1, seed_T=7, seed_u=8)
    v = synth.conditioned_variants(g, 1, max_reactions=10, seed=seed)[0]
    md = tmp / "models" / name
    (md / "rounding").mkdir(parents=True)
    (md / "gem").mkdir()
    r = md / "rounding"
    _write(r / f"{name}_rounding_A.csv", g["A"])
    _write(r / f"{name}_rounding_b.csv", g["b"].reshape(-1, 1))
    _write(r / f"{name}_rounding_start.csv", g["start"].reshape(-1, 1))
    _write(r / f"{name}_rounding_T.csv", g["T"])
    _write(r / f"{name}_rounding_shift.csv", g["shift"].reshape(-1, 1))
    _write(r / f"{name}_rounding_extra_A.csv", v["extra_A"])
    _write(r / f"{name}_rounding_extra_b.csv", v["extra_b"].reshape(-1, 1))
    _write(md / "gem" / "l_bounds.csv", v["l_new"].reshape(-1, 1))
    _write(md / "gem" / "u_bounds.csv", v["u_new"].reshape(-1, 1))
    (md / "gem" / "reaction_ids.txt").write_text("".join(f"R_{k}\n" for k in range(130)))
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
    _check_filter_outputs(run, md, V_, 1e-6)


def _check_filter_outputs(run, md, V_, eps):
    """valid_mask.npy / valid_fraction.txt / bounds_report.json as
    src/engine/bounds_filter.cpp:65-180 writes them, recomputed here."""
    lb = np.loadtxt(md / "gem" / "l_bounds.csv", delimiter=",").reshape(-1)
    ub = np.loadtxt(md / "gem" / "u_bounds.csv", delimiter=",").reshape(-1)
    x = V_.astype(np.float64)
    viol = np.maximum((lb - x) - eps, (x - ub) - eps)
    worst = np.where(viol > 0, viol, 0.0).max(axis=1)
    mask = np.load(run / "valid_mask.npy")
    assert mask.dtype == np.uint8 and mask.shape == (V_.shape[0],)
    assert np.array_equal(mask, (worst == 0).astype(np.uint8))
    assert float((run / "valid_fraction.txt").read_text()) == pytest.approx(mask.mean(), rel=1e-11)
    valid = np.load(run / "samples_valid.npy")
    assert np.array_equal(valid, V_[mask == 1])
    rep = json.loads((run / "bounds_report.json").read_text())
    assert rep["n_total"] == V_.shape[0] and rep["n_valid"] == int(mask.sum())
    assert rep["max_violation"] == pytest.approx(worst.max(), rel=1e-11, abs=0)
    assert rep["mean_violation"] == pytest.approx(worst.mean(), rel=1e-9, abs=1e-300)
    assert rep["p99_violation"] == pytest.approx(np.sort(worst)[(99 * (len(worst) - 1)) // 100], rel=1e-11, abs=0)
    by_rxn = np.where(viol > 0, viol, 0.0).max(axis=0)
    top = [t["index"] for t in rep["top_violations"]]
    want = [int(k) for k in np.argsort(-by_rxn, kind="stable")[:10] if by_rxn[k] > 0]
    assert sorted(top) == sorted(want)
    assert all(t["reaction"] == f"R_{t['index']}" for t in rep["top_violations"])
    assert rep["outputs"]["samples_valid"].endswith("samples_valid.npy")


def test_bulk_two_workers_skip_and_failure(cuda, tmp_path):
    """naja sample bulk (src/engine/job_bulk.cpp:115-267): two worker threads
    on GPU 0 share three models; a job's samples are those `sample run`
    gives for the same model directory and GPU; --skip-existing with
    --resume-from reruns nothing; a model whose start is infeasible fails on
    its own and fails the run."""
    for k, name in enumerate(("B1", "B2", "B3")):
        _model_dir(tmp_path, name, seed=10 + k)
    root = tmp_path / "models"
    lst = tmp_path / "list.txt"
    lst.write_text("B1\nB2\nB3\n")
    flags = ["--n-chains", 2, "--n-samples", 60, "--backmap", "--write-npy", "--bounds-policy", "filter",
             "--resync-interval", 256, "--thinning", 3]
    out = tmp_path / "out"
    r = _run("sample", "bulk", "--models-root", root, "--model-list", lst, "--out-root", out, "--name", "RUN",
             "--gpus", "0,0", *flags)
    assert r.returncode == 0, r.stderr + r.stdout
    assert "bulk sampling :: 3 jobs across 2 gpu(s)" in r.stdout and "completed : 3 / 3" in r.stdout
    run = next(out.iterdir())
    rows = [line.split(",") for line in (run / "bulk_summary.csv").read_text().splitlines()]
    assert rows[0] == ["model", "status", "elapsed_s", "device_id", "message", "output_dir", "inherited_from_base"]
    assert sorted(r_[0] for r_ in rows[1:]) == ["B1", "B2", "B3"]
    assert all(r_[1] == "OK" and r_[3] == "0" for r_ in rows[1:])
    for name in ("B1", "B2", "B3"):
        jobs = list((run / name).iterdir())
        assert len(jobs) == 1 and jobs[0].name.startswith(f"{name}_") and jobs[0].name.endswith("_001")
        V_ = np.load(jobs[0] / "samples.npy")
        assert V_.shape == (120, 130)
        for f in ("profile.json", "config_used.txt", "valid_mask.npy", "valid_fraction.txt", "bounds_report.json"):
            assert (jobs[0] / f).stat().st_size > 0
    # the same job through `sample run` (same model directory string, same GPU): same seed, same samples
    single = tmp_path / "single"
    r = _run("sample", "run", "--model-dir", root / "B2", "--out-root", single, "--gpu", 0, *flags)
    assert r.returncode == 0, r.stderr + r.stdout
    assert np.array_equal(np.load(next(single.iterdir()) / "samples.npy"),
                          np.load(next((run / "B2").iterdir()) / "samples.npy"))
    # resume: every model is complete, nothing runs again
    r = _run("sample", "bulk", "--models-root", root, "--model-list", lst, "--resume-from", run, "--name", "RUN",
             "--gpus", "0", "--skip-existing", *flags)
    assert r.returncode == 0, r.stderr + r.stdout
    assert r.stdout.count("-> SKIP") == 3 and (run / "run_manifest_resume.json").exists()
    assert all(len(list((run / n).iterdir())) == 1 for n in ("B1", "B2", "B3"))
    # an infeasible start fails that job only
    _write(root / "B3" / "rounding" / "B3_rounding_start.csv", np.full((40, 1), 1e6))
    out2 = tmp_path / "out2"
    r = _run("sample", "bulk", "--models-root", root, "--model-list", lst, "--out-root", out2, "--name", "RUN",
             "--gpus", "0", *flags)
    assert r.returncode == 1 and "bulk sampling failed" in r.stderr
    rows = {r_.split(",")[0]: r_.split(",") for r_ in (next(out2.iterdir()) / "bulk_summary.csv").read_text().splitlines()[1:]}
    assert rows["B1"][1] == "OK" and rows["B2"][1] == "OK" and rows["B3"][1] == "FAIL"
    assert "infeasible start point" in rows["B3"][4]


def _schedule(path, d, seed):
    rng = np.random.default_rng(seed)
    perm = rng.permutation(d)
    th = rng.uniform(-np.pi, np.pi, d // 2)
    with open(path, "w") as f:
        f.write("# i,j,c,s\n")
        for k in range(d // 2):
            f.write(f"{perm[2 * k]},{perm[2 * k + 1]},{float(np.cos(th[k]))!r},{float(np.sin(th[k]))!r}\n")


def test_pair_schedule_and_warmup_rounding(cuda, tmp_path):
    """--pair-schedule and --iter-rounding-* select Jacobi-pair steps
    (src/rounding/plan.cpp:12-62): the runs succeed, print the reference's
    phase lines, stay feasible and differ from the run without them."""
    md, A, b = _model_dir(tmp_path)
    sched = tmp_path / "sched.csv"
    _schedule(sched, 40, 1)
    common = ["--model-dir", md, "--n-chains", 2, "--n-samples", 150, "--pair-prob", 0.4, "--resync-interval", 64,
              "--write-npy", "--precision", "fp64"]
    outs = {}
    for name, extra in (("plain", []), ("file", ["--pair-schedule", sched]),
                        ("warmup", ["--iter-rounding-passes", 2, "--iter-rounding-warmup", 300])):
        r = _run("sample", "run", *common, "--out-root", tmp_path / name, *extra)
        assert r.returncode == 0, r.stderr + r.stdout
        if name == "file":
            assert "> loading pair schedule" in r.stdout.splitlines()
        if name == "warmup":
            assert "> iterative rounding-lite (warmup)" in r.stdout.splitlines()
        Y = np.load(next((tmp_path / name).iterdir()) / "samples.npy").astype(np.float64)
        assert (Y @ A.T - b).max() <= 1e-4 * np.abs(b).max()
        outs[name] = Y
    assert not np.array_equal(outs["plain"], outs["file"]) and not np.array_equal(outs["plain"], outs["warmup"])
    bad = tmp_path / "bad.csv"
    bad.write_text("0,1,1\n")
    r = _run("sample", "run", *common, "--out-root", tmp_path / "bad", "--pair-schedule", bad)
    assert r.returncode == 1 and "expected 4 columns" in r.stderr


def test_affine_hull_reduction(cuda, tmp_path):
    """--affine-hull-tol (src/engine/job_sampling.cu:196-235, 299-303): two
    rows tight at the start pin a plane; the chains sample inside it and the
    composed backmap returns points of the original polytope on that plane."""
    d = 12
    rng = np.random.default_rng(5)
    a = rng.standard_normal(d)
    A = np.vstack([np.eye(d), -np.eye(d), a, -a])
    b = np.concatenate([np.ones(d), np.ones(d), [0.0, 0.0]])
    md = tmp_path / "models" / "H12"
    (md / "rounding").mkdir(parents=True)
    r_ = md / "rounding"
    _write(r_ / "H12_rounding_A.csv", A)
    _write(r_ / "H12_rounding_b.csv", b.reshape(-1, 1))
    _write(r_ / "H12_rounding_start.csv", np.zeros((d, 1)))
    _write(r_ / "H12_rounding_T.csv", np.eye(d))
    _write(r_ / "H12_rounding_shift.csv", np.zeros((d, 1)))
    r = _run("sample", "run", "--model-dir", md, "--out-root", tmp_path / "o1", "--n-chains", 2, "--n-samples", 300,
             "--affine-hull-tol", 1e-9, "--write-npy", "--verbose", "--resync-interval", 100)
    assert r.returncode == 0, r.stderr + r.stdout
    assert "affine_hull_dim  11 (from 12)" in r.stdout
    Z = np.load(next((tmp_path / "o1").iterdir()) / "samples.npy")
    assert Z.shape == (600, 11)
    r = _run("sample", "run", "--model-dir", md, "--out-root", tmp_path / "o2", "--n-chains", 2, "--n-samples", 300,
             "--affine-hull-tol", 1e-9, "--write-npy", "--backmap", "--backmap-mode", "fp64", "--resync-interval", 100,
             "--thinning", 50)
    assert r.returncode == 0, r.stderr + r.stdout
    Y = np.load(next((tmp_path / "o2").iterdir()) / "samples.npy").astype(np.float64)
    assert Y.shape == (600, d)
    assert np.abs(Y @ a).max() <= 1e-5  # on the plane a y = 0
    assert (np.abs(Y).max() <= 1.0 + 1e-5) and Y.std(axis=0).min() > 0.05  # inside the box, and moving


def test_calibrate_rounding(cuda, tmp_path):
    """naja sample calibrate-rounding (src/cli/sample/cmd_calibrate_rounding.cpp:24-195):
    with one pass, every pair's (c, s) is the Jacobi rotation of the pair's
    warm-up moments averaged over the models, each model's warm-up being one
    chain of --warmup samples with the pairs at angle 0 and seed ^ model ^ 1."""
    root = tmp_path / "models"
    names = []
    for k in range(2):
        g = synth.genome_shaped(n=120, d=30, density=0.12, seed_T=40 + k, seed_u=50 + k)
        md = root / f"M{k}"
        (md / "rounding").mkdir(parents=True)
        _write(md / "rounding" / f"M{k}_rounding_A.csv", g["A"])
        _write(md / "rounding" / f"M{k}_rounding_b.csv", g["b"].reshape(-1, 1))
        _write(md / "rounding" / f"M{k}_rounding_start.csv", g["start"].reshape(-1, 1))
        names.append((f"M{k}", g))
    (tmp_path / "list.txt").write_text("# models\nM0\n\nM1\n")
    out = tmp_path / "sched.csv"
    r = _run("sample", "calibrate-rounding", "--models-root", root, "--model-list", tmp_path / "list.txt", "--out",
             out, "--warmup", 400, "--passes", 1, "--pair-prob", 0.3, "--seed", 9)
    assert r.returncode == 0, r.stderr + r.stdout
    assert r.stdout.startswith("OK") and "pairs            :: 15" in r.stdout
    rows = np.loadtxt(out, delimiter=",", ndmin=2)
    i, j = rows[:, 0].astype(int), rows[:, 1].astype(int)
    assert sorted(np.concatenate([i, j]).tolist()) == list(range(30))
    from naja_b200 import Polytope

    sv = np.zeros((3, 15))
    for mi, (_, g) in enumerate(names):
        P = Polytope(g["A"], g["b"])
        W = P.run(g["start"], 400, 1, 1, seed=9 ^ mi ^ 1, pair_prob=0.3, pair_mode=2,
                  pairs=(i, j, np.ones(15), np.zeros(15)), precision="fp64", rng="mrg", out_dtype="f64")
        di, dj = W[:, i] - W[:, i].mean(axis=0), W[:, j] - W[:, j].mean(axis=0)
        sv += np.stack([(di * di).mean(axis=0), (dj * dj).mean(axis=0), (di * dj).mean(axis=0)])
    vi, vj, cij = sv / 2
    th = 0.5 * np.arctan2(2 * cij, vi - vj)
    want_c = np.where(cij == 0, 1.0, np.cos(th))
    want_s = np.where(cij == 0, 0.0, np.sin(th))
    assert np.allclose(rows[:, 2], want_c, atol=2e-5) and np.allclose(rows[:, 3], want_s, atol=2e-5)
