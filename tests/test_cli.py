"""The `naja` command line's host logic (CPU): flags, the model-directory
contract, the run directory and its files, and the phase lines that the
reference's tests/test_sample_cli_dry_run.sh checks."""
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
EXE = ROOT / "naja_b200" / "bin" / "naja"


def _model(tmp, name="MODEL_X", extra=False, backmap=False):
    md = tmp / "models" / name
    (md / "rounding").mkdir(parents=True)
    (md / "gem").mkdir()
    r = md / "rounding"
    (r / f"{name}_rounding_A.csv").write_text("1,0\n0,1\n-1,0\n0,-1\n")
    (r / f"{name}_rounding_b.csv").write_text("1\n1\n1\n1\n")
    (r / f"{name}_rounding_start.csv").write_text("0\n0\n")
    if extra:
        (r / f"{name}_rounding_extra_A.csv").write_text("1,1\n")
        (r / f"{name}_rounding_extra_b.csv").write_text("1.5\n")
    if backmap:
        (r / f"{name}_rounding_T.csv").write_text("1,0\n0,1\n1,1\n")
        (r / f"{name}_rounding_shift.csv").write_text("0\n0\n0\n")
        (md / "gem" / "l_bounds.csv").write_text("-1\n-1\n-2\n")
        (md / "gem" / "u_bounds.csv").write_text("1\n1\n2\n")
    return md


def _run(*args):
    return subprocess.run([str(EXE), *map(str, args)], capture_output=True, text=True)


@pytest.fixture(scope="module", autouse=True)
def _exe():
    if not EXE.exists():
        pytest.skip("naja CLI not built")


def test_dry_run_phase_lines_and_files(tmp_path):
    md = _model(tmp_path)
    r = _run("sample", "run", "--model-dir", md, "--out-root", tmp_path / "out", "--gpu", 0, "--n-chains", 1,
             "--n-samples", 1, "--bounds-policy", "ignore", "--dry-run")
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    for want in ("> validate model contract", "> write generated config", "> dry-run: not executing sampling"):
        assert want in lines
    runs = list((tmp_path / "out").iterdir())
    assert len(runs) == 1 and runs[0].name.startswith("MODEL_X_") and runs[0].name.endswith("_001")
    cfg = (runs[0] / "config_generated.txt").read_text()
    assert "MODEL_NAME=MODEL_X" in cfg and "N_CHAINS=1" in cfg and "TPB_SS=128" in cfg
    man = json.loads((runs[0] / "run_manifest.json").read_text())
    assert man["argv"][:3] == ["naja", "sample", "run"]
    assert man["config"]["n_chains"] == 1 and man["config"]["bounds_policy"] == "ignore"
    assert len(man["engine"]["sha256"]) == 64
    assert man["resolved_paths"]["A"].endswith("MODEL_X_rounding_A.csv")
    # a second run gets the next index
    _run("sample", "run", "--model-dir", md, "--out-root", tmp_path / "out", "--n-chains", 1, "--n-samples", 1,
         "--dry-run")
    assert sorted(p.name[-3:] for p in (tmp_path / "out").iterdir()) == ["001", "002"]


def test_contract_errors(tmp_path):
    md = _model(tmp_path)
    (md / "rounding" / "MODEL_X_rounding_b.csv").write_text("")
    r = _run("sample", "run", "--model-dir", md, "--out-root", tmp_path / "out", "--n-chains", 1, "--n-samples", 1,
             "--dry-run")
    assert r.returncode == 1 and "empty rounding_b" in r.stderr
    md2 = _model(tmp_path / "b")
    (md2 / "rounding" / "MODEL_X_rounding_extra_A.csv").write_text("1,1\n")
    r = _run("sample", "run", "--model-dir", md2, "--out-root", tmp_path / "out", "--n-chains", 1, "--n-samples", 1,
             "--dry-run")
    assert r.returncode == 1 and "both-present or both-absent" in r.stderr
    r = _run("sample", "run", "--model-dir", _model(tmp_path / "c"), "--out-root", tmp_path / "out", "--n-chains", 1,
             "--n-samples", 1, "--backmap", "--dry-run")
    assert r.returncode == 1 and "missing rounding_T" in r.stderr


def test_usage_errors(tmp_path):
    md = _model(tmp_path)
    base = ["sample", "run", "--model-dir", md, "--out-root", tmp_path / "out"]
    assert _run(*base, "--n-samples", 1).returncode == 2  # missing --n-chains
    assert _run(*base, "--n-chains", 1, "--n-samples", 1, "--bogus").returncode == 2
    assert _run(*base, "--n-chains", 1, "--n-samples", 1, "--pair-prob", 2).returncode == 2
    r = _run(*base, "--n-chains", 1, "--n-samples", 1, "--bounds-policy", "filter")
    assert r.returncode == 1 and "requires --backmap" in r.stderr
    assert _run("validate").returncode == 2


def _bulk_models(tmp, names=("M1", "M2")):
    for n in names:
        _model(tmp, n)
    lst = tmp / "models.txt"
    lst.write_text("# models\n" + "\n".join(names) + "\n\n")
    return tmp / "models", lst


def test_bulk_dry_run_files(tmp_path):
    root, lst = _bulk_models(tmp_path)
    r = _run("sample", "bulk", "--models-root", root, "--model-list", lst, "--out-root", tmp_path / "out",
             "--name", "RUN", "--gpus", "0,1", "--n-chains", 2, "--n-samples", 3, "--dry-run")
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    for want in ("> validate model contracts", "> write generated bulk config", "> dry-run: not executing bulk sampling"):
        assert want in lines
    runs = list((tmp_path / "out").iterdir())
    assert len(runs) == 1 and runs[0].name.startswith("RUN_") and runs[0].name.endswith("_001")
    cfg = (runs[0] / "bulk_config_generated.txt").read_text()
    assert "GPU_LIST=0,1" in cfg and f"BULK_MODEL_LIST={lst}" in cfg and "N_CHAINS=2" in cfg
    man = json.loads((runs[0] / "run_manifest.json").read_text())
    assert man["argv"][:3] == ["naja", "sample", "bulk"]
    # resuming into the same run directory writes the resume manifest beside the first
    r = _run("sample", "bulk", "--models-root", root, "--model-list", lst, "--resume-from", runs[0], "--name", "RUN",
             "--gpus", "0", "--n-chains", 2, "--n-samples", 3, "--dry-run", "--skip-existing")
    assert r.returncode == 0, r.stderr
    assert (runs[0] / "run_manifest_resume.json").exists()
    lines = r.stdout.splitlines()
    assert "  jobs            2" in lines and "  skip_existing   true" in lines


def test_bulk_usage_and_contract_errors(tmp_path):
    root, lst = _bulk_models(tmp_path)
    base = ["sample", "bulk", "--models-root", root, "--model-list", lst, "--out-root", tmp_path / "out",
            "--name", "RUN", "--n-chains", 1, "--n-samples", 1, "--dry-run"]
    assert _run(*base).returncode == 2  # missing --gpus
    assert _run(*base, "--gpus", "x").returncode == 2
    assert _run(*base, "--gpus", "0", "--bogus").returncode == 2
    r = _run("sample", "bulk", "--models-root", root, "--model-list", lst, "--name", "RUN", "--gpus", "0",
             "--n-chains", 1, "--n-samples", 1, "--dry-run")
    assert r.returncode == 2 and "--out-root" in r.stderr
    # every model's contract is checked before anything runs
    (root / "M2" / "rounding" / "M2_rounding_b.csv").write_text("")
    r = _run(*base, "--gpus", "0")
    assert r.returncode == 1 and "empty rounding_b" in r.stderr
    assert not (tmp_path / "out").exists()
    empty = tmp_path / "empty.txt"
    empty.write_text("# nothing\n")
    r = _run("sample", "bulk", "--models-root", root, "--model-list", empty, "--out-root", tmp_path / "out",
             "--name", "RUN", "--gpus", "0", "--n-chains", 1, "--n-samples", 1, "--dry-run")
    assert r.returncode == 1


def test_bulk_skip_existing_and_failures_on_the_host(tmp_path):
    """--skip-existing takes a model as done when one of its job directories
    holds non-empty samples.npy and profile.json (plus valid_mask.npy,
    valid_fraction.txt and bounds_report.json under the bounds filter); the
    newest such directory is reported.  A model that is not done runs, and
    here (no GPU) fails on its own: FAIL with its message in
    bulk_summary.csv, the others SKIP, exit status 1."""
    import os
    import time

    import torch

    if torch.cuda.is_available():
        pytest.skip("the failing job needs a host without a GPU")
    names = ("M1", "M2", "M3")
    for n in names:
        _model(tmp_path, n, backmap=True)
    root, lst = tmp_path / "models", tmp_path / "models.txt"
    lst.write_text("\n".join(names) + "\n")
    for n in names:
        (root / n / "rounding" / "INHERITED_FROM.txt").write_text("base_model_dir=/models/base\n")
    run = tmp_path / "out" / "RUN_20260101_001"
    files = ("samples.npy", "profile.json")
    filt = ("valid_mask.npy", "valid_fraction.txt", "bounds_report.json")
    for n in names:
        for idx, extra in ((1, ()), (2, filt)):
            job = run / n / f"{n}_20260101_00{idx}"
            job.mkdir(parents=True)
            for f in files + extra:
                (job / f).write_text("x")
            os.utime(job, (time.time() - 100 * (3 - idx), time.time() - 100 * (3 - idx)))
    (run / "M3" / "M3_20260101_002" / "samples.npy").write_text("")  # empty: not complete
    (run / "M3" / "M3_20260101_001" / "profile.json").unlink()
    r = _run("sample", "bulk", "--models-root", root, "--model-list", lst, "--resume-from", run, "--name", "RUN",
             "--gpus", "0", "--n-chains", 1, "--n-samples", 2, "--skip-existing")
    assert r.returncode == 1 and "bulk sampling failed" in r.stderr
    assert r.stdout.count("-> SKIP") == 2 and "M3 -> FAIL" in r.stdout
    rows = {line.split(",")[0]: line.split(",") for line in (run / "bulk_summary.csv").read_text().splitlines()[1:]}
    assert rows["M1"][1] == rows["M2"][1] == "SKIP" and rows["M3"][1] == "FAIL"
    assert rows["M1"][5].endswith("M1_20260101_002")  # the newest complete directory
    assert rows["M3"][4] and rows["M3"][5].startswith(str(run / "M3" / "M3_"))
    assert all(r_[6] == "/models/base" for r_ in rows.values())
    # under the bounds filter only directories with the filter's outputs count
    (run / "M1" / "M1_20260101_002" / "bounds_report.json").unlink()
    r = _run("sample", "bulk", "--models-root", root, "--model-list", lst, "--resume-from", run, "--name", "RUN",
             "--gpus", "0", "--n-chains", 1, "--n-samples", 2, "--skip-existing", "--backmap",
             "--bounds-policy", "filter")
    assert r.returncode == 1, r.stderr
    assert "M2 -> SKIP" in r.stdout and "M1 -> FAIL" in r.stdout and "M3 -> FAIL" in r.stdout
