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
