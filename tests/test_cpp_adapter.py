"""The header-only C++ adapter (include/naja/gpusamplers.hpp) compiles as a
drop-in for the reference's naja::gpu API and, on a GPU, runs correctly."""
import os
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
SRC = ROOT / "tests" / "cpp" / "adapter_drop_in.cpp"
CUDA = Path("/usr/local/cuda")


def _compile(out: Path):
    cxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"
    cmd = [cxx, "-std=c++17", "-O1", "-I", str(ROOT / "include"), "-I", str(CUDA / "include"), str(SRC), "-o",
           str(out), "-L", str(ROOT / "naja_b200"), "-lnaja_b200", f"-Wl,-rpath,{ROOT / 'naja_b200'}",
           "-L", str(CUDA / "lib64"), "-lcudart", f"-Wl,-rpath,{CUDA / 'lib64'}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def test_adapter_compiles(tmp_path):
    _compile(tmp_path / "adapter")
    assert (tmp_path / "adapter").exists()


@pytest.mark.gpu
def test_adapter_runs(cuda, tmp_path):
    exe = tmp_path / "adapter"
    _compile(exe)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "adapter ok" in r.stdout


def test_rounding_header_host_logic(tmp_path):
    """include/naja/rounding.hpp: Jacobi rotation, schedule CSV, pairing and
    affine-hull basis (host code only; links the library, runs no kernel)."""
    exe = tmp_path / "rounding_host"
    cxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"
    cmd = [cxx, "-std=c++17", "-O1", "-I", str(ROOT / "include"), str(ROOT / "tests" / "cpp" / "rounding_host.cpp"),
           "-o", str(exe), "-L", str(ROOT / "naja_b200"), "-lnaja_b200", f"-Wl,-rpath,{ROOT / 'naja_b200'}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "rounding host ok" in r.stdout
