"""Builds libnaja_b200.so (sm_100a) in-tree with nvcc.

Each CUDA translation unit is compiled in parallel into naja_b200/_build/;
the CHR step kernel is split into one unit per (element type, consumer
thread count).  Objects are rebuilt when their source or any header in
csrc/ or include/ is newer.  Usage: python -m naja_b200.build [-j N] [--clean]
"""
from __future__ import annotations

import argparse
import hashlib
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "_build"
LIB = PKG / "libnaja_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: the CHR kernels spell every fused multiply-add they mean
# (__fma_rn / __fmaf_rn); nothing else may be contracted, so the device
# arithmetic is reproducible bit for bit by the CPU restatement.
BASE = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include")]
CHR_THREADS = (32, 64, 128, 256, 448, 512, 992)


def _units():
    units = []
    for real in ("float", "double"):
        for nt in CHR_THREADS:
            units.append((f"chr_{real}_{nt}", CSRC / "chr_inst.cu",
                          ["-fmad=false", f"-DNAJA_CHR_REAL={real}", f"-DNAJA_CHR_NT={nt}"]))
    for nt in (128, 256, 512):
        units.append((f"chr_batched_{nt}", CSRC / "chr_batched_inst.cu", ["-fmad=false", f"-DNAJA_CHR_NT={nt}"]))
    units.append(("chr_sparse", CSRC / "chr_sparse_inst.cu", ["-fmad=false"]))
    units.append(("chr_host", CSRC / "chr_host.cu", ["-fmad=false"]))
    units.append(("capi", CSRC / "capi.cu", []))
    units.append(("pipeline", CSRC / "pipeline.cu", []))
    units.append(("validate", CSRC / "validate.cu", ["-fmad=false"]))
    units.append(("backmap", CSRC / "backmap.cu", ["-fmad=false"]))
    units.append(("backmap_tc", CSRC / "backmap_tc.cu", []))
    units.append(("mlp", CSRC / "mlp.cu", []))
    return units


def _inputs_digest(src: Path, cmd: list[str]) -> str:
    """Hash of the unit's source, every header it may include and its command.

    Content hashes, not mtimes: an edit made while another build is still
    compiling the old text must not be mistaken for up to date."""
    h = hashlib.sha256(" ".join(cmd).encode())
    for p in [src, *sorted(CSRC.glob("*.cuh")), *sorted((ROOT / "include").glob("*.h"))]:
        h.update(p.name.encode())
        h.update(p.read_bytes())
    return h.hexdigest()


def _compile(name, src, flags, force, verbose):
    obj = OUT / f"{name}.o"
    stamp = OUT / f"{name}.sha256"
    cmd = [NVCC, *ARCH, *BASE, *flags, "-c", str(src), "-o", str(obj)]
    digest = _inputs_digest(src, cmd)
    if not force and obj.exists() and stamp.exists() and stamp.read_text() == digest:
        return obj, None
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"{' '.join(cmd)}\n{r.stdout}{r.stderr}"
    stamp.write_text(digest)
    return obj, None


def build(jobs: int | None = None, force: bool = False, verbose: bool = False) -> Path:
    OUT.mkdir(exist_ok=True)
    units = _units()
    jobs = jobs or max(1, min(len(units), os.cpu_count() or 4))
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        results = list(ex.map(lambda u: _compile(*u, force, verbose), units))
    errors = [e for _, e in results if e]
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n\n".join(errors))
    objs = [o for o, _ in results]
    link_stamp = OUT / "link.sha256"
    h = hashlib.sha256()
    for o in objs:
        h.update(o.read_bytes())
    if force or not LIB.exists() or not link_stamp.exists() or link_stamp.read_text() != h.hexdigest():
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(tmp), *map(str, objs)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}{r.stderr}")
        os.replace(tmp, LIB)
        link_stamp.write_text(h.hexdigest())
    _build_cli(force)
    return LIB


CLI_SRC = PKG / "cli" / "naja_cli.cpp"
CLI = PKG / "bin" / "naja"


def _build_cli(force: bool = False) -> Path:
    """The `naja` command line (host C++ over the C ABI), linked to the
    in-tree library through an $ORIGIN-relative rpath."""
    cmd = ["/usr/bin/g++", "-O2", "-std=c++17", "-Wall", "-I", str(ROOT / "include"), str(CLI_SRC), "-L", str(PKG),
           "-lnaja_b200", "-Wl,-rpath,$ORIGIN/..", "-o", str(CLI)]
    stamp = OUT / "cli.sha256"
    h = hashlib.sha256(" ".join(cmd).encode())
    h.update(CLI_SRC.read_bytes())
    h.update((ROOT / "include" / "naja_chr.h").read_bytes())
    if force or not CLI.exists() or not stamp.exists() or stamp.read_text() != h.hexdigest():
        CLI.parent.mkdir(exist_ok=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"g++ failed:\n{' '.join(cmd)}\n{r.stdout}{r.stderr}")
        stamp.write_text(h.hexdigest())
    return CLI


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args(argv)
    if a.clean and OUT.exists():
        shutil.rmtree(OUT)
    lib = build(a.j, force=a.clean, verbose=a.v)
    print(lib)


if __name__ == "__main__":
    sys.exit(main())
