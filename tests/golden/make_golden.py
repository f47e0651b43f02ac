"""Records golden vectors from the reference's own implementation.

Test infrastructure only.  The fixtures pin the CPU oracle (oracle/) to the
reference itself, so the CPU test suite checks the restatement without the
reference tree or a GPU:

  validate  (CPU, needs oracle/_ref/libnaja_validate_ref.so, built from the
            reference's src/validate/mcmc.cpp and extern/kissfft by
            oracle/refharness/Makefile): seeded sample matrices and the
            reference's compute_ess / compute_split_rhat outputs
            -> tests/golden/validate_ref.npz
  chr       (GPU box, needs oracle/_ref/libnaja_ref.so, the reference's
            src/gpu kernel): small polytopes sampled by the reference's
            CoordinateHitAndRun with its cuRAND MRG32k3a streams, plus the
            uniform tape of those streams recorded by calling cuRAND
            -> tests/golden/chr_ref.npz

Usage: python tests/golden/make_golden.py validate|chr
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))


def _ar1(rng, n, rho, mean=0.0):
    x = np.empty(n)
    x[0] = rng.standard_normal()
    e = rng.standard_normal(n) * np.sqrt(max(1.0 - rho * rho, 1e-12))
    for t in range(1, n):
        x[t] = rho * x[t - 1] + e[t]
    return x + mean


def validate_cases():
    """(name, samples (n_total, dim) float32 in the reference's chain-window layout, n_chains)."""
    rng = np.random.default_rng(20260)
    cases = []
    # AR(1) dims with a spread of autocorrelation, 4 chains x 400
    rhos = [0.0, 0.3, 0.6, 0.9, 0.95, -0.5]
    chains = [np.stack([_ar1(rng, 400, r) for r in rhos], axis=1) for _ in range(4)]
    cases.append(("ar1_4x400", np.concatenate(chains).astype(np.float32), 4))
    # chains with different means: split-R-hat well above 1
    chains = [np.stack([_ar1(rng, 500, 0.7, mean=c * s) for s in (0.0, 0.2, 1.0, 3.0)], axis=1) for c in range(8)]
    cases.append(("shifted_8x500", np.concatenate(chains).astype(np.float32), 8))
    # a constant dim next to white noise; shortest allowed chains
    x = rng.standard_normal((4 * 6, 3))
    x[:, 1] = 2.5
    cases.append(("const_4x6", x.astype(np.float32), 4))
    # trending series (no negative pair before n/2) and odd lengths
    t = np.arange(301)
    chains = [np.stack([np.sin(t / 40.0 + c), t / 300.0 + 0.01 * rng.standard_normal(301)], axis=1) for c in range(3)]
    cases.append(("trend_3x301", np.concatenate(chains).astype(np.float32), 3))
    return cases


def make_validate():
    lib = C.CDLL(str(ROOT / "oracle" / "_ref" / "libnaja_validate_ref.so"))
    vp, i = C.c_void_p, C.c_int
    for f in (lib.ref_compute_ess, lib.ref_compute_split_rhat):
        f.argtypes = [vp, i, i, i, vp, vp]
        f.restype = i
    lib.ref_validate_last_error.restype = C.c_char_p
    out = {}
    for name, S, k in validate_cases():
        S = np.ascontiguousarray(S, dtype=np.float32)
        n_total, dim = S.shape
        ess = np.zeros(dim, np.float32)
        ess_s = np.zeros(4, np.float32)
        rh = np.zeros(dim, np.float32)
        rh_s = np.zeros(4, np.float32)
        if lib.ref_compute_ess(S.ctypes.data, dim, n_total, k, ess.ctypes.data, ess_s.ctypes.data):
            raise RuntimeError(lib.ref_validate_last_error().decode())
        if lib.ref_compute_split_rhat(S.ctypes.data, dim, n_total, k, rh.ctypes.data, rh_s.ctypes.data):
            raise RuntimeError(lib.ref_validate_last_error().decode())
        out[f"{name}/samples"] = S
        out[f"{name}/n_chains"] = np.array(k)
        out[f"{name}/ess"] = ess
        out[f"{name}/ess_summary"] = ess_s
        out[f"{name}/rhat"] = rh
        out[f"{name}/rhat_summary"] = rh_s
    np.savez_compressed(HERE / "validate_ref.npz", **out)
    print("wrote", HERE / "validate_ref.npz", sorted({k.split('/')[0] for k in out}))


def chr_cases():
    from naja_b200 import synth

    g = synth.genome_shaped(n=130, d=40, density=0.1, seed_T=7, seed_u=8)
    return [
        ("cube8", *synth.cube(8), dict(nspc=30, thinning=5, nchains=3, seed=77, pair_prob=0.0, tpb=128)),
        ("simplex6", *synth.simplex(6), dict(nspc=30, thinning=7, nchains=3, seed=5, pair_prob=0.3, tpb=64,
                                             resync_interval=10 ** 6)),
        ("slab6", *synth.thin_slab(6, 1e-4), dict(nspc=25, thinning=4, nchains=2, seed=9, pair_prob=0.5, tpb=32)),
        ("genome130x40", g["A"], g["b"], g["start"], dict(nspc=20, thinning=6, nchains=3, seed=3, pair_prob=0.3,
                                                           tpb=256)),
    ]


def make_chr():
    import oracle.oracle as O
    from naja_b200 import mrg_tape

    out = {}
    for name, A, b, x0, kw in chr_cases():
        kw = dict(kw)
        nspc, thin, k = kw.pop("nspc"), kw.pop("thinning"), kw.pop("nchains")
        ref, _, _ = O.reference_chr_run(A, b, x0, nspc, thin, k, want_v=False, **kw)
        tape = mrg_tape(kw["seed"], k, 4 * nspc * thin + 8)
        out[f"{name}/A"] = np.asarray(A, np.float64)
        out[f"{name}/b"] = np.asarray(b, np.float64)
        out[f"{name}/x0"] = np.asarray(x0, np.float64)
        out[f"{name}/config"] = np.array([nspc, thin, k, kw.get("resync_interval", 0)], np.int64)
        out[f"{name}/pair_prob"] = np.array(kw["pair_prob"])
        out[f"{name}/seed"] = np.array(kw["seed"], np.int64)
        out[f"{name}/tape"] = np.asarray(tape, np.float64)
        out[f"{name}/samples"] = np.asarray(ref, np.float64)
    np.savez_compressed(HERE / "chr_ref.npz", **out)
    print("wrote", HERE / "chr_ref.npz", sorted({k.split('/')[0] for k in out}))


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else ""
    if what == "validate":
        make_validate()
    elif what == "chr":
        make_chr()
    else:
        sys.exit(__doc__)
