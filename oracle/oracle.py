"""TEST INFRASTRUCTURE ONLY -- ctypes binding of the CPU oracle
(oracle/_build/liboracle.so, built by oracle/Makefile).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module; the product (naja_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists() or LIB.stat().st_mtime < max(p.stat().st_mtime for p in HERE.glob("*.c")):
            build()
        lib = C.CDLL(str(LIB))
        vp, i, d, u64, l = C.c_void_p, C.c_int, C.c_double, C.c_uint64, C.c_long
        lib.oracle_chr_run.argtypes = [i, i, vp, i, vp, vp, i, i, i, i, u64, d, i, d, i, i,
                                       vp, vp, vp, vp, i, i, i, vp, l, u64, i, vp, vp, vp, i]
        lib.oracle_chr_run.restype = i
        lib.oracle_philox4x32_10.argtypes = [vp, C.c_uint32, C.c_uint32, vp]
        lib.oracle_philox4x32_10.restype = None
        lib.oracle_ess.argtypes = [vp, l, i, i, i, vp]
        lib.oracle_ess.restype = i
        lib.oracle_split_rhat.argtypes = [vp, l, i, i, i, vp]
        lib.oracle_split_rhat.restype = i
        lib.oracle_ess_series.argtypes = [vp, l]
        lib.oracle_ess_series.restype = d
        _lib = lib
    return _lib


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def philox(ctr, key):
    c = np.ascontiguousarray(np.asarray(ctr, dtype=np.uint32))
    out = np.empty(4, dtype=np.uint32)
    load().oracle_philox4x32_10(_p(c), int(key[0]), int(key[1]), _p(out))
    return out


def chr_run(A, b, X0, nspc, thinning, nchains, *, seed=0, pair_prob=0.0, resync_interval=0, ksparse_prob=0.0,
            ksparse_k=8, pair_mode=1, pairs=None, precision="fp32", tape=None, step_offset=0, pair_variant=0,
            trace=False, x_final=False, threads=None):
    """CPU CHR.  A (m, d); X0 (nchains, d) or (d,); returns samples (nspc*nchains, d) float64
    [, trace (nchains, steps, 2)] [, X_final (nchains, d)]."""
    A = np.asfortranarray(np.asarray(A, dtype=np.float64))
    m, d = A.shape
    b = np.ascontiguousarray(np.asarray(b, dtype=np.float64).reshape(-1))
    X = np.asarray(X0, dtype=np.float64)
    if X.ndim == 1:
        X = np.broadcast_to(X, (nchains, d))
    X = np.ascontiguousarray(X)
    samples = np.zeros((nspc * nchains, d), dtype=np.float64)
    tr = np.zeros((nchains, nspc * thinning, 2), dtype=np.int32) if trace else None
    xf = np.zeros((nchains, d), dtype=np.float64) if x_final else None
    pi = pj = pc = ps = None
    npairs = 0
    if pairs is not None:
        pi = np.ascontiguousarray(np.asarray(pairs[0], dtype=np.int32))
        pj = np.ascontiguousarray(np.asarray(pairs[1], dtype=np.int32))
        pc = np.ascontiguousarray(np.asarray(pairs[2], dtype=np.float64))
        ps = np.ascontiguousarray(np.asarray(pairs[3], dtype=np.float64))
        npairs = len(pi)
    tape_arr = None
    stride = 0
    rng = 0
    if tape is not None:
        tape_arr = np.ascontiguousarray(np.asarray(tape, dtype=np.float64))
        stride = tape_arr.shape[1]
        rng = 1
    prec = 1 if precision == "fp64" else 0
    nthreads = threads or os.cpu_count() or 1
    st = load().oracle_chr_run(m, d, _p(A), m, _p(b), _p(X), d, int(nspc), int(thinning), int(nchains),
                               int(seed) & 0xFFFFFFFFFFFFFFFF, float(pair_prob), int(resync_interval),
                               float(ksparse_prob), int(ksparse_k), int(pair_mode), _p(pi), _p(pj), _p(pc), _p(ps),
                               npairs, prec, rng, _p(tape_arr), stride, int(step_offset), int(pair_variant),
                               _p(samples), _p(xf), _p(tr), int(nthreads))
    if st != 0:
        raise RuntimeError(f"oracle_chr_run failed with status {st}")
    out = [samples]
    if trace:
        out.append(tr)
    if x_final:
        out.append(xf)
    return out[0] if len(out) == 1 else tuple(out)


def ess(samples, n_chains, layout=1):
    s = np.ascontiguousarray(np.asarray(samples, dtype=np.float32))
    N, dim = s.shape
    out = np.empty((dim, n_chains), dtype=np.float64)
    st = load().oracle_ess(_p(s), N, dim, n_chains, layout, _p(out))
    if st:
        raise RuntimeError("oracle_ess failed")
    return out


def split_rhat(samples, n_chains, layout=1):
    s = np.ascontiguousarray(np.asarray(samples, dtype=np.float32))
    N, dim = s.shape
    out = np.empty(dim, dtype=np.float64)
    st = load().oracle_split_rhat(_p(s), N, dim, n_chains, layout, _p(out))
    if st:
        raise RuntimeError("oracle_split_rhat failed")
    return out


def ess_series(x):
    x = np.ascontiguousarray(np.asarray(x, dtype=np.float64))
    return load().oracle_ess_series(_p(x), len(x))


# ---------------------------------------------------------------- reference
REF_LIB = HERE / "_ref" / "libnaja_ref.so"
_ref = None


def reference_available() -> bool:
    return REF_LIB.exists()


def _load_ref():
    global _ref
    if _ref is None:
        lib = C.CDLL(str(REF_LIB))
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        lib.ref_chr_run.argtypes = [vp, i, i, vp, vp, i, i, i, i, i, d, i, d, i, i, vp, vp, vp, vp, i,
                                    vp, i, vp, vp, vp, vp]
        lib.ref_chr_run.restype = i
        lib.ref_last_error.restype = C.c_char_p
        _ref = lib
    return _ref


def reference_chr_run(A, b, X0, nspc, thinning, nchains, *, tpb=128, seed=0, pair_prob=0.0, resync_interval=0,
                      ksparse_prob=0.0, ksparse_k=8, pair_mode=1, pairs=None, T=None, shift=None,
                      want_samples=True, want_v=True):
    """The reference's own CoordinateHitAndRun[+backmap_into] (oracle/_ref build).

    Returns (samples (nspc*nchains, d) or None, V (nspc*nchains, n) or None, sampling_ms)."""
    A = np.asfortranarray(np.asarray(A, dtype=np.float64))
    m, d = A.shape
    b = np.ascontiguousarray(np.asarray(b, dtype=np.float64).reshape(-1))
    X = np.asarray(X0, dtype=np.float64)
    if X.ndim == 1:
        X = np.broadcast_to(X, (nchains, d))
    X = np.ascontiguousarray(X)  # (nchains, d) row-major == d x nchains column-major
    N = nspc * nchains
    S = np.empty((N, d), dtype=np.float64) if want_samples else None
    V = Tm = sh = None
    n = 0
    if T is not None:
        Tm = np.asfortranarray(np.asarray(T, dtype=np.float64))
        n = Tm.shape[0]
        sh = np.ascontiguousarray(np.asarray(shift, dtype=np.float64))
        V = np.empty((N, n), dtype=np.float64) if (want_samples and want_v) else None
    pi = pj = pc = ps = None
    npairs = 0
    if pairs is not None:
        pi = np.ascontiguousarray(np.asarray(pairs[0], dtype=np.int32))
        pj = np.ascontiguousarray(np.asarray(pairs[1], dtype=np.int32))
        pc = np.ascontiguousarray(np.asarray(pairs[2], dtype=np.float64))
        ps = np.ascontiguousarray(np.asarray(pairs[3], dtype=np.float64))
        npairs = len(pi)
    ms = C.c_double(0.0)
    lib = _load_ref()
    st = lib.ref_chr_run(_p(A), m, d, _p(b), _p(X), int(nspc), int(thinning), int(nchains), int(tpb), int(seed),
                         float(pair_prob), int(resync_interval), float(ksparse_prob), int(ksparse_k), int(pair_mode),
                         _p(pi), _p(pj), _p(pc), _p(ps), npairs, _p(Tm), n, _p(sh), _p(S), _p(V), C.byref(ms))
    if st != 0:
        raise RuntimeError("reference run failed: " + lib.ref_last_error().decode())
    return S, V, ms.value


def ess_fft(samples, n_chains, layout=1):
    """Geyer ESS per (dim, chain) with an FFT autocovariance (numpy, FP64).

    The same estimator as `ess` (mcmc.cpp:59-76), evaluated for whole
    batches of series at once; used where the direct-sum oracle would be too
    slow (long, slowly mixing chains)."""
    s = np.asarray(samples, dtype=np.float64)
    N, dim = s.shape
    spc = N // n_chains
    if layout == 1:
        x = s[: spc * n_chains].reshape(spc, n_chains, dim).transpose(2, 1, 0)  # dim, chain, t
    else:
        x = s[: spc * n_chains].reshape(n_chains, spc, dim).transpose(2, 0, 1)
    out = np.empty((dim, n_chains))
    nfft = 1 << int(np.ceil(np.log2(2 * spc)))
    for d0 in range(0, dim, 64):
        blk = x[d0:d0 + 64]
        y = blk - blk.mean(axis=2, keepdims=True)
        f = np.fft.rfft(y, nfft, axis=2)
        acov = np.fft.irfft(f * np.conj(f), nfft, axis=2)[:, :, :spc] / spc
        var = acov[:, :, 0]
        rho = acov / np.where(var > 1e-30, var, 1.0)[:, :, None]
        kmax = spc // 2
        pairs = rho[:, :, 1:2 * kmax - 1:2][:, :, : kmax - 1] + rho[:, :, 2:2 * kmax:2][:, :, : kmax - 1]
        neg = pairs < 0
        first = np.where(neg.any(axis=2), neg.argmax(axis=2), pairs.shape[2])
        csum = np.concatenate([np.zeros(pairs.shape[:2] + (1,)), np.cumsum(pairs, axis=2)], axis=2)
        tau = 1.0 + 2.0 * np.take_along_axis(csum, first[:, :, None], axis=2)[:, :, 0]
        tau = np.maximum(tau, 1.0)
        e = spc / tau
        e[var < 1e-30] = 1.0
        out[d0:d0 + 64] = e
    if spc < 4:
        out[:] = spc
    return out
