#!/usr/bin/env python
"""Benchmark of the CHR sampler on the genome-shaped workload.

Workload (one "step" = one full sampling job): the seeded genome-shaped
polytope n=2600 reactions, d=700, A=[T;-T] (m=5200), T 8% dense N(0,1),
bounds log-uniform on [1,1000]; 16 chains x 12500 samples, thinning 116,
pair-prob 0.3, start y=0, followed by the backmap V = T y + shift of all
200,000 samples to n=2600.  Synthetic data stands in for a rounded
genome-scale model (none ships with the reference).

The headline samples the polytope rounded by its whole Dikin ellipsoid
(y = M z + c, M = H^-1/2 at the analytic centre; --rounding): the chains run
in z on A M, every sample is mapped to y = M z + c (FP64 kernel) for the
metric and to reaction space with the composed T' = T M, shift' = T c +
shift.  The affine map leaves the uniform target unchanged.

value  = chain-correct min-ESS / second of the timed job (ESS per dim summed
         over de-interleaved chains, min over dims, in y; seconds = sampling +
         maps with inputs resident in HBM), gated by split-R-hat and bounds
         violations, which the line reports; `plain` repeats it without the
         rounding, `gate_run` samples on until split-R-hat < 1.01.
e2e    = the same min-ESS over the job run from host buffers through the C
         ABI: rounding, polytope upload, sampling, backmap, and the
         back-transformed samples copied to pinned host memory (wall clock).
roofline: the step kernel, algorithmic bytes per CHR step
         4*m*(1+p_pair) + 4*d/thinning (one FP32 column of A per coordinate,
         two per pair step, plus the amortised sample write) over its
         CUDA-event duration, against MEASURED_PEAKS.json hbm_gbs.
cpu_baseline: the CPU oracle (same algorithm, same tier, bit-identical
         trajectory) on a bounded sample of the workload on the host cores;
         its min-ESS/s is the GPU run's min-ESS per CHR step times the CPU's
         CHR steps per second.

`--impl reference` times the reference's own sampler (see _reference_arm).
Multi-GPU (torchrun): each rank runs an independent replica with its own
chain streams (weak scaling, no data-path collective); per-dim ESS sums are
combined after timing.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "min-ESS/sec at split-R-hat<1.01, learned-rounded vs plain CHR, 1 B200"
UNIT = "min-ESS/s"
L2_FLUSH_BYTES = 256 << 20
# DRAM bytes (read + write) of one launch of the headline step kernel,
# chr_kernel<float, 448, 3, uniform> on the rounded genome-shaped job (n
# 2600, d 700, 16 chains x 12,500 samples, thinning 116, pair 0.3, resync
# 2048, FP32, Philox seed 0), which runs as 709 launches of 2,048 steps:
# one 1-pass ncu capture of a whole job's launches gave
# dram__bytes_read.sum 10.766 GB + dram__bytes_write.sum 22.5 KB over 709.
# Reported as roofline.traffic only for that exact workload.
HEADLINE_TRAFFIC_BYTES = 10.766e9 / 709 + 22.5e3 / 709


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self._t = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


class Workload:
    def __init__(self, a):
        from naja_b200 import synth

        self.n, self.d = a.n, a.d
        g = synth.genome_shaped(n=a.n, d=a.d, density=0.08, seed_T=0, seed_u=1)
        self.g = g
        self.A, self.b, self.T, self.shift, self.start = g["A"], g["b"], g["T"], g["shift"], g["start"]
        self.m = self.A.shape[0]
        self.nchains, self.nspc, self.thin, self.pair = a.nchains, a.nspc, a.thinning, a.pair_prob
        self.steps = self.nchains * self.nspc * self.thin
        self.bytes_per_step = 4.0 * self.m * (1.0 + self.pair) + 4.0 * self.d / self.thin
        # what the compressed-column kernel reads per step: a column's (value, row) entries, padded to pairs
        nz = (self.A.astype(np.float32) != 0).sum(axis=0)
        entries = np.maximum(2, nz + (nz & 1)).mean()
        self.compressed_bytes_per_step = 8.0 * entries * (1.0 + self.pair) + 4.0 * self.d / self.thin

    def config(self, a):
        return {"workload": f"genome-shaped polytope n={self.n} d={self.d} m={self.m}, {self.nchains} chains x "
                            f"{self.nspc} samples, thinning {self.thin}, pair-prob {self.pair}, backmap to n={self.n}",
                "n": self.n, "d": self.d, "m": self.m, "chains": self.nchains, "samples_per_chain": self.nspc,
                "thinning": self.thin, "pair_prob": self.pair, "precision": a.precision,
                "resync_interval": a.resync, "backmap": a.backmap_mode, "rng": "philox", "step_kernel": a.sparse,
                "rounding": a.rounding,
                "l2": "256 MiB written between timed steps"}


def _gate(torch, W, samples_dev, ess, rhat):
    """split-R-hat and bounds checks on the fp32 output (outside the timed region).

    Polytope rows: A y <= b + 1e-6 max(1, |b|) on every sample.  GEM bounds:
    the reference's rule (src/validate/bounds_check.cpp:8-39): v = T y + shift
    in FP64 from the fp32 samples, violation when max(l - v, v - u) - 1e-6 > 0,
    on <= 1000 evenly spaced samples."""
    A = torch.from_numpy(W.A).to(samples_dev.device)
    b = torch.from_numpy(W.b).to(samples_dev.device)
    tol = 1e-6 * torch.clamp(b.abs(), min=1.0)
    viol = 0
    worst = 0.0
    for s0 in range(0, samples_dev.shape[0], 20000):
        r = samples_dev[s0:s0 + 20000].double() @ A.T - b
        viol += int((r > tol).sum())
        worst = max(worst, float(r.max()))
    step = max(1, samples_dev.shape[0] // 1000)
    y = samples_dev[::step].double()
    T = torch.from_numpy(W.T).to(y.device)
    v = y @ T.T + torch.from_numpy(W.shift).to(y.device)
    u = torch.from_numpy(W.g["u"]).to(v.device)
    lo = torch.from_numpy(W.g["l"]).to(v.device)
    gem = torch.maximum(lo - v - 1e-6, v - u - 1e-6)
    return {"rhat_max": float(np.max(rhat)), "rhat_gate_1_01": bool(np.max(rhat) < 1.01),
            "bounds_violations": viol, "bounds_worst": worst,
            "gem_bounds_violations": int((gem > 0).sum()), "gem_bounds_checked": int(gem.numel())}


def _backmap_error(torch, Tm, shift, samples_dev, V_dev, mode):
    """Backmap error of `mode` against an FP64 GEMM of the same samples on
    4096 evenly spaced ones."""
    step = max(1, samples_dev.shape[0] // 4096)
    y = samples_dev[::step].double()
    T = torch.from_numpy(Tm).to(y.device)
    sh = torch.from_numpy(shift).to(y.device)
    ref = y @ T.T + sh
    got = V_dev[::step].double()
    scale = y.abs() @ T.abs().T + sh.abs()
    err = (got - ref).abs()
    nz = ref.abs() > 1e-3 * ref.abs().max()
    rel = err[nz] / ref.abs()[nz]
    return {"mode": mode, "samples": int(y.shape[0]), "max_rel": float(rel.max()),
            "rms_rel": float(torch.sqrt((rel ** 2).mean())),
            "max_normalised": float((err / scale.clamp(min=1e-300)).max()),
            "note": "relative error over |v| > 1e-3 max|v|; normalised = |err| / (|T||y| + |shift|)"}


def _chr_launches(W, a, choice):
    """Kernels one CHR run launches: a run with a recompute interval K
    shorter than the run and m d >= 2^19 runs in segments of K steps, each a
    slack-recompute kernel and a step kernel (either step kernel)."""
    total = W.nspc * W.thin
    if 0 < a.resync < total and W.m * W.d >= (1 << 19):
        return 2 * (-(-total // a.resync))
    return 1


def _headline_traffic(a, W, choice):
    """The captured DRAM bytes of the headline launch, where this run is that
    launch's workload (else None: traffic was not captured for it)."""
    same = (W.n, W.d, W.nchains, W.nspc, W.thin, W.pair, a.resync, a.precision, a.seed, a.rounding) == \
        (2600, 700, 16, 12500, 116, 0.3, 2048, "fp32", 0, "dikin_full")
    return HEADLINE_TRAFFIC_BYTES if same and choice["kernel"] != "columns" and choice["threads"] == 448 else None


def _dgemm_backmap_ms(torch, T_dev, sh_dev, Z):
    """The reference's backmap (cuBLAS DGEMM V = T Y, then + shift per
    column; src/gpu/backmap.cu:20-48) on the same samples, FP64 operands
    prepared untimed; mean of three after one warm-up."""
    Zd = Z.double()
    Td = T_dev.double()
    out = torch.empty((Z.shape[0], Td.shape[0]), dtype=torch.float64, device=Z.device)
    ms = []
    for k in range(4):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(Zd, Td.T, out=out)
        out.add_(sh_dev.double())
        e1.record()
        torch.cuda.synchronize()
        if k:
            ms.append(e0.elapsed_time(e1))
    del Zd, Td, out
    return statistics.mean(ms)


def _backmap_roofline(W, ms, mode):
    flops = 2.0 * W.n * W.d * W.nspc * W.nchains
    p = ROOT / "MEASURED_PEAKS.json"
    bf16 = float(json.loads(p.read_text())["bf16_tflops"]) if p.exists() else 1590.0
    src = "measured" if p.exists() else "fallback"
    if mode == "fp64":
        return {"bound": "fp64 SIMT", "achieved": flops / (ms / 1e3) / 1e12, "unit": "TFLOP/s", "flops": flops}
    peak = bf16 if mode == "bf16x3" else bf16 / 2.0
    ach = flops / (ms / 1e3) / 1e12
    return {"bound": "tensor", "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak, "flops": flops,
            "peak_source": f"{src} bf16" + ("" if mode == "bf16x3" else " / 2 (tf32 rate)"),
            "note": "algorithmic FLOPs 2 n d N; the three split products are not credited"}


def _r(x, n=4):
    """x to n significant digits (numbers only)."""
    if isinstance(x, float):
        return float(f"{x:.{n}g}")
    return x


def _compact(line):
    """The printed line: every section summarised so that the whole line stays
    near 3,000 characters (the full sections go to --detail-file)."""
    out = {k: line[k] for k in line if k not in _SECTIONS}
    # the workload string already states the sizes
    out["config"] = {k: v for k, v in line["config"].items()
                     if k not in ("n", "d", "m", "chains", "samples_per_chain", "thinning", "pair_prob")}
    rf = dict(line["roofline"])
    for k in ("bytes_definition", "compressed_bytes_per_chr_step", "chr_steps_per_launch", "kernel_threads"):
        rf.pop(k, None)
    if "rounding" in line:
        out.pop("rounding")
        out["rounding_s"] = _r(line["rounding"].get("seconds", 0.0), 3)
    out["roofline"] = {k: _r(v) for k, v in rf.items()}
    for k in ("value", "ms_per_step", "chr_steps_per_s", "min_ess"):
        out[k] = _r(line[k], 6)
    g = line.get("gate")
    if g:
        out["gate"] = {k: _r(v) for k, v in g.items() if k in ("rhat_max", "rhat_gate_1_01", "bounds_violations",
                                                                 "gem_bounds_violations")}
    bm = line.get("backmap")
    if bm:
        out["backmap"] = {"mode": bm["mode"], "ms": _r(bm["ms"]), "max_rel": _r(bm["error_vs_fp64"]["max_rel"], 3),
                          "tflops": _r(bm["roofline"]["achieved"], 3), "frac": _r(bm["roofline"].get("frac", 0.0), 3),
                          "y_map_ms": _r(bm.get("y_map_ms", 0.0), 3), "dgemm_ms": _r(bm.get("cublas_dgemm_ms"), 3)}
    if "e2e" in line:
        out["e2e"] = {k: _r(v, 5) for k, v in line["e2e"].items() if k != "timing"}
    if "cpu_baseline" in line:
        cb = line["cpu_baseline"]
        out["cpu_baseline"] = {"value": _r(cb["value"]), "unit": cb["unit"], "cores": cb["cores"], "kind": cb["kind"],
                               "sample": cb["sample"].split(" of the same workload")[0]}
    if "plain" in line:
        p = line["plain"]
        out["plain"] = {"value": _r(p["value"]), "rhat_max": _r(p["rhat_max"]), "M_steps_s": _r(p["chr_steps_per_s"] / 1e6),
                        "kernel": p["roofline"]["kernel"], "frac": _r(p["roofline"]["frac"], 3)}
    if "fp64_tier" in line:
        f = line["fp64_tier"]
        out["fp64_tier"] = {"value": _r(f["value"]), "ms": _r(f["ms_per_job"]), "rhat_max": _r(f["rhat_max"])}
    if "unit_cube" in line:
        u = line["unit_cube"]
        out["unit_cube"] = {"M_steps_s": _r(u["chr_steps_per_s"] / 1e6), "mean_dev_se": _r(u["mean_max_dev_in_se"], 3),
                            "var_dev_se": _r(u["var_max_dev_in_se"], 3), "rhat_max": _r(u["rhat_max"])}
    if "batched" in line:
        b = line["batched"]
        sh = b["shape"]
        out["batched"] = {"M_steps_s": _r(b["chr_steps_per_s"] / 1e6), "frac": _r(b["roofline"]["frac"], 3),
                          "shape": f"{sh['threads']}t x{sh['slots']} {'columns' if sh['sparse'] else 'dense'}"}
    if "gate_run" in line:
        out["gate_run"] = {k: {"reached": r["reached"], "s": _r(r["seconds"], 3), "rhat": _r(r["rhat_max"]),
                               "min_ess_s": _r(r["min_ess_per_s"]), "viol": r["bounds_violations"]}
                           for k, r in line["gate_run"]["methods"].items()}
    if "precision_study" in line:
        ps = line["precision_study"]
        out["precision_study"] = {
            "tier,K,t/fp64,drift_rel,agree_step,viol": [
                [r["tier"], r["K"], _r(r.get("time_vs_fp64", 1.0), 3), _r(r["slack_drift"]["max_rel"], 2),
                 r.get("agree_1e-3_through_step_min", 0), r["bound_violations"]] for r in ps["chr"]],
            # C3 backmap ms / max rel. error per mode: tc modes only (the full table is in the detail file)
            "bm_ms_maxrel": {m: [_r(v["ms_200k"], 3), _r(v["max_rel"], 2)] for m, v in ps["backmap"].items()
                             if m in ("bf16x3", "tf32x3")}}
    if "learned_rounding" in line:
        lr = line["learned_rounding"]
        out["learned_rounding"] = {
            "train": lr["train"]["variants"], "test": lr["test_variants"],
            "mse": [_r(lr["test_mse_std_units"]), _r(lr["test_mse_mean_predictor"])],
            "min_ess_s,rhat,passed": {k: [_r(v["min_ess_per_s_median"]), _r(v["rhat_max"]), v["passed"]]
                                      for k, v in lr["methods"].items()},
            **{k: _r(v, 3) for k, v in lr.items() if k.startswith("learned_vs_")}}
    return out


_SECTIONS = ("roofline", "gate", "backmap", "e2e", "cpu_baseline", "plain", "fp64_tier", "unit_cube", "batched",
             "gate_run", "precision_study", "learned_rounding", "reference_semantics_validate", "job_ms", "chr_ms")


def _stats(v):
    """min / median / max of per-step times (the per-step lists go to --detail-file)."""
    return {"min": float(min(v)), "median": float(statistics.median(v)), "max": float(max(v)), "n": len(v)}


def _cpu_baseline(W, a, min_ess_per_step, R):
    """The oracle on the host cores, on the polytope the headline samples
    (rounded when it is), one thread per chain: the oracle parallelises over
    chains, so at most `chains` threads are used whatever the host has."""
    import oracle.oracle as O

    cores = min(os.cpu_count() or 1, W.nchains)
    nspc = 2
    t0 = time.perf_counter()
    O.chr_run(R.A, R.b, R.z0, nspc, W.thin, W.nchains, seed=a.seed, pair_prob=W.pair, resync_interval=a.resync,
              precision=a.precision, threads=cores)
    dt = time.perf_counter() - t0
    nspc = max(2, min(W.nspc, int(nspc * a.cpu_seconds / max(dt, 1e-3))))
    t0 = time.perf_counter()
    O.chr_run(R.A, R.b, R.z0, nspc, W.thin, W.nchains, seed=a.seed, pair_prob=W.pair, resync_interval=a.resync,
              precision=a.precision, threads=cores)
    dt = time.perf_counter() - t0
    steps_s = W.nchains * nspc * W.thin / dt
    return {"value": min_ess_per_step * steps_s, "unit": UNIT, "cores": cores, "kind": "port",
            "steps_per_s": steps_s, "host_cores": os.cpu_count(),
            "sample": f"{W.nchains} chains x {nspc} samples (thinning {W.thin}) of the same workload, CPU oracle "
                      f"{a.precision} tier, {cores} threads, {dt:.1f} s; min-ESS/s = GPU min-ESS per CHR step x "
                      f"CPU CHR steps/s (identical trajectory)"}


def replica_seed(seed: int, rank: int) -> int:
    """Philox key of rank `rank`'s replica: every rank samples the same
    workload from its own streams into its own buffers (weak scaling)."""
    return (int(seed) + 0x9E3779B97F4A7C15 * int(rank)) & 0xFFFFFFFFFFFFFFFF


def reduce_over_ranks(per_dim_ess, total_ms: float, world: int, device):
    """Whole-job figures over the replicas: per-dimension ESS summed over every
    rank's chains, device time the maximum over ranks."""
    import torch

    per_dim = np.asarray(per_dim_ess, dtype=np.float64)
    if world <= 1:
        return per_dim, float(total_ms)
    t = torch.from_numpy(per_dim.copy()).to(device)
    torch.distributed.all_reduce(t)
    m = torch.tensor([float(total_ms)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(m, op=torch.distributed.ReduceOp.MAX)
    return t.cpu().numpy(), float(m.item())


def _ours(a, rank, world):
    import torch

    import naja_b200 as nb
    from naja_b200 import validate as nv

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    from naja_b200 import gate as ng

    W = Workload(a)
    # the rounding y = M z + c, the rounded polytope and the composed backmap
    # T' = T M, shift' = T c + shift are set up once (untimed here; e2e times them)
    R = ng.make_rounding(a.rounding, W.A, W.b, W.start, device=dev.index)
    rounded = R.info["method"] != "identity"
    P = nb.Polytope(R.A, R.b, device=dev.index)
    Tp, shp = R.compose_backmap(W.T, W.shift)
    T_dev = torch.from_numpy(Tp).to(dev)
    sh_dev = torch.from_numpy(shp).to(dev)
    M_dev = torch.from_numpy(np.ascontiguousarray(R.M)).to(dev)
    c_dev = torch.from_numpy(R.c).to(dev)
    x0 = torch.from_numpy(np.broadcast_to(R.z0, (W.nchains, W.d)).copy()).to(dev)
    samples = torch.empty((W.nspc * W.nchains, W.d), dtype=torch.float32, device=dev)
    zbuf = torch.empty_like(samples) if rounded else samples
    V = torch.empty((W.nspc * W.nchains, W.n), dtype=torch.float32, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    seed = replica_seed(a.seed, rank)

    def job():
        P.run(x0, W.nspc, W.thin, W.nchains, out=zbuf, seed=seed, pair_prob=W.pair,
              resync_interval=a.resync, precision=a.precision, sparse=a.sparse, tpb=a.tpb)
        e_mid = torch.cuda.Event(enable_timing=True)
        e_ymap = torch.cuda.Event(enable_timing=True)
        e_mid.record()
        if rounded:
            nb.backmap(M_dev, c_dev, zbuf, mode="fp64", out=samples)  # y = M z + c for the metric
        e_ymap.record()
        nb.backmap(T_dev, sh_dev, zbuf, mode=a.backmap_mode, out=V)  # v = T' z + shift'
        return e_mid, e_ymap

    for _ in range(a.warmup):
        job()
        flush.zero_()
    torch.cuda.synchronize()
    P.check()
    if world > 1:
        torch.distributed.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    mids = []
    with ClockSampler(dev.index if world == 1 else int(os.environ.get("LOCAL_RANK", 0))) as clk:
        torch.cuda.synchronize()
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record()
        for k in range(a.steps):
            ev[k][0].record()
            mids.append(job())
            ev[k][1].record()
            flush.zero_()
        g1.record()
        torch.cuda.synchronize()
    P.check()
    total_ms = g0.elapsed_time(g1)
    job_ms = [ev[k][0].elapsed_time(ev[k][1]) for k in range(a.steps)]
    chr_ms = [ev[k][0].elapsed_time(mids[k][0]) for k in range(a.steps)]
    ymap_ms = [mids[k][0].elapsed_time(mids[k][1]) for k in range(a.steps)]
    bm_ms = [mids[k][1].elapsed_time(ev[k][1]) for k in range(a.steps)]
    # metric on the last job's samples
    ess, rhat = nv.ess_rhat(samples, W.nchains, layout=1)
    per_dim, total_ms = reduce_over_ranks(ess.sum(axis=1), total_ms, world, dev)
    min_ess = float(per_dim.min())
    ms_per_step = total_ms / a.steps
    value = min_ess / (ms_per_step / 1e3)  # min-ESS already sums every rank's chains
    gate = _gate(torch, W, samples, ess, rhat)
    bm_err = _backmap_error(torch, Tp, shp, zbuf, V, a.backmap_mode)
    dgemm_ms = _dgemm_backmap_ms(torch, T_dev, sh_dev, zbuf) if rank == 0 else None
    ref_sem = nv.summary(*nv.ess_rhat(samples, W.nchains, layout=0))
    peak, peak_kind = _peaks()
    choice = P.kernel_choice(W.nspc, W.thin, W.nchains, pair_prob=W.pair, resync_interval=a.resync,
                             precision=a.precision, sparse=a.sparse, tpb=a.tpb)
    chr_mean = statistics.mean(chr_ms)
    achieved = W.bytes_per_step * W.steps / (chr_mean / 1e3) / 1e9
    n_chr = _chr_launches(W, a, choice)
    steps_per_s = W.steps * world / (ms_per_step / 1e3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if a.precision == "fp32" else "f64", "data": "synthetic (seeded genome-shaped generator)",
        "config": W.config(a),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": _headline_traffic(a, W, choice), "peak_source": peak_kind,
                     "kernel": "chr_sparse_kernel" if choice["kernel"] == "columns" else "chr_kernel",
                     "kernel_threads": choice["threads"], "kernel_ms": chr_mean,
                     "bytes_per_chr_step": W.bytes_per_step,
                     "bytes_definition": "4 m (1 + p_pair) + 4 d / thinning: one FP32 column per coordinate step, "
                                         "two per pair step, plus the amortised sample write",
                     "compressed_bytes_per_chr_step": W.compressed_bytes_per_step,
                     # the job's step-kernel launches (one per recompute interval when segmented);
                     # achieved is their aggregate rate, traffic one launch's DRAM bytes
                     "chr_steps_per_launch": a.resync * W.nchains if n_chr > 1 else W.steps,
                     "launches_per_job": n_chr // 2 if n_chr > 1 else 1},
        "chr_steps_per_s": steps_per_s, "min_ess": min_ess,
        "rounding": {k: v for k, v in R.info.items() if k in ("method", "newton_iterations", "seconds")},
        "job_ms": _stats(job_ms), "chr_ms": _stats(chr_ms),
        "gate": gate,
        "backmap": {"mode": a.backmap_mode, "ms": statistics.mean(bm_ms), "error_vs_fp64": bm_err,
                    "roofline": _backmap_roofline(W, statistics.mean(bm_ms), a.backmap_mode),
                    # y = M z + c of the rounded job (FP64 SIMT, for the metric), timed apart
                    "y_map_ms": statistics.mean(ymap_ms),
                    # the reference's backmap_into (src/gpu/backmap.cu:20-48): cuBLAS DGEMM + shift
                    "cublas_dgemm_ms": dgemm_ms},
        "reference_semantics_validate": {k: ref_sem[k] for k in ("status", "ess", "rhat")},
        # per step: the CHR run (one step kernel, or per recompute interval one
        # slack-recompute kernel and one step kernel), the y map (one FP64
        # kernel) when rounded, then the backmap (one FP64 kernel, or operand
        # split x2 + tcgen05 GEMM)
        "gpu_launches": a.steps * (_chr_launches(W, a, choice) + (1 if rounded else 0)
                                   + (1 if a.backmap_mode == "fp64" else 3)),
    }
    line["clocks"] = clk.summary()
    detail = {"job_ms": job_ms, "chr_ms": chr_ms, "backmap_ms": bm_ms, "y_map_ms": ymap_ms}
    if rank == 0 and rounded:
        line["plain"] = _plain_figure(a, W, torch, dev)
    if rank == 0 and a.fp64_figure:
        line["fp64_tier"] = _fp64_figure(a, W, P, x0, torch, dev, M_dev, c_dev, T_dev, sh_dev)
    if rank == 0 and a.cube:
        line["unit_cube"] = _unit_cube(a, torch, dev)
    if a.e2e and rank == 0:
        line["e2e"] = _e2e(a, W, torch, dev, min_ess)
    if rank == 0 and world == 1 and not a.no_cpu:
        line["cpu_baseline"] = _cpu_baseline(W, a, min_ess / W.steps, R)
    if rank == 0 and a.batch_models > 0:
        line["batched"] = _batched(a, torch, dev)
    if rank == 0 and a.gate_budget_s > 0:
        line["gate_run"] = _gate_run(a)
    if rank == 0 and a.precision_figures:
        line["precision_study"] = _precision_study(a)
    if rank == 0 and a.learned_train > 0:
        line["learned_rounding"], detail["learned_rounding"] = _learned(a)
    detail["line"] = line
    if rank == 0 and a.detail_file:
        Path(a.detail_file).parent.mkdir(parents=True, exist_ok=True)
        Path(a.detail_file).write_text(json.dumps(detail))
    P.close()
    return _compact(line)


def _e2e(a, W, torch, dev, min_ess):
    """The same job from host buffers through the public API, wall-clock per
    job: the rounding (FP64 on the GPU for dikin_full: analytic centre,
    barrier Hessian, its inverse square root, A M and T M), the polytope's
    creation, then
    sampling, backmap and the copy of every back-mapped sample to pinned
    host memory overlapped chunk by chunk (naja_chr_run_backmapped)."""
    import naja_b200 as nb
    from naja_b200 import gate as ng
    from naja_b200.pipeline import sample_backmapped

    pinned_out = torch.empty((W.nspc * W.nchains, W.n), dtype=torch.float32, pin_memory=True)
    times, h2d = [], 0
    for k in range(a.warmup + a.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        R = ng.make_rounding(a.rounding, W.A, W.b, W.start, device=dev.index)
        z0 = np.ascontiguousarray(np.broadcast_to(R.z0, (W.nchains, W.d)))
        dv = R.info.get("dev")
        if dv is not None:
            # rounded on the GPU: compose T' = T M, shift' = T c + shift there too
            T_d = torch.from_numpy(W.T).to(dev)
            Tp, shp = T_d @ dv["M"], T_d @ dv["c"] + torch.from_numpy(W.shift).to(dev)
            P = nb.Polytope(dv["A"], dv["b"], device=dev.index)
            h2d = W.A.nbytes + W.b.nbytes + W.T.nbytes + W.shift.nbytes + z0.nbytes
        else:
            Tp, shp = R.compose_backmap(W.T, W.shift)
            P = nb.Polytope(R.A, R.b, device=dev.index)
            h2d = R.A.nbytes + R.b.nbytes + z0.nbytes + Tp.nbytes + shp.nbytes
        # sampling, backmap and copy to host overlapped chunk by chunk (same samples as one launch)
        sample_backmapped(P, Tp, shp, z0, W.nspc, W.thin, W.nchains, pinned_out, mode=a.backmap_mode,
                          seed=a.seed, pair_prob=W.pair, resync_interval=a.resync, precision=a.precision,
                          sparse=a.sparse, tpb=a.tpb)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        P.close()
        if k >= a.warmup:
            times.append(dt * 1e3)
    ms = statistics.mean(times)
    return {"value": min_ess / (ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(pinned_out.numel() * 4), "ms_per_step": ms,
            "timing": "wall clock per job with a device synchronise on both sides; rounding (FP64 on the GPU for "
                      "dikin_full) inside the timed region"}


def _plain_figure(a, W, torch, dev):
    """The same job without rounding (plain CHR on the polytope as given,
    the compressed-column kernel): min-ESS/s of the last of two timed jobs
    and that kernel's roofline."""
    import naja_b200 as nb
    from naja_b200 import validate as nv

    P = nb.Polytope(W.A, W.b, device=dev.index)
    x0 = torch.from_numpy(np.broadcast_to(W.start, (W.nchains, W.d)).copy()).to(dev)
    samples = torch.empty((W.nspc * W.nchains, W.d), dtype=torch.float32, device=dev)
    V = torch.empty((W.nspc * W.nchains, W.n), dtype=torch.float32, device=dev)
    T_dev = torch.from_numpy(W.T).to(dev)
    sh_dev = torch.from_numpy(W.shift).to(dev)
    chr_ms, job_ms = [], []
    for k in range(3):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        P.run(x0, W.nspc, W.thin, W.nchains, out=samples, seed=a.seed, pair_prob=W.pair, resync_interval=a.resync,
              precision=a.precision, sparse=a.sparse, tpb=a.tpb)
        e1.record()
        nb.backmap(T_dev, sh_dev, samples, mode=a.backmap_mode, out=V)
        e2.record()
        torch.cuda.synchronize()
        if k:
            chr_ms.append(e0.elapsed_time(e1))
            job_ms.append(e0.elapsed_time(e2))
    P.check()
    ess, rhat = nv.ess_rhat(samples, W.nchains, layout=1)
    min_ess = float(ess.sum(axis=1).min())
    choice = P.kernel_choice(W.nspc, W.thin, W.nchains, pair_prob=W.pair, resync_interval=a.resync,
                             precision=a.precision, sparse=a.sparse, tpb=a.tpb)
    peak, peak_kind = _peaks()
    cm = statistics.mean(chr_ms)
    ach = W.bytes_per_step * W.steps / (cm / 1e3) / 1e9
    P.close()
    return {"value": min_ess / (statistics.mean(job_ms) / 1e3), "unit": UNIT, "min_ess": min_ess,
            "rhat_max": float(rhat.max()), "ms_per_job": statistics.mean(job_ms), "chr_ms": cm,
            "chr_steps_per_s": W.steps / (cm / 1e3),
            "roofline": {"kernel": "chr_sparse_kernel" if choice["kernel"] == "columns" else "chr_kernel",
                         "threads": choice["threads"], "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak, "peak_source": peak_kind,
                         "compressed_bytes_per_chr_step": W.compressed_bytes_per_step}}


def _batched(a, torch, dev):
    """Conditioned-variant batch: 64 models = the genome-shaped polytope plus
    0-200 extra rows each (bounds of up to 100 reactions tightened by a factor
    in [0.05, 0.5], the extra-row rule of cmd_prepare.cpp:111-156), 8 chains x
    4000 samples per model, thinning 116, pair-prob 0.3 (the genome workload's
    settings), all in one persistent launch replayed from a CUDA graph; launch
    shape from the autotuner.  Separate polytopes per model: A is read from
    HBM (the batch's FP32 A is ~1 GB, far beyond L2)."""
    import naja_b200 as nb
    from naja_b200 import autotune, synth
    from naja_b200.batch import Batch

    base = synth.genome_shaped(n=a.n, d=a.d, density=0.08, seed_T=0, seed_u=1)
    variants = synth.conditioned_variants(base, a.batch_models, max_reactions=100, seed=2)
    polys = [nb.Polytope(np.vstack([base["A"], v["extra_A"]]), np.concatenate([base["b"], v["extra_b"]]),
                         device=dev.index) for v in variants]
    B = Batch(polys)
    nch, nspc, thin = a.batch_chains, a.batch_nspc, a.thinning
    X = [torch.zeros((nch, a.d), dtype=torch.float64, device=dev) for _ in polys]
    outs = [torch.empty((nspc * nch, a.d), dtype=torch.float32, device=dev) for _ in polys]
    kw = dict(seed=a.seed, pair_prob=a.pair_prob, resync_interval=a.resync)
    if a.batch_shape:
        from naja_b200.batch import Shape

        shape, table = Shape(*(int(v) for v in a.batch_shape.split(","))), {}
    else:
        shape, table = autotune.tune(B, X, outs, nch, thin, **kw)
    g = B.capture(X, outs, nspc, thin, nch, shape=shape, **kw)
    g.launch()
    torch.cuda.synchronize()
    g.check()
    times = []
    for _ in range(max(1, a.steps)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g.launch()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    g.check()
    ms = statistics.mean(times)
    ms_rows = [p.m for p in polys]
    steps = len(polys) * nch * nspc * thin
    bytes_total = sum(nch * nspc * thin * (4.0 * m * (1 + a.pair_prob) + 4.0 * a.d / thin) for m in ms_rows)
    peak, src = _peaks()
    ach = bytes_total / (ms / 1e3) / 1e9
    g.close()
    return {"workload": f"{len(polys)} conditioned variants (m {min(ms_rows)}-{max(ms_rows)}) x {nch} chains x "
                        f"{nspc} samples, thinning {thin}, pair-prob {a.pair_prob}, one persistent launch in a CUDA graph",
            "shape": {"threads": shape.threads, "slots": shape.slots, "slack_smem": shape.slack_smem,
                      "ctas_per_sm": shape.ctas_per_sm, "sparse": shape.sparse},
            "ms": ms, "chr_steps_per_s": steps / (ms / 1e3),
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                         "peak_source": src, "bytes_per_chr_step": bytes_total / steps},
            "autotune_top": sorted(({"shape": str(k), "M_steps_per_s": v / 1e6} for k, v in table.items()),
                                   key=lambda r: -r["M_steps_per_s"])[:5]}


def _gate_run(a):
    """The metric at its gate: the genome-shaped workload's 16 chains
    (thinning 116, pair-prob 0.3, resync 2048, FP32 tier, Philox seed 0)
    continued chunk by chunk (12,500 samples per chain per chunk) until
    split-R-hat < 1.01 with no bound violations, or until the time budget;
    per rounding: plain (none), the reference's Dikin preconditioner and the
    whole-ellipsoid Dikin rounding.  Seconds include computing the rounding,
    every chunk's sampling and back-map to y, and the R-hat checks."""
    from naja_b200 import gate, synth

    g = synth.genome_shaped(n=a.n, d=a.d, density=0.08, seed_T=0, seed_u=1)
    out = {"workload": f"genome-shaped n={a.n} d={a.d}, {a.nchains} chains, chunks of {a.nspc} samples x thinning "
                       f"{a.thinning}, pair-prob {a.pair_prob}, until split-R-hat < 1.01 or {a.gate_budget_s:.0f} s",
           "methods": {}}
    for method, adapt in (("none", 0), ("dikin", 0), ("dikin_full", 0)):
        r = gate.sample_to_gate(g["A"], g["b"], g["start"], method=method, adapt_after=adapt, nchains=a.nchains,
                                thinning=a.thinning, chunk_nspc=a.nspc, pair_prob=a.pair_prob,
                                resync_interval=a.resync, seed=a.seed, budget_s=a.gate_budget_s)
        r["curve"] = [[round(c["seconds"], 2), round(c["rhat_max"], 4)] for c in r["curve"]]
        out["methods"][r["method"]] = r
    m = out["methods"]
    best = max(m.values(), key=lambda r: (r["reached"], r["min_ess_per_s"]))
    out["best"] = best["method"]
    out["reached"] = [k for k, r in m.items() if r["reached"]]
    return out


def _precision_study(a):
    """FP32 tier with its FP64 slack recompute every K steps against the FP64
    tier, and the split-precision backmap against FP64, on the genome-shaped
    polytope at d=1500, n=7000 (m=14000): 8 chains x 200 samples, thinning
    256 (51,200 steps, a multiple of every K), pair-prob 0.3, identical
    Philox streams for every run.  Per run: kernel time, polytope bound
    violations (A y <= b + 1e-6 max(1,|b|)); the slack drift after the last
    K steps, |slack32 - (b - A x)| in FP64 at the final state (max, RMS, max
    relative to max(1, |b|)); the position divergence from the FP64 run (max
    and RMS over all saved coordinates relative to the coordinate's range in
    the FP64 run) and the horizon over which positions agree (the step of a
    chain's last saved sample before the first one that differs by more than
    1e-3 of a coordinate's range: minimum and median over chains).  Backmap: max / RMS
    relative error over 20,000 samples (|v| > 1e-3 max|v|) and the time of
    200,000 samples per mode."""
    import torch

    from naja_b200 import Polytope, backmap, synth

    g = synth.genome_shaped(n=7000, d=1500, density=0.08, seed_T=0, seed_u=1)
    A, b = g["A"], g["b"]
    dev = torch.device("cuda:0")
    P = Polytope(A, b)
    nch, nspc, thin, d = 8, 200, 256, 1500
    X0 = np.zeros((nch, d))
    At = torch.from_numpy(A).to(dev)
    bt = torch.from_numpy(b).to(dev)
    tol = 1e-6 * torch.clamp(bt.abs(), min=1.0)

    def run(precision, K):
        P.run(X0, 2, thin, nch, seed=a.seed, pair_prob=0.3, precision=precision, resync_interval=K)  # warm
        out = torch.empty((nspc * nch, d), dtype=torch.float64, device=dev)
        xf = torch.empty((nch, d), dtype=torch.float64, device=dev)
        sf = torch.empty((nch, A.shape[0]), dtype=torch.float64 if precision == "fp64" else torch.float32,
                         device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        P.run(X0, nspc, thin, nch, seed=a.seed, pair_prob=0.3, precision=precision, resync_interval=K, out=out,
              out_dtype="f64", X_final=xf, slack_final=sf)
        e1.record()
        torch.cuda.synchronize()
        P.check()
        r = out @ At.T - bt
        exact = bt - xf @ At.T
        drift = (sf.double() - exact).abs()
        return out, e0.elapsed_time(e1), int((r > tol).sum()), float(r.max()), {
            "max": float(drift.max()), "rms": float(drift.pow(2).mean().sqrt()),
            "max_rel": float((drift / torch.clamp(bt.abs(), min=1.0)).max())}

    ref, t64, v64, w64, dr64 = run("fp64", 0)
    span = (ref.max(dim=0).values - ref.min(dim=0).values).clamp(min=1e-12)
    rows = [{"tier": "fp64", "K": 0, "ms": t64, "bound_violations": v64, "worst_violation": w64,
             "slack_drift": dr64}]
    for K in (0, 1024, 256, 64):
        y, t, v, w, dr = run("fp32", K)
        rel = (y - ref).abs() / span
        per_sample = rel.view(nspc, nch, d).amax(dim=2)  # (sample, chain)
        off = (per_sample > 1e-3).cpu().numpy()
        first = np.where(off.any(axis=0), off.argmax(axis=0), nspc)  # first diverging saved sample per chain
        # saved sample s follows step s * thin + 1: agreement holds through the step of the sample before
        horizon = np.where(first < nspc, (first - 1) * thin + 1, nspc * thin)
        rows.append({"tier": "fp32", "K": K, "ms": t, "time_vs_fp64": t / t64, "bound_violations": v,
                     "worst_violation": w, "slack_drift": dr, "divergence_max": float(rel.max()),
                     "divergence_rms": float(rel.pow(2).mean().sqrt()),
                     "agree_1e-3_through_step_min": int(horizon.min()),
                     "agree_1e-3_through_step_median": float(np.median(horizon))})
    T = torch.from_numpy(g["T"]).to(dev)
    sh = torch.from_numpy(g["shift"]).to(dev)
    Y = ref.float()
    Ybig = Y.repeat((200000 + Y.shape[0] - 1) // Y.shape[0], 1)[:200000].contiguous()
    bm = {}
    ysub = Ybig[:20000]
    vref = ysub.double() @ T.T + sh
    nz = vref.abs() > 1e-3 * vref.abs().max()
    for mode in ("fp64", "bf16x3", "tf32x3"):
        V = torch.empty((20000, 7000), dtype=torch.float32, device=dev)
        backmap(g["T"], g["shift"], ysub, mode=mode, out=V)
        rel = ((V.double() - vref).abs()[nz] / vref.abs()[nz])
        Vb = torch.empty((200000, 7000), dtype=torch.float32, device=dev)
        backmap(T, sh, Ybig, mode=mode, out=Vb)  # warm
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        backmap(T, sh, Ybig, mode=mode, out=Vb)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        bm[mode] = {"max_rel": float(rel.max()), "rms_rel": float(rel.pow(2).mean().sqrt()), "ms_200k": ms,
                    "tflops": 2.0 * 7000 * 1500 * 200000 / (ms / 1e3) / 1e12}
        del V, Vb
    Yd, Td = Ybig.double(), T.double()
    Vd = torch.empty((200000, 7000), dtype=torch.float64, device=dev)
    ms = []
    for k in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(Yd, Td.T, out=Vd)  # the reference's backmap_into: cuBLAS DGEMM, then + shift
        Vd.add_(sh.double())
        e1.record()
        torch.cuda.synchronize()
        if k:
            ms.append(e0.elapsed_time(e1))
    bm["cublas_dgemm"] = {"max_rel": 0.0, "rms_rel": 0.0, "ms_200k": statistics.mean(ms),
                          "tflops": 2.0 * 7000 * 1500 * 200000 / (statistics.mean(ms) / 1e3) / 1e12}
    del Yd, Td, Vd
    P.close()
    return {"workload": "genome-shaped n=7000 d=1500 m=14000, 8 chains x 200 samples, thinning 256, pair 0.3",
            "chr": rows, "backmap": bm}


def _learned(a):
    """Learned rounding on conditioned variants of the genome-shaped polytope
    (the batched-variant generator): the network, trained on the project's
    kernels from plain-CHR sample covariances of the training variants in
    the base model's rounded coordinates (training time reported
    separately), predicts each held-out variant's rounding; every method
    (plain, the reference's Dikin, whole-ellipsoid Dikin per variant, the
    base rounding alone, learned) then samples all held-out variants in
    batched launches, 8 chains each, thinning 116, pair-prob 0.3, until
    split-R-hat < 1.01 or the budget; min-ESS (chain-summed, y-space) per
    variant over its share of the batch time plus its rounding time."""
    from naja_b200 import learned

    full = learned.run_experiment(n=a.n, d=a.d, n_train=a.learned_train, n_test=a.learned_test,
                                  nchains=8, nspc_train=a.learned_nspc, thinning=a.thinning,
                                  pair_prob=a.pair_prob, epochs=a.learned_epochs, resync=a.resync, seed=a.seed,
                                  gate_budget_s=a.learned_budget_s)
    return _strip_lists(full), full


def _strip_lists(obj):
    """The same record without lists longer than 8 values (kept in --detail-file)."""
    if isinstance(obj, dict):
        return {k: _strip_lists(v) for k, v in obj.items() if not (isinstance(v, list) and len(v) > 8)}
    return obj


def _fp64_figure(a, W, P, x0, torch, dev, M_dev, c_dev, T_dev, sh_dev):
    """The same job in the FP64 tier (the reference's arithmetic): FP64 A,
    slack, ratios and alpha, samples written as float.  Two timed jobs after
    one warm-up; min-ESS/s of the last job, sampling + backmap time."""
    from naja_b200 import backmap
    from naja_b200 import validate as nv

    z = torch.empty((W.nspc * W.nchains, W.d), dtype=torch.float32, device=dev)
    samples = torch.empty_like(z)
    V = torch.empty((W.nspc * W.nchains, W.n), dtype=torch.float32, device=dev)
    times = []
    for k in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        P.run(x0, W.nspc, W.thin, W.nchains, out=z, seed=a.seed, pair_prob=W.pair, resync_interval=0,
              precision="fp64", sparse=a.sparse)
        backmap(M_dev, c_dev, z, mode="fp64", out=samples)
        backmap(T_dev, sh_dev, z, mode=a.backmap_mode, out=V)
        e1.record()
        torch.cuda.synchronize()
        if k:
            times.append(e0.elapsed_time(e1))
    P.check()
    ess, rhat = nv.ess_rhat(samples, W.nchains, layout=1)
    ms = statistics.mean(times)
    min_ess = float(ess.sum(axis=1).min())
    choice = P.kernel_choice(W.nspc, W.thin, W.nchains, pair_prob=W.pair, precision="fp64", sparse=a.sparse)
    return {"value": min_ess / (ms / 1e3), "unit": UNIT, "ms_per_job": ms, "min_ess": min_ess,
            "rhat_max": float(rhat.max()), "chr_steps_per_s": W.steps / (ms / 1e3),
            "kernel": choice["kernel"], "threads": choice["threads"],
            "note": "FP64 tier (no FP32 slack, no recompute needed), same workload and streams"}


def _unit_cube(a, torch, dev):
    """The unit-cube workload [0,1]^50 (A = [I; -I], b = [1; 0], start at the
    centre), 4 chains x 2000 samples, thinning 8, pair-prob 0, Philox seed 0,
    FP32 tier: chain-steps/s, the largest deviation of a coordinate's mean
    from 1/2 and variance from 1/12 in units of its standard error at the
    measured ESS, split-R-hat and min-ESS/s."""
    from naja_b200 import Polytope, synth
    from naja_b200 import validate as nv

    A, b, x0 = synth.unit_cube_stacked(50)
    P = Polytope(A, b, device=dev.index)
    nspc, thin, nch = 2000, 8, 4
    out = torch.empty((nspc * nch, 50), dtype=torch.float32, device=dev)
    times = []
    for k in range(4):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        P.run(x0, nspc, thin, nch, out=out, seed=0, pair_prob=0.0, precision="fp32")
        e1.record()
        torch.cuda.synchronize()
        if k:
            times.append(e0.elapsed_time(e1))
    P.check()
    ess, rhat = nv.ess_rhat(out, nch, layout=1)
    per_dim = ess.sum(axis=1)
    y = out.double().cpu().numpy()
    z_mean = np.abs(y.mean(axis=0) - 0.5) / np.sqrt((1 / 12) / per_dim)
    z_var = np.abs(y.var(axis=0, ddof=1) - 1 / 12) / np.sqrt((1 / 80 - 1 / 144) / per_dim)
    ms = statistics.mean(times)
    choice = P.kernel_choice(nspc, thin, nch)
    P.close()
    return {"workload": "unit cube [0,1]^50, 4 chains x 2000 samples, thinning 8, pair-prob 0, seed 0",
            "ms": ms, "chr_steps_per_s": nch * nspc * thin / (ms / 1e3), "kernel": choice["kernel"],
            "mean_max_dev_in_se": float(z_mean.max()), "var_max_dev_in_se": float(z_var.max()),
            "rhat_max": float(rhat.max()), "min_ess": float(per_dim.min()),
            "min_ess_per_s": float(per_dim.min()) / (ms / 1e3)}


def _reference_arm(a, rank, world):
    """The reference's own implementation of the path, timed on this box.

    The reference implements CHR only in CUDA (src/gpu/chr.cu of
    quothbonney/naja); it has no CPU sampler.  Its sources, compiled
    unmodified for sm_100a into oracle/_ref/, are run through their own API
    (CoordinateHitAndRun, then backmap_into as CoordinateHitAndRunBackmap
    does) with the reference's defaults: FP64, cuRAND MRG32k3a, 128 threads
    per chain.  Time = the call plus cudaDeviceSynchronize, as
    src/engine/job_sampling.cu measures sampling.  Every timed step is the
    whole job (the same chains, samples per chain, polytope, thinning,
    pair-prob and backmap as this project's arm); its min-ESS comes from the
    ESS estimator (FFT autocovariance, FP64) on the reference's own samples.
    Without the reference build the CPU restatement of the same algorithm
    (oracle/) is timed instead, on a bounded sample of the workload.
    """
    import oracle.oracle as O

    W = Workload(a)
    if O.reference_available() and not a.ref_cpu:
        cal_nspc = 20
        # The full workload in every timed step; warm-up steps are short runs
        # (they only warm the context, module loading and cuBLAS).
        nspc = W.nspc
        times = []
        S = None
        for k in range(a.warmup + a.steps):
            timed = k >= a.warmup
            last = k == a.warmup + a.steps - 1
            S_k, _, ms = O.reference_chr_run(W.A, W.b, W.start, nspc if timed else cal_nspc, W.thin, W.nchains,
                                             tpb=128, seed=a.seed, pair_prob=W.pair, T=W.T, shift=W.shift,
                                             want_samples=last, want_v=False)
            if timed:
                times.append(ms / 1e3)
            if last:
                S = S_k
        kind, cores = "reference", 0
        sample = (f"reference CoordinateHitAndRun + backmap_into (FP64, cuRAND MRG32k3a, 128 threads/chain) "
                  f"compiled from its sources for sm_100a: the full workload ({W.nchains} chains x {nspc} samples, "
                  f"thinning {W.thin}, backmap to n={W.n}) in every timed step; warm-up steps {cal_nspc} samples; "
                  f"min-ESS from its own samples of the last step")
        dtype = "f64"
    else:
        cores = os.cpu_count() or 1
        nspc = 2
        t0 = time.perf_counter()
        O.chr_run(W.A, W.b, W.start, nspc, W.thin, W.nchains, seed=a.seed, pair_prob=W.pair, precision="fp64",
                  threads=min(cores, W.nchains))
        dt = time.perf_counter() - t0
        nspc = max(50, min(W.nspc, int(nspc * a.cpu_seconds / max(dt, 1e-3))))
        times = []
        for k in range(a.warmup + a.steps):
            t0 = time.perf_counter()
            S = O.chr_run(W.A, W.b, W.start, nspc, W.thin, W.nchains, seed=a.seed, pair_prob=W.pair,
                          precision="fp64", threads=min(cores, W.nchains))
            if k >= a.warmup:
                times.append(time.perf_counter() - t0)
        kind, cores = "port", min(cores, W.nchains)
        sample = (f"CPU restatement of the reference kernel (FP64), {cores} threads: {W.nchains} chains x {nspc} "
                  f"samples (thinning {W.thin}), no backmap")
        dtype = "f64"
    dt = statistics.mean(times)
    steps_s = W.nchains * nspc * W.thin / dt
    ess = O.ess_fft(S.astype(np.float32), W.nchains, layout=1).sum(axis=1)
    rhat = O.split_rhat(S.astype(np.float32), W.nchains, layout=1)
    min_ess = float(ess.min())
    value = min_ess / dt
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": dtype, "data": "synthetic (seeded genome-shaped generator)",
            "config": W.config(a), "chr_steps_per_s": steps_s, "min_ess": min_ess, "rhat_max": float(rhat.max()),
            "samples_per_chain_timed": nspc,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=2600)
    ap.add_argument("--d", type=int, default=700)
    ap.add_argument("--nchains", type=int, default=16)
    ap.add_argument("--nspc", type=int, default=12500)
    ap.add_argument("--thinning", type=int, default=116)
    ap.add_argument("--pair-prob", type=float, default=0.3)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--resync", type=int, default=2048)
    ap.add_argument("--tpb", type=int, default=-1, help="consumer threads per chain (-1 = automatic)")
    ap.add_argument("--sparse", default="auto", choices=["auto", "dense", "columns"],
                    help="step kernel: compressed columns, dense, or the library's automatic choice")
    ap.add_argument("--backmap-mode", default="tf32x3", choices=["fp64", "bf16x3", "tf32x3"])
    ap.add_argument("--rounding", default="dikin_full", choices=["none", "dikin", "dikin_full"],
                    help="rounding of the headline job: whole-ellipsoid Dikin (default), the reference's "
                         "Dikin preconditioner, or none (plain CHR)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--batch-models", type=int, default=64, help="batched-variant section (0 = skip)")
    ap.add_argument("--batch-chains", type=int, default=8)
    ap.add_argument("--batch-nspc", type=int, default=4000)
    ap.add_argument("--batch-shape", default="", help="threads,slots,slack_smem,ctas_per_sm[,sparse] (skips the autotuner)")
    ap.add_argument("--ref-cpu", action="store_true", help="reference arm: time the CPU restatement")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--learned-train", type=int, default=1024,
                    help="learned-rounding section: training variants (0 = skip)")
    ap.add_argument("--learned-test", type=int, default=16)
    ap.add_argument("--learned-nspc", type=int, default=1500, help="samples per chain of each training variant")
    ap.add_argument("--learned-budget-s", type=float, default=60.0,
                    help="learned-rounding section: seconds per method of the held-out run to the gate")
    ap.add_argument("--learned-epochs", type=int, default=60)
    ap.add_argument("--no-fp64-figure", dest="fp64_figure", action="store_false",
                    help="skip the FP64-tier figure of the same job")
    ap.add_argument("--no-cube", dest="cube", action="store_false", help="skip the unit-cube workload")
    ap.add_argument("--gate-budget-s", type=float, default=60.0,
                    help="run-to-gate section: seconds per rounding method (0 = skip)")
    ap.add_argument("--detail-file", default="",
                    help="write per-step times and per-variant records here (JSON)")
    ap.add_argument("--no-precision-study", dest="precision_figures", action="store_false",
                    help="skip the FP32/FP64 tier and backmap precision section")
    ap.add_argument("--precision-study", action="store_true",
                    help="run only the FP32/FP64 tier and backmap precision study and print it")
    a = ap.parse_args(argv)
    if a.warmup < 3:
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if a.precision_study:
        print(json.dumps(_precision_study(a)))
        return
    if a.impl == "reference":
        # rank 0 alone times the reference; the other ranks exit without work
        if rank == 0:
            print(json.dumps(_reference_arm(a, rank, world)))
        return
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        line = _ours(a, rank, world)
        if rank == 0 and line is not None:
            print(json.dumps(line))
    finally:
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
