"""Benchmark of the FDTD time-stepping path on B200.

Workload (one GPU): the non-uniform mesh of 200x160x120 cells with seeded
graded spacing (1-8 mm, neighbour ratio <= 1.3), 8-cell UPML on every face,
one Debye block, a TFSF plane wave, 16 time-domain points and a 64x64 plane
of frequency-domain observers over 200 frequencies; N_out = 216x176x136 =
5,170,176 outer-box cells.  A step is one leapfrog time step of the whole
grid (src/simulation.c:156-222).  The metric is Mcell-updates/s =
N_out * steps / time (the reference's spi/cell denominator, src/timer.c:95).

--gpus N runs N independent replicas, one per GPU (the path does not shard;
per-GPU work is fixed, scaling "weak").  --impl reference times the
reference's own CPU build on the host cores instead.
"""
from __future__ import annotations

import os

# Before any CUDA context exists: 32 hardware work queues, so the batch and
# serve workloads' many streams do not share queues (the package sets the
# same default when it is imported first).
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

import argparse
import json
import shutil
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

B_ALG = {"fp32": 4, "fp64": 8}        # bytes per word
WORDS_E, WORDS_H = 15, 12             # algorithmic words per cell of the E and H sweeps
NOMINAL_HBM_GBS = 8000.0              # the B200's nominal HBM3e bandwidth, for the "% of 8 TB/s" figure
# The UPML sweeps also read and write their auxiliaries: PP and P per E
# component (4 words), B per H component (2 words).  These are overhead on
# the algorithmic basis (not credited in `roofline.achieved`); they appear
# only under the separate `*_with_upml_aux` keys.
WORDS_PML_E, WORDS_PML_H = WORDS_E + 12, WORDS_H + 6
WORKLOAD = dict(nt=4000, dims=(200, 160, 120), plane=64, nfreq=200, npml=8, ntd=16)
# Outer-box cells: the mesh plus its UPML layers on both sides of each axis
# (src/grid.c:357-387), the reference's spi/cell denominator (src/timer.c:95).
N_OUT = ((WORKLOAD["dims"][0] + 2 * WORKLOAD["npml"]) * (WORKLOAD["dims"][1] + 2 * WORKLOAD["npml"]) *
         (WORKLOAD["dims"][2] + 2 * WORKLOAD["npml"]))
# Both arms print this config.
CONFIG = {"workload": "graded 200x160x120, UPML8, Debye, TFSF, 64x64x200 DFT plane + 16 TD",
          "n_out_cells": N_OUT, "precision": "fp32", "l2": "inputs larger than L2 (~370 MB/GPU)"}
FP32_REFERENCE_ERROR = ROOT / "tests" / "golden" / "fp32_reference_error.json.gz"


def rank_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def init_dist(world: int, backend: str = "nccl"):
    """The process group for N > 1 replicas (None for one process), with a
    short timeout so ranks that wait for a lost peer end with an error."""
    if world <= 1:
        return None
    import torch.distributed as dist
    from datetime import timedelta

    dist.init_process_group(backend, timeout=timedelta(seconds=120))
    return dist


def max_over_ranks(value: float, dist, device="cuda") -> float:
    """The largest of every rank's value; every rank must call it."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist, device="cuda") -> float:
    """The sum of every rank's value; every rank must call it."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def replica_throughput(n_out: int, steps: int, ms_max: float, world: int) -> float:
    """Whole-job Mcell-updates/s of `world` replicas of n_out cells that each
    ran `steps` steps, timed by the slowest rank's ms."""
    return world * n_out * steps / (ms_max * 1e-3) / 1e6


def make_mesh(directory: Path, nt: int, plane: int = None) -> Path:
    from vulture_b200 import meshgen

    kw = dict(WORKLOAD)
    kw["nt"] = nt
    if plane is not None:
        kw["plane"] = plane
    return Path(meshgen.write(meshgen.graded_upml(seed=2, **kw), directory / "graded_upml.mesh"))


# Untimed steps before a timed region, inside the clock record: 128 (two
# 64-step blocks, about 20 ms of config 2) bring the GPU out of the idle
# clocks it drops to while the clock sampler starts, then the W warm-up steps,
# which also capture the short step graphs the timed steps replay.
PREHEAT_STEPS = 128


def warm_then_time(g, args, dist, local):
    """PREHEAT_STEPS + W untimed steps, then exactly K timed steps (the
    engine's run_ms: CUDA events on its stream), with a barrier and a device
    synchronisation on both sides; returns the clock record."""
    import torch

    with ClockSampler(local) as clk:
        g.run(PREHEAT_STEPS + args.warmup)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        g.run(args.steps)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    return clk


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.out = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.out = tempfile.NamedTemporaryFile("w+", delete=False, suffix=".csv")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        if not self.out:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        with open(self.out.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_record(kernel: str, precision: str):
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    return d.get(f"{kernel}:{precision}")


def scaled_traffic(kernel: str, precision: str, cells: float):
    """DRAM bytes per launch of a kernel whose ncu capture ran on a smaller
    case of the same workload ({"bytes": B, "cells": C} in traffic.json):
    B scaled by the cells this launch updates, since the traffic grows in
    proportion.  A plain number is already per launch at full size."""
    rec = traffic_record(kernel, precision)
    if isinstance(rec, dict):
        return rec["bytes"] * cells / rec["cells"]
    return rec


def time_reference(binary: str, mesh_dir: Path, nt_lo: int, nt_hi: int, threads: int, plane=None):
    """Per-step throughput of a reference build: two runs of the same mesh
    with nt_lo and nt_hi steps; the difference removes set-up and output.
    Loads nothing of this repository's native code."""
    walls = []
    for nt in (nt_lo, nt_hi):
        d = Path(tempfile.mkdtemp(prefix="vb_cpu_", dir=mesh_dir))
        make_mesh(d, nt, plane)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        t0 = time.perf_counter()
        r = subprocess.run([binary, "-n", str(threads), "graded_upml.mesh"], cwd=d, env=env, capture_output=True,
                           text=True)
        walls.append(time.perf_counter() - t0)
        if r.returncode != 0:
            raise RuntimeError(f"reference run failed: {r.stderr[-400:]}")
        shutil.rmtree(d, ignore_errors=True)
    dt = walls[1] - walls[0]
    return N_OUT * (nt_hi - nt_lo) / dt / 1e6, walls


def run_reference_arm(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return
    binary = ROOT / "oracle" / "_ref" / "vulture_ref_f32_omp"
    base = {"metric": "Mcell-updates/s", "unit": "Mcell-updates/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32", "data": "synthetic", "config": dict(CONFIG)}
    if not binary.exists():
        base["unavailable"] = "reference CPU build (oracle/_ref) not present"
        print(json.dumps(base))
        return
    threads = os.cpu_count() or 1
    # A bounded sample: the reference spends ~0.2 s per step in its serial
    # point-DFT loop on this workload, so K timed steps are capped.
    k = max(2, min(args.steps, 60))
    w = max(1, min(args.warmup, 5))
    work = Path(tempfile.mkdtemp(prefix="vb_refarm_"))
    value, walls = time_reference(str(binary), work, w, w + k, threads)
    shutil.rmtree(work, ignore_errors=True)
    base.update({"value": value, "ms_per_step": N_OUT / (value * 1e6) * 1e3,
                 "cpu_baseline": {"value": value, "unit": "Mcell-updates/s", "cores": threads, "kind": "reference",
                                  "sample": f"graded 200x160x120 UPML mesh, vulture_ref_f32_omp -n {threads}, runs of {w} and "
                                            f"{w + k} steps, difference of wall times {walls}"},
                 "e2e": {"value": value, "unit": "Mcell-updates/s", "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": 0}})
    print(json.dumps(base))


def _db_errors(re, im, re64, im64):
    """Per result (FD point x component): the largest |dB| difference of the
    FP32 DFT magnitude against FP64 over the frequencies whose FP64 magnitude
    is within 60 dB of that result's peak; NaN for a result that is zero."""
    import numpy as np

    mag, mag64 = np.hypot(re, im), np.hypot(re64, im64)
    out = np.full(mag64.shape[:2], np.nan)
    for q in range(mag64.shape[0]):
        for c in range(mag64.shape[1]):
            ref = mag64[q, c]
            peak = ref.max()
            if peak <= 0:
                continue
            sel = ref > peak * 1e-3
            out[q, c] = np.abs(20 * np.log10(np.maximum(mag[q, c][sel], 1e-300)) - 20 * np.log10(ref[sel])).max()
    return out


def error_report(td, re, im, td64, re64, im64, steps, fd_names=None):
    """FP32 against FP64 on the same steps: time-domain relative L2 per point
    observer, and the frequency-domain magnitude error in dB per result
    (observer point and component) over the frequencies whose FP64 magnitude
    is within 60 dB of that result's peak.  With the reference's own FP32
    error on the same mesh and steps (tests/golden/fp32_reference_error.json.gz,
    made by the reference's FP32 and FP64 builds), each result is also
    compared with it."""
    import numpy as np

    a, b = td[:steps], td64[:steps]
    td_err, td_norm = [], []
    for q in range(b.shape[1]):
        den = np.sqrt((b[:, q, :] ** 2).sum())
        td_norm.append(float(den))
        td_err.append(float(np.sqrt(((a[:, q, :] - b[:, q, :]) ** 2).sum()) / den) if den > 0 else 0.0)
    dbm = _db_errors(re, im, re64, im64)
    db = dbm[~np.isnan(dbm)]
    if db.size == 0:
        db = np.zeros(1)
    # Points the pulse has not reached within the run hold only round-off
    # in FP64; those below 1e-3 of the largest point's norm are listed but
    # left out of the maximum.
    top = max(td_norm) if td_norm else 0.0
    live = [e for e, n in zip(td_err, td_norm) if n >= 1e-3 * top and n > 0]
    edges = [0.0, 1e-6, 1e-5, 1e-4, 1e-3, 1e-2, 1e-1, float("inf")]
    hist = {f"<={hi:g}" if hi != float("inf") else f">{lo:g}": int(((db > lo) & (db <= hi)).sum()) if lo > 0
            else int((db <= hi).sum()) for lo, hi in zip(edges[:-1], edges[1:])}
    rep = {"steps": steps, "td_rel_l2_max": max(live) if live else 0.0, "td_bound": 1e-4,
           "td_points": len(live), "td_points_below_1e-3_of_peak": len(td_err) - len(live),
           "td_rel_l2": td_err, "td_norm": td_norm, "fd_db_max": float(db.max()), "fd_db_median": float(np.median(db)),
           "fd_db_p99": float(np.percentile(db, 99)), "fd_results": int(db.size),
           "fd_share_within_1e-3_db": float((db <= 1e-3).mean()), "fd_bound_db": 1e-3, "fd_db_histogram": hist}
    if fd_names is not None and FP32_REFERENCE_ERROR.exists():
        import gzip

        with gzip.open(FP32_REFERENCE_ERROR, "rt") as fh:
            ref = json.load(fh)
        if ref["mesh"]["nt"] == steps:
            mine, theirs = [], []
            for q, name in enumerate(fd_names):
                r = ref["fd_db"].get(name)
                if r is None:
                    continue
                for c in range(6):
                    if not np.isnan(dbm[q, c]) and r[c] is not None:
                        mine.append(dbm[q, c])
                        theirs.append(r[c])
            mine, theirs = np.array(mine), np.array(theirs)
            ref_td = [v["rel_l2"] for v in ref["td"].values() if v["norm"] >= 1e-3 * max(
                w["norm"] for w in ref["td"].values())]
            rep["vs_reference_fp32"] = {
                "what": "the reference's own FP32 build against its FP64 build, same mesh and steps, same measures",
                "results_compared": int(mine.size),
                "share_engine_le_reference": float((mine <= theirs).mean()) if mine.size else None,
                "share_engine_le_max_reference_1e-3_db": float((mine <= np.maximum(theirs, 1e-3)).mean())
                if mine.size else None,
                "reference_fd_db_median": float(np.median(theirs)) if theirs.size else None,
                "reference_fd_db_p99": float(np.percentile(theirs, 99)) if theirs.size else None,
                "reference_fd_db_max": float(theirs.max()) if theirs.size else None,
                "reference_td_rel_l2_max": max(ref_td) if ref_td else None}
    return rep


def kernel_split(g, steps_per_block: int = 64):
    """Device time per step of each kernel of a step, each timed alone with
    CUDA events on the engine's stream (warm, 20 launches): the sweeps, every
    other part the problem has, and the 64-step DFT fold divided over its
    steps.  Call on an engine whose results are no longer needed."""
    from vulture_b200 import _native as N

    out = {}
    names = {N.VGPU_K_BULK_E: "k_sweep_tma<E,bulk>", N.VGPU_K_BULK_H: "k_sweep_tma<H,bulk>",
             N.VGPU_K_PML_E: "k_sweep_tma<E,UPML>", N.VGPU_K_PML_H: "k_sweep_tma<H,UPML>"}
    for kid, name in list(names.items()) + [(v, k) for k, v in N.STEP_KERNELS.items()]:
        try:
            ms, _ = g.time_kernel(kid, warmup=3, iters=20)
        except N.NativeError:
            continue           # not part of this problem's step
        out[name] = ms / steps_per_block if kid == N.STEP_KERNELS["dft_fold_64"] else ms
    tot = sum(out.values())
    scalar = None
    if "dft_fold_64" in out:
        scalar, _ = g.time_kernel(N.VGPU_K_DFT_BLOCK_SCALAR, warmup=3, iters=20)
    return {"ms_per_step": out, "sum_ms": tot,
            "dft_fold_64_ms": {"tensor_core_m16n8k4": out["dft_fold_64"] * steps_per_block, "scalar": scalar}
            if scalar is not None else None,
            "share": {k: v / tot for k, v in out.items()} if tot > 0 else {},
            "what": "each kernel of a step timed alone (CUDA events, warm, 20 launches); the DFT fold of a "
                    "64-step block divided by 64; the sum omits the launch gaps of a real step"}


def full_run_legs(args, m, prec, e2e_run, dist, world, n_out, nt_full):
    """The workload's whole run (its own 4000 steps) end to end through the C
    ABI, and the same run in plain FP64: the FP64 path's throughput and the
    FP32 error per result against it."""
    full = e2e_run(prec, nt_full)
    full_wall = max_over_ranks(full["wall_s"], dist)
    e2e_full = {"steps": nt_full, "value": world * n_out * nt_full / full_wall / 1e6, "unit": "Mcell-updates/s",
                "wall_s": full_wall, "create_s": full["create_s"], "step_s": full["step_s"],
                "read_s": full["read_s"], "h2d_bytes": full["h2d"], "d2h_bytes": full["d2h"],
                "device_mcell_per_s": n_out * nt_full / (full["run_ms"] * 1e-3) / 1e6,
                "what": "the workload's whole run through the C ABI: create + all steps + observer read-back"}
    fp64 = None
    fp32_error = None
    if prec == "fp32" and not args.no_fp64:
        f64 = e2e_run("fp64", nt_full)
        fp64 = n_out * nt_full / (f64["run_ms"] * 1e-3) / 1e6
        names = [m.observer_name(True, q) for q in range(m.num_fd)]
        fp32_error = error_report(full["td"], full["re"], full["im"], f64["td"], f64["re"], f64["im"], nt_full,
                                  names)

    return e2e_full, fp64, fp32_error


def run_gpu_arm(args):
    import numpy as np
    import torch

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dist = init_dist(world)
    import vulture_b200 as vb
    from vulture_b200 import _native as N

    prec = args.precision
    work = Path(tempfile.mkdtemp(prefix=f"vb_bench_{rank}_"))
    nt = max(WORKLOAD["nt"], PREHEAT_STEPS + args.warmup + args.steps)
    mesh_path = make_mesh(work, nt)
    old = os.getcwd()
    os.chdir(work)
    m = vb.Mesh(mesh_path.name)
    os.chdir(old)
    n_out = m.num_cells
    assert n_out == N_OUT, (n_out, N_OUT)

    # Device-resident timing: untimed steps, then exactly K timed steps.
    g = vb.GpuRun(m, prec)
    clk = warm_then_time(g, args, dist, local)
    st = g.stats()
    ms = st.run_ms
    launches = int(st.kernel_launches)
    g.check_finite()
    ms = max_over_ranks(ms, dist)
    value = replica_throughput(n_out, args.steps, ms, world)

    # Roofline of the dominant kernel, each sweep timed live on the engine's
    # stream with CUDA events.  Algorithmic bytes: 15 (E) or 12 (H) words per
    # updated cell, bulk and UPML points alike; the UPML auxiliaries' words
    # are overhead, reported apart under *_with_upml_aux.
    # A mesh with UPML regions runs each half step as one launch of the UPML
    # kernel (bulk, mixed and UPML tiles); the bulk kernel then has no tiles.
    kern = {}
    for name, kid, wb, wp in (("k_sweep_tma<E,bulk>", N.VGPU_K_BULK_E, WORDS_E, WORDS_PML_E),
                              ("k_sweep_tma<H,bulk>", N.VGPU_K_BULK_H, WORDS_H, WORDS_PML_H),
                              ("k_sweep_tma<E,UPML>", N.VGPU_K_PML_E, WORDS_E, WORDS_PML_E),
                              ("k_sweep_tma<H,UPML>", N.VGPU_K_PML_H, WORDS_H, WORDS_PML_H)):
        bp, pp = g.sweep_points(kid)
        if not bp and not pp:
            continue
        kms, pts = g.time_kernel(kid, warmup=3, iters=20)
        nbytes = wb * (bp + pp) / 3.0 * B_ALG[prec]
        aux_bytes = (wb * bp + wp * pp) / 3.0 * B_ALG[prec]
        kern[name] = dict(ms=kms, cells=pts / 3.0, bulk_points=bp, pml_points=pp, bytes=nbytes,
                          gbs=nbytes / (kms * 1e-3) / 1e9, bytes_with_upml_aux=aux_bytes,
                          gbs_with_upml_aux=aux_bytes / (kms * 1e-3) / 1e9)
    split = kernel_split(g)
    g.close()
    peak, peak_kind = peaks()
    dom = max(kern, key=lambda k: kern[k]["ms"])
    achieved = kern[dom]["bytes"] / (kern[dom]["ms"] * 1e-3) / 1e9
    tr = traffic_record(dom, prec)

    # End to end through the C ABI with host buffers: create (host->device
    # upload of the problem), K steps, read the observers back
    # (device->host), each phase on the wall clock.
    def e2e_run(precision, steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        gg = vb.GpuRun(m, precision)
        t1 = time.perf_counter()
        gg.run(steps)
        t2 = time.perf_counter()
        td_ = gg.td(steps)
        re_, im_ = gg.dft()
        t3 = time.perf_counter()
        s_ = gg.stats()
        gg.close()
        return dict(td=td_, re=re_, im=im_, create_s=t1 - t0, step_s=t2 - t1, read_s=t3 - t2, wall_s=t3 - t0,
                    h2d=int(s_.h2d_bytes), d2h=td_.nbytes + re_.nbytes + im_.nbytes, run_ms=s_.run_ms)

    # One untimed pass first (allocator caches, page-locked result blocks),
    # as the W warm-up steps precede the timed ones.
    e2e_run(prec, args.steps)
    k = e2e_run(prec, args.steps)
    e2e_wall = max_over_ranks(k["wall_s"], dist)
    e2e = {"value": world * n_out * args.steps / e2e_wall / 1e6, "unit": "Mcell-updates/s",
           "h2d_bytes_per_step": k["h2d"] / args.steps, "d2h_bytes_per_step": k["d2h"] / args.steps,
           "wall_s": e2e_wall, "create_s": k["create_s"], "step_s": k["step_s"], "read_s": k["read_s"],
           "what": f"vgpu_create (problem upload, {k['h2d']} bytes host->device) + K steps + observer read-back; "
                   f"at K = {args.steps} creation is {100 * k['create_s'] / k['wall_s']:.0f}% of the wall time; "
                   "one untimed pass before it"}
    # Its results go: their page-locked blocks return to the cache for the
    # next read.
    k = None

    # The workload's whole run (its own 4000 steps) end to end, and the same
    # run in plain FP64: the FP32 error per result against it, and the FP64
    # path's throughput.
    nt_full = m.num_steps
    e2e_full = fp64 = fp32_error = None
    if not args.no_full_run:
        e2e_full, fp64, fp32_error = full_run_legs(args, m, prec, e2e_run, dist, world, n_out, nt_full)

    sub = {}
    sub = {}
    if not args.no_enclosure:
        sub["enclosure"] = enclosure_workload(args, dist)
    if not args.no_batch:
        sub["batch"] = batch_workload(args, dist)
    if not args.no_serve:
        sub["serve"] = serve_workload(args, dist)

    cpu = None
    if rank == 0 and not args.no_cpu:
        binary = ROOT / "oracle" / "_ref" / "vulture_ref_f32_omp"
        if binary.exists():
            threads = os.cpu_count() or 1
            cw = Path(tempfile.mkdtemp(prefix="vb_cpub_"))
            try:
                v, walls = time_reference(str(binary), cw, 5, 45, threads)
                v2, walls2 = time_reference(str(binary), cw, 5, 45, threads, plane=0)
                cpu = {"value": v, "unit": "Mcell-updates/s", "cores": threads, "kind": "reference",
                       "sample": f"graded 200x160x120 UPML mesh on vulture_ref_f32_omp -n {threads}: runs of 5 and 45 steps, "
                                 f"difference of wall times {[round(x, 2) for x in walls]} s",
                       "without_fd_plane": v2}
            except Exception as exc:  # the baseline is reported, never required
                cpu = {"value": None, "error": str(exc)[:300]}
            shutil.rmtree(cw, ignore_errors=True)

    os.chdir(old)
    shutil.rmtree(work, ignore_errors=True)
    if rank == 0:
        out = {
            "metric": "Mcell-updates/s", "value": value, "unit": "Mcell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "untimed_steps_before": PREHEAT_STEPS + args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": prec,
            "data": "synthetic", "config": dict(CONFIG, precision=prec),
            "step_roofline": {"bytes_per_cell": (WORDS_E + WORDS_H) * B_ALG[prec],
                              "achieved_gbs": value / world * 1e6 * (WORDS_E + WORDS_H) * B_ALG[prec] / 1e9,
                              "frac": value / world * 1e6 * (WORDS_E + WORDS_H) * B_ALG[prec] / 1e9 / peak,
                              "pct_of_8tbs": 100 * value / world * 1e6 * (WORDS_E + WORDS_H) * B_ALG[prec]
                              / 1e9 / NOMINAL_HBM_GBS,
                              "what": "whole step: cell-updates/s x 27 algorithmic words per cell, of measured; "
                                      "pct_of_8tbs of the nominal 8 TB/s"},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": tr, "kernels": kern,
                         "achieved_with_upml_aux": kern[dom]["gbs_with_upml_aux"],
                         "frac_with_upml_aux": kern[dom]["gbs_with_upml_aux"] / peak,
                         "words_per_cell": {"E": WORDS_E, "H": WORDS_H},
                         "what": "algorithmic bytes (15 E / 12 H words per updated cell, UPML auxiliaries not "
                                 "credited) of the longest sweep launch over its CUDA-event time, of measured"},
            "kernel_split": split,
            "e2e": e2e,
            "e2e_full_run": e2e_full,
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "fp64_value": fp64,
            "fp32_error": fp32_error,
            **sub,
            "cpu_baseline": cpu,
        }
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def _meshes_dir(texts, prefix):
    from vulture_b200 import meshgen

    d = Path(tempfile.mkdtemp(prefix=prefix))
    return d, [meshgen.write(t, d / f"m{q:03d}.mesh") for q, t in enumerate(texts)]


def _sweep_bytes(g, prec):
    """Algorithmic bytes of one step of an engine: the four sweeps' points by
    the bulk or UPML word count."""
    from vulture_b200 import _native as N

    tot = 0.0
    for kid, wb, wp in ((N.VGPU_K_BULK_E, WORDS_E, WORDS_PML_E), (N.VGPU_K_BULK_H, WORDS_H, WORDS_PML_H),
                        (N.VGPU_K_PML_E, WORDS_E, WORDS_PML_E), (N.VGPU_K_PML_H, WORDS_H, WORDS_PML_H)):
        bp, pp = g.sweep_points(kid)
        tot += (wb * bp + wp * pp) / 3.0 * B_ALG[prec]
    return tot


def enclosure_workload(args, dist=None, cpu=False):
    """The shielded enclosure at its stated size: 400x300x250 graded cells,
    first-order Mur outer boundary, a thin-walled SIBC box with a seeded
    aperture, 4 PEC thin wires, TFSF illumination, 8 FD points and a 128x128
    FD plane over 500 frequencies, 20000 steps; FP32 fields, FP64 DFT.
    Device-resident K steps after W, the longest sweep's roofline, the
    per-kernel split of a step, and the whole 20000-step run end to end
    through the C ABI (create, step, read back)."""
    import torch

    import vulture_b200 as vb
    from vulture_b200 import _native as N
    from vulture_b200 import meshgen

    rank, world, local = rank_info()
    work = Path(tempfile.mkdtemp(prefix=f"vb_encl_{rank}_"))
    dims = tuple(getattr(args, "enclosure_dims", None) or (400, 300, 250))
    text = meshgen.shielded_enclosure(seed=3, nt=20000, dims=dims, plane=128, nfreq=500)
    path = Path(meshgen.write(text, work / "enclosure.mesh"))
    m = vb.Mesh(path)
    n_out = m.num_cells
    prec = "fp32"
    g = vb.GpuRun(m, prec)
    clk = warm_then_time(g, args, dist, local)
    st = g.stats()
    ms = max_over_ranks(st.run_ms, dist)
    value = replica_throughput(n_out, args.steps, ms, world)
    kern = {}
    for name, kid, wb in (("k_sweep_tma<E,bulk>", N.VGPU_K_BULK_E, WORDS_E), ("k_sweep_tma<H,bulk>", N.VGPU_K_BULK_H, WORDS_H),
                          ("k_sweep_tma<E,UPML>", N.VGPU_K_PML_E, WORDS_E), ("k_sweep_tma<H,UPML>", N.VGPU_K_PML_H, WORDS_H)):
        bp, pp = g.sweep_points(kid)
        if not bp and not pp:
            continue
        kms, pts = g.time_kernel(kid, warmup=3, iters=20)
        nbytes = wb * (bp + pp) / 3.0 * B_ALG[prec]
        kern[name] = dict(ms=kms, cells=pts / 3.0, bytes=nbytes, gbs=nbytes / (kms * 1e-3) / 1e9)
    split = kernel_split(g)
    g.close()
    peak, peak_kind = peaks()
    dom = max(kern, key=lambda k: kern[k]["ms"])
    # The whole run through the C ABI.
    full = None
    if not args.no_full_run:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g2 = vb.GpuRun(m, prec)
        t1 = time.perf_counter()
        g2.run()
        t2 = time.perf_counter()
        re, im = g2.dft()
        t3 = time.perf_counter()
        s2 = g2.stats()
        g2.close()
        full_wall = max_over_ranks(t3 - t0, dist)
        full = {"steps": m.num_steps, "value": world * n_out * m.num_steps / full_wall / 1e6,
                "unit": "Mcell-updates/s", "wall_s": full_wall, "create_s": t1 - t0, "step_s": t2 - t1,
                "read_s": t3 - t2, "h2d_bytes": int(s2.h2d_bytes), "d2h_bytes": re.nbytes + im.nbytes,
                "device_mcell_per_s": n_out * m.num_steps / (s2.run_ms * 1e-3) / 1e6}
    out = {
        "metric": "Mcell-updates/s", "value": value, "unit": "Mcell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "dtype": prec,
        "untimed_steps_before": PREHEAT_STEPS + args.warmup,
        "config": {"workload": "shielded enclosure {}x{}x{} graded, Mur, SIBC box with aperture, 4 PEC wires, "
                               "TFSF, 128x128 + 8 FD points x 500 frequencies, 20000 steps".format(*dims),
                   "n_out_cells": n_out, "precision": prec, "dft": "fp64"},
        "step_roofline": {"bytes_per_cell": (WORDS_E + WORDS_H) * B_ALG[prec],
                          "frac": value / world * 1e6 * (WORDS_E + WORDS_H) * B_ALG[prec] / 1e9 / peak,
                          "pct_of_8tbs": 100 * value / world * 1e6 * (WORDS_E + WORDS_H) * B_ALG[prec] / 1e9
                          / NOMINAL_HBM_GBS},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": kern[dom]["gbs"], "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": kern[dom]["gbs"] / peak,
                     "traffic": scaled_traffic(dom, prec, kern[dom]["cells"]), "kernels": kern},
        "kernel_split": split,
        "e2e_full_run": full,
        "clocks": clk.summary()}
    if cpu and rank == 0:
        binary = ROOT / "oracle" / "_ref" / "vulture_ref_f32_omp"
        if binary.exists():
            threads = os.cpu_count() or 1
            walls = []
            for nt in (2, 6):
                d = Path(tempfile.mkdtemp(prefix="vb_cpue_", dir=work))
                meshgen.write(meshgen.shielded_enclosure(seed=3, nt=nt, dims=dims, plane=128, nfreq=500),
                              d / "enclosure.mesh")
                t0 = time.perf_counter()
                r = subprocess.run([str(binary), "-n", str(threads), "enclosure.mesh"], cwd=d, capture_output=True,
                                   env=dict(os.environ, OMP_NUM_THREADS=str(threads)))
                walls.append(time.perf_counter() - t0)
                if r.returncode:
                    walls = None
                    break
            if walls:
                v = n_out * 4 / (walls[1] - walls[0]) / 1e6
                out["cpu_baseline"] = {"value": v, "unit": "Mcell-updates/s", "cores": threads, "kind": "reference",
                                       "sample": f"enclosure mesh on vulture_ref_f32_omp -n {threads}: runs of 2 and 6 "
                                                 f"steps, difference of wall times {[round(x, 2) for x in walls]} s"}
    shutil.rmtree(work, ignore_errors=True)
    return out


def batch_workload(args, dist=None):
    """Many independent meshes of uneven size (seeded PEC/dielectric slabs,
    6-cell UPML, a hard or soft dipole), FP32, solved together (solve_batch:
    engines created one after another, then stepped as one group -- one
    sweep launch per half step over every mesh's tiles, march depth chosen
    by the autotuner -- or, with --batch-mode streams, side by side on one
    stream per engine), against the plain FP64 path solving them one after
    another.  Solves/s counts create + steps + observer read-back.  The FP64
    path's solves/s is measured on a sample of the meshes (every
    len/fp64_sample-th, which are drawn independently like the rest): the
    mean time per solve of the sample, over the whole batch."""
    import torch

    import vulture_b200 as vb
    from vulture_b200 import meshgen
    from vulture_b200.serve import solve_batch

    rank, world, local = rank_info()
    rng = __import__("random").Random(4 + rank)
    texts = [meshgen.batch_mesh(rng, q, nmin=32, nmax=160, ntmin=args.batch_steps[0], ntmax=args.batch_steps[1])
             for q in range(args.batch_count)]
    d, paths = _meshes_dir(texts, "vb_batch_")
    meshes = [vb.Mesh(p) for p in paths]
    cell_updates = sum(m.num_cells * m.num_steps for m in meshes)
    # Warm-up: one small solve of each precision (module load, caches).
    for prec in ("fp32", "fp64"):
        vb.GpuRun(meshes[0], prec).run(min(64, meshes[0].num_steps)).close()
    torch.cuda.synchronize()

    # The grouped path's tile tuning, chosen by timing a sample of the
    # meshes (autotune.tune; cached per device and size mix).  It runs before
    # the timed batch and is reported apart.
    tuning, tune_rec = None, None
    if args.batch_mode in ("grouped", "both"):
        from vulture_b200 import autotune

        tuning, tune_rec = autotune.tune(meshes, "fp32", use_cache=False)
        torch.cuda.synchronize()

    # End to end: engines created one after another, then stepped together
    # (solve_batch), then every solve's observers read back.
    def timed_batch(grouped):
        if dist:
            dist.barrier()
        with ClockSampler(local) as clk:
            t0 = time.perf_counter()
            runs = solve_batch(meshes, "fp32", grouped=grouped, tuning=tuning if grouped else None)
            for r in runs:
                r.td()
                r.dft()
            wall = time.perf_counter() - t0
        create = max(r.batch_started for r in runs)
        step = max(r.batch_finished for r in runs) - create
        rep = runs[0].batch_report
        if rep is not None:
            # The report counts every kernel of the call, per-engine block-end work included.
            n_launch = rep["launches"]
        else:
            n_launch = sum(int(r.stats().kernel_launches) for r in runs)
        nb = sum(_sweep_bytes(r, "fp32") * r.mesh.num_steps for r in runs)
        for r in runs:
            r.close()
        return {"wall": wall, "create": create, "step": step, "launches": n_launch, "bytes": nb, "report": rep,
                "clk": clk}

    modes = {"grouped": [True], "streams": [False], "both": [False, True]}[args.batch_mode]
    legs = {g: timed_batch(g) for g in modes}
    main = legs[modes[0]]
    wall32, create_s, step_s, launches, nbytes, clk = (main["wall"], main["create"], main["step"], main["launches"],
                                                       main["bytes"], main["clk"])
    # The plain FP64 path: one solve after another, each created, run to its
    # end and read back.
    stride = max(1, len(meshes) // max(1, args.batch_fp64_sample))
    sample = meshes[::stride]
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for m in sample:
        g = vb.GpuRun(m, "fp64").run()
        g.td()
        g.dft()
        g.close()
    wall64_sample = time.perf_counter() - t0
    wall64 = wall64_sample / len(sample) * len(meshes)
    # Whole job: every rank's solves over the slowest rank's time.
    wall32, wall64, step_s, create_s = (max_over_ranks(v, dist) for v in (wall32, wall64, step_s, create_s))
    solves = sum_over_ranks(len(meshes), dist)
    nbytes = sum_over_ranks(nbytes, dist)
    cell_updates = int(sum_over_ranks(cell_updates, dist))
    launches = int(sum_over_ranks(launches, dist))
    peak, peak_kind = peaks()
    shutil.rmtree(d, ignore_errors=True)
    sps32, sps64 = solves / wall32, solves / wall64
    step_mcell = cell_updates / step_s / 1e6
    return {
        "metric": "batched solves/s", "value": sps32, "unit": "solves/s", "n_gpus": world,
        "higher_is_better": True, "dtype": "fp32",
        "config": {"workload": f"{len(meshes)} meshes, per-axis 32-160 cells, 6-cell UPML, PEC/dielectric "
                               f"slabs, dipole; {args.batch_steps[0]}-{args.batch_steps[1]} steps each",
                   "cell_updates": cell_updates,
                   "batch": ("solve_batch: engines created one after another, then vgpu_run_grouped (one sweep "
                             "launch per half step over every mesh's tiles, autotuned march depth)"
                             if modes[0] else "solve_batch: engines created one after another, then "
                             "vgpu_run_batch, one stream per engine")},
        "wall_s": wall32, "create_s": create_s, "step_s": step_s,
        "mcell_updates_per_s_stepping": step_mcell,
        "mcell_updates_per_s_e2e": cell_updates / wall32 / 1e6,
        "step_roofline": {"bytes_per_cell": (WORDS_E + WORDS_H) * B_ALG["fp32"],
                          "frac": step_mcell * 1e6 * (WORDS_E + WORDS_H) * B_ALG["fp32"] / 1e9 / peak / world,
                          "pct_of_8tbs": 100 * step_mcell * 1e6 * (WORDS_E + WORDS_H) * B_ALG["fp32"] / 1e9
                          / NOMINAL_HBM_GBS / world,
                          "peak": peak, "peak_kind": peak_kind,
                          "what": "stepping: cell-updates/s x 27 algorithmic words per cell, of measured"},
        "sweep_bytes_gbs_with_upml_aux": nbytes / step_s / 1e9 / world,
        "fp64_sequential_solves_per_s": sps64,
        "fp64_sample": {"solves": len(sample), "of": len(meshes), "wall_s": wall64_sample,
                        "what": "plain FP64 path, one solve after another (create, run, read back), on every "
                                f"{stride}-th mesh; whole-batch time = sample mean x {len(meshes)}"},
        "speedup_vs_fp64_sequential": sps32 / sps64, "target_speedup": 3.0,
        "grouped": (legs[True] and {"solves_per_s": solves / legs[True]["wall"] if world == 1 else None,
                                    "wall_s": legs[True]["wall"], "step_s": legs[True]["step"],
                                    "mcell_updates_per_s_stepping": cell_updates / legs[True]["step"] / 1e6,
                                    "gpu_launches": legs[True]["launches"],
                                    **{k: legs[True]["report"][k] for k in ("grouped", "rebuilds", "tiles",
                                                                            "group_ms")},
                                    "what": "the same batch through vgpu_run_grouped: one sweep launch per half "
                                            "step over every mesh's tiles, march depth and chunk autotuned"})
                   if True in legs else None,
        "tuning": tune_rec and {"march_depth": tune_rec["depth"], "blocks_per_sm": tune_rec["blocks_per_sm"],
                                "group_chunk": tune_rec["chunk"],
                                "tune_s": tune_rec["tune_s"], "sample_meshes": tune_rec["sample"],
                                "steps": tune_rec["steps"],
                                "trials": [{k: round(t[k], 1) if isinstance(t[k], float) else t[k]
                                            for k in ("depth", "blocks_per_sm", "chunk", "mcell_per_s")}
                                           for t in tune_rec["trials"]],
                                "what": "chosen before the timed batch by timing a sample of the meshes grouped"},
        "gpu_launches": launches, "clocks": clk.summary()}


def serve_workload(args, dist=None):
    """A seeded Poisson stream of solve requests (lognormal sizes, UPML or
    Mur, optional Debye block and TFSF source), FP32, served with admission
    by an HBM budget and continuous batching; the same stream solved one at a
    time by the plain FP64 path gives the comparison latencies."""
    import random

    import torch

    import vulture_b200 as vb
    from vulture_b200 import meshgen
    from vulture_b200.serve import Request, Server, latency_summary

    rank, world, local = rank_info()
    rng = random.Random(5 + rank)
    texts = [meshgen.serving_request(rng, q, nmin=48, nmax=args.serve_nmax, ntmin=args.serve_steps[0],
                                     ntmax=args.serve_steps[1]) for q in range(args.serve_count)]
    arrivals, t = [], 0.0
    for _ in texts:
        t += rng.expovariate(args.serve_rate)
        arrivals.append(t)
    d, paths = _meshes_dir(texts, "vb_serve_")
    warm = vb.Mesh(paths[0])
    for prec in ("fp32", "fp64"):
        vb.GpuRun(warm, prec).run(min(64, warm.num_steps)).close()
    torch.cuda.synchronize()
    cells = [vb.Mesh(p).num_cells for p in paths]

    def serve(prec, budget, slots):
        reqs = [Request(tx, arrival=a, precision=prec, tag=str(q)) for q, (tx, a) in enumerate(zip(texts, arrivals))]
        srv = Server(budget, max_active=slots)
        done = srv.run(reqs, keep_results=False)
        return srv, done

    if dist:
        dist.barrier()
    with ClockSampler(local) as clk:
        srv, done = serve("fp32", int(args.serve_budget_gb * 2**30), args.serve_slots)
    s32 = latency_summary(done)
    # Plain FP64: the same stream, one solve at a time.
    if dist:
        dist.barrier()
    srv64, done64 = serve("fp64", int(args.serve_budget_gb * 2**30), 1)
    s64 = latency_summary(done64)
    # Whole job: the worst rank's latencies, every rank's solves/s added.
    for summ in (s32, s64):
        for key in ("p50_s", "p99_s", "mean_s"):
            summ[key] = max_over_ranks(summ[key] if summ[key] is not None else float("inf"), dist)
        summ["solves_per_s"] = sum_over_ranks(summ["solves_per_s"], dist)
        summ["cell_updates"] = int(sum_over_ranks(summ["cell_updates"], dist))
    shutil.rmtree(d, ignore_errors=True)
    return {
        "metric": "p99 latency", "value": s32["p99_s"], "unit": "s", "n_gpus": world, "higher_is_better": False,
        "dtype": "fp32",
        "config": {"workload": f"{len(done)} requests, Poisson rate {args.serve_rate}/s, per-axis 48-"
                               f"{args.serve_nmax} lognormal, {args.serve_steps[0]}-{args.serve_steps[1]} "
                               f"steps, UPML or Mur, Debye, TFSF or dipole",
                   "budget_gb": args.serve_budget_gb, "slots": args.serve_slots,
                   "largest_request_cells": max(cells)},
        "fp32": s32, "fp64_one_at_a_time": s64,
        "p99_ratio_fp64_over_fp32": s64["p99_s"] / s32["p99_s"],
        "solves_per_s_ratio": s32["solves_per_s"] / s64["solves_per_s"],
        "peak_active": srv.peak_active, "peak_budget_bytes": srv.peak_bytes, "clocks": clk.summary()}


def _standalone(args, fn):
    """--workload batch|serve: the sub-object alone as the bench line."""
    import torch

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dist = init_dist(world)
    out = fn(args, dist)
    if rank == 0:
        out.setdefault("steps", 1)
        out.setdefault("warmup", 1)
        out.update({"scaling": "weak", "vs_baseline": None, "data": "synthetic"})
        if out.get("e2e_full_run"):
            f = out["e2e_full_run"]
            out["e2e"] = {"value": f["value"], "unit": f["unit"], "h2d_bytes_per_step": f["h2d_bytes"] / f["steps"],
                          "d2h_bytes_per_step": f["d2h_bytes"] / f["steps"], "what": "the whole run, create to read-back"}
        else:
            out["e2e"] = {"value": out["value"], "unit": out["unit"], "h2d_bytes_per_step": None,
                          "d2h_bytes_per_step": None}
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--workload", default="graded", choices=["graded", "enclosure", "batch", "serve"])
    ap.add_argument("--no-enclosure", action="store_true", help="graded workload without the enclosure sub-object")
    ap.add_argument("--no-full-run", action="store_true",
                    help="without the whole-run e2e legs (and the graded workload's FP32-error leg)")
    ap.add_argument("--no-batch", action="store_true", help="graded workload without the batch sub-object")
    ap.add_argument("--no-serve", action="store_true", help="graded workload without the serve sub-object")
    ap.add_argument("--enclosure-dims", type=int, nargs=3, default=[400, 300, 250],
                    help="cells per axis of the enclosure workload (its stated size by default; smaller for an ncu "
                         "capture)")
    ap.add_argument("--batch-count", type=int, default=256)
    ap.add_argument("--batch-steps", type=int, nargs=2, default=[2000, 8000])
    ap.add_argument("--batch-fp64-sample", type=int, default=32)
    ap.add_argument("--batch-mode", default="both", choices=["grouped", "streams", "both"],
                    help="streams: vgpu_run_batch, one stream per engine; grouped: vgpu_run_grouped (autotuned "
                         "tiles); both: the two, streams (the faster) as the value and grouped beside it")
    ap.add_argument("--serve-count", type=int, default=24)
    ap.add_argument("--serve-rate", type=float, default=6.0)
    ap.add_argument("--serve-nmax", type=int, default=256)
    ap.add_argument("--serve-steps", type=int, nargs=2, default=[2000, 20000])
    ap.add_argument("--serve-budget-gb", type=float, default=32.0)
    ap.add_argument("--serve-slots", type=int, default=4)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference_arm(args)
    elif args.workload == "enclosure":
        _standalone(args, lambda a, d: enclosure_workload(a, d, cpu=not a.no_cpu))
    elif args.workload == "batch":
        _standalone(args, batch_workload)
    elif args.workload == "serve":
        _standalone(args, serve_workload)
    else:
        run_gpu_arm(args)


if __name__ == "__main__":
    main()
