"""Sweep tiling autotuner for grouped batches.

A grouped batch (vgpu_run_grouped) runs one sweep launch per half step over
the tiles of every mesh.  Three knobs shape those launches without changing
any result: the march depth (planes of i a tile walks, 1..32), a cap on
resident sweep blocks per SM, and the chunk of consecutive tiles a block
takes from its launch's counter at a time.  The built-in rule sizes tiles
for one mesh alone (about 16 tiles per SM); inside a group there are tiles
enough for longer marches, which re-read fewer halo planes, while larger
chunks change mesh less often but end a launch less evenly.

tune() measures instead of guessing: a sample of the batch's meshes (spread
over its sizes) is created at each candidate setting, stepped as a group for
a short run, and timed on the device; the fastest setting wins.  Results are
cached in a JSON file per (device, precision, size mix), so a later batch of
the same kind reuses them without timing.
"""
from __future__ import annotations

import json
import math
import os
import time
from pathlib import Path

from .solver import GpuRun, run_grouped, set_sweep_tuning

# (march depth, blocks per SM, group chunk); (0, 0, 0) is the built-in rule.
CANDIDATES = [(0, 0, 4), (0, 0, 16), (8, 0, 4), (8, 0, 16), (16, 0, 4), (32, 0, 2), (16, 2, 4)]


def cache_path() -> Path:
    p = os.environ.get("VULTURE_B200_TUNE_CACHE")
    if p:
        return Path(p)
    return Path(os.path.expanduser("~")) / ".cache" / "vulture_b200" / "autotune.json"


def size_class(cells: int) -> int:
    """floor(log4(cells)): one class spans a factor of 4 in cells."""
    return int(math.log(max(cells, 1), 4))


def signature(meshes, precision: str) -> str:
    """Device, precision and the batch's mix of size classes (shares rounded
    to tenths), the cache key of a tuning."""
    import torch

    dev = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    hist = {}
    for m in meshes:
        c = size_class(m.num_cells)
        hist[c] = hist.get(c, 0) + 1
    mix = ",".join(f"{c}:{round(n / len(meshes), 1)}" for c, n in sorted(hist.items()))
    return f"{dev}|{precision}|{mix}"


def _load(path: Path) -> dict:
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def _sample(meshes, count: int):
    """count meshes spread evenly over the batch sorted by size."""
    order = sorted(range(len(meshes)), key=lambda q: meshes[q].num_cells)
    if len(order) <= count:
        return [meshes[q] for q in order]
    return [meshes[order[round(k * (len(order) - 1) / (count - 1))]] for k in range(count)]


def time_setting(sample, precision: str, depth: int, blocks: int, chunk: int, steps: int) -> dict:
    """One candidate: the sample created under the setting and run as a
    group for `steps` steps (fewer where a mesh has fewer)."""
    set_sweep_tuning(depth, blocks, chunk)
    runs = []
    try:
        runs = [GpuRun(m, precision) for m in sample]
        nsteps = [min(steps, m.num_steps) for m in sample]
        rep = run_grouped(runs, nsteps)
    finally:
        for r in runs:
            r.close()
        set_sweep_tuning(0, 0, 0)
    cell_updates = sum(m.num_cells * n for m, n in zip(sample, nsteps))
    return {"depth": depth, "blocks_per_sm": blocks, "chunk": chunk, "group_ms": rep["group_ms"],
            "mcell_per_s": cell_updates / (rep["group_ms"] * 1e-3) / 1e6 if rep["group_ms"] > 0 else 0.0,
            "tiles": rep["tiles"]}


def tune(meshes, precision: str = "fp32", sample: int = 16, steps: int = 128, use_cache: bool = True):
    """The fastest (march depth, blocks per SM, group chunk) for grouped
    runs of meshes like these, and the record of how it was chosen."""
    key = signature(meshes, precision)
    path = cache_path()
    cache = _load(path) if use_cache else {}
    if key in cache:
        rec = dict(cache[key])
        rec["cached"] = True
        return (rec["depth"], rec["blocks_per_sm"], rec["chunk"]), rec
    picked = _sample(meshes, sample)
    t0 = time.perf_counter()
    # Untimed first pass: module load, kernel attributes, caches.
    time_setting(picked[:2], precision, 0, 0, 0, min(steps, 16))
    trials = [time_setting(picked, precision, d, b, c, steps) for d, b, c in CANDIDATES]
    best = max(trials, key=lambda t: t["mcell_per_s"])
    rec = {"depth": best["depth"], "blocks_per_sm": best["blocks_per_sm"], "chunk": best["chunk"], "trials": trials,
           "sample": len(picked), "steps": steps, "tune_s": time.perf_counter() - t0, "key": key}
    if use_cache:
        cache = _load(path)
        cache[key] = {k: rec[k] for k in ("depth", "blocks_per_sm", "chunk", "trials", "sample", "steps", "tune_s",
                                          "key")}
        try:
            path.parent.mkdir(parents=True, exist_ok=True)
            tmp = path.with_suffix(".tmp")
            tmp.write_text(json.dumps(cache, indent=1))
            tmp.replace(path)
        except OSError:
            pass
    rec["cached"] = False
    return (best["depth"], best["blocks_per_sm"], best["chunk"]), rec
