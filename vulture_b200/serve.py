"""Serving loop over the asynchronous engine entry points.

Solve requests (a mesh text, an arrival time and a precision) are admitted
while their estimated device footprint fits an HBM budget, and the admitted
solves share the device by continuous batching: every turn each active solve
whose stream has drained gets its next 64-step blocks queued
(vgpu_enqueue), a finished solve is retired at once (its observers read, its
memory freed) and the next waiting request takes its place.  Each solve runs
on its own engine and stream, so its results are the ones a solo run gives.

The reference runs one mesh per process (src/vulture.c:77-197); serving has
no counterpart there and is built on the same per-mesh engine.
"""
from __future__ import annotations

import os
import tempfile
import time
from collections import deque
from dataclasses import dataclass

import numpy as np

from .solver import GpuRun, Mesh

_WORD = {"fp32": 4, "fp64": 8}


@dataclass
class Request:
    mesh_text: str
    arrival: float = 0.0          # seconds after the start of Server.run
    precision: str = "fp32"
    tag: str = ""
    admitted: float | None = None
    completed: float | None = None
    cell_updates: int = 0
    td: np.ndarray | None = None
    dft: tuple | None = None
    device_bytes: int = 0         # the engine's own count once created
    estimate: int = 0             # the admission estimate

    @property
    def latency(self) -> float:
        return self.completed - self.arrival


def footprint_estimate(mesh: Mesh, precision: str) -> int:
    """Upper estimate of an engine's device bytes: six field volumes, up to
    nine coefficient or auxiliary volumes and the index bytes, with 30 %
    slack for padding and boundary lists, plus observer buffers and a fixed
    64 MB for the per-engine blocks (DFT staging, TFSF lists, headers)."""
    w = _WORD[precision]
    cells = mesh.num_cells
    vol = int(1.3 * cells * (15 * w + 2))
    obs = (mesh.num_td * 6 * mesh.num_output_steps * 8 + mesh.num_fd * 6 * (2 * mesh.num_freq * 8 + 64 * w))
    return vol + obs + (64 << 20)


class Server:
    """Admission by HBM budget plus continuous batching of 64-step blocks."""

    def __init__(self, budget_bytes: int, max_inflight_blocks: int = 2, block_steps: int = 64):
        self.budget = int(budget_bytes)
        self.max_inflight = max(1, int(max_inflight_blocks))
        self.block_steps = block_steps
        self.peak_bytes = 0
        self.peak_active = 0

    def run(self, requests, keep_results: bool = True):
        """Serve the requests (sorted by arrival); returns them completed."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        pending = deque(reqs)
        waiting: deque = deque()
        active = []                     # (request, mesh, run, path)
        used = 0
        head = None                     # the parsed mesh of the next request to admit
        tmp = tempfile.mkdtemp(prefix="vgpu_serve_")
        t0 = time.perf_counter()
        try:
            while pending or waiting or active:
                now = time.perf_counter() - t0
                while pending and pending[0].arrival <= now:
                    waiting.append(pending.popleft())
                # Admission: first come, first served, while the estimate fits
                # (a request larger than the whole budget runs alone).
                while waiting:
                    r = waiting[0]
                    if head is None or head[0] is not r:
                        path = os.path.join(tmp, f"req{id(r)}.msh")
                        with open(path, "w") as f:
                            f.write(r.mesh_text)
                        mesh = Mesh(path)
                        head = (r, mesh, path, footprint_estimate(mesh, r.precision))
                    _, mesh, path, est = head
                    if active and used + est > self.budget:
                        break
                    waiting.popleft()
                    head = None
                    r.estimate = est
                    r.admitted = time.perf_counter() - t0
                    run = GpuRun(mesh, r.precision)
                    r.device_bytes = int(run.stats().device_bytes)
                    used += est
                    active.append((r, mesh, run, path))
                self.peak_bytes = max(self.peak_bytes, used)
                self.peak_active = max(self.peak_active, len(active))
                progressed = False
                still = []
                for r, mesh, run, path in active:
                    if not run.done():
                        still.append((r, mesh, run, path))
                        continue
                    if run.step >= mesh.num_steps:
                        run.synchronize()
                        r.completed = time.perf_counter() - t0
                        r.cell_updates = mesh.num_cells * mesh.num_steps
                        if keep_results:
                            r.td = run.td()
                            r.dft = run.dft()
                        run.close()
                        mesh.close()
                        os.unlink(path)
                        used -= r.estimate
                        progressed = True
                        continue
                    for _ in range(self.max_inflight):
                        if not run.enqueue(self.block_steps):
                            break
                    progressed = True
                    still.append((r, mesh, run, path))
                active = still
                if not progressed:
                    if not active and pending:
                        time.sleep(max(0.0, min(pending[0].arrival - (time.perf_counter() - t0), 0.01)))
                    else:
                        time.sleep(50e-6)
        finally:
            for r, mesh, run, path in active:
                run.close()
                mesh.close()
            if head is not None:
                head[1].close()
            try:
                for f in os.listdir(tmp):
                    os.unlink(os.path.join(tmp, f))
                os.rmdir(tmp)
            except OSError:
                pass
        return reqs


def latency_summary(reqs):
    """p50 / p99 latency (arrival to completion) and completed solves/s."""
    lat = np.array([r.latency for r in reqs])
    span = max(r.completed for r in reqs) - min(r.arrival for r in reqs)
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "solves_per_s": len(reqs) / span if span > 0 else float("inf"),
            "cell_updates": int(sum(r.cell_updates for r in reqs))}
