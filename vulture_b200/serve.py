"""Serving loop over the asynchronous engine entry points.

Solve requests (a mesh text, an arrival time and a precision) are admitted
first come, first served while a solve slot is free and their estimated
device footprint fits an HBM budget.  The admitted solves share the device
by continuous batching: every turn each active solve whose stream has
drained gets its next 64-step blocks queued (vgpu_enqueue), a finished solve
is retired at once (its observers read, its memory freed) and the next
waiting request takes its place.  Mesh set-up and engine creation run on
worker threads, so the device keeps stepping the active solves meanwhile.
Each solve runs on its own engine and stream, so its results are the ones a
solo run gives.

The reference runs one mesh per process (src/vulture.c:77-197); serving has
no counterpart there and is built on the same per-mesh engine.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .solver import GpuRun, Mesh, run_batch, run_grouped, set_sweep_tuning

_WORD = {"fp32": 4, "fp64": 8}


@dataclass
class Request:
    mesh_text: str
    arrival: float = 0.0          # seconds after the start of Server.run
    precision: str = "fp32"
    tag: str = ""
    admitted: float | None = None
    started: float | None = None  # engine created, first block queued
    completed: float | None = None
    cell_updates: int = 0
    td: np.ndarray | None = None
    dft: tuple | None = None
    device_bytes: int = 0         # the engine's own count once created
    estimate: int = 0             # the admission estimate
    error: str | None = None      # why the solve failed (bad mesh, engine error); None if it ran

    @property
    def latency(self) -> float:
        return self.completed - self.arrival


def _worker_pool(workers: int) -> ThreadPoolExecutor:
    """Threads that create engines on the calling thread's CUDA device (a
    thread's current device is its own).  Without a device the workers keep
    their default; creating an engine then reports the missing device."""
    dev = C.c_int32(-1)
    if N.lib().vgpu_get_device(C.byref(dev)) != 0:
        dev.value = -1

    def init():
        if dev.value >= 0:
            N.check_gpu(N.lib().vgpu_set_device(dev.value))

    return ThreadPoolExecutor(workers, initializer=init)


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
    """Admission by solve slots and HBM budget, continuous batching of
    64-step blocks.

    budget_bytes: device bytes the admitted solves may hold together (by
    their estimates); a request larger than the whole budget runs alone.
    max_active: solves stepping side by side.  max_inflight_blocks: blocks
    queued per solve each time its stream drains.  workers: host threads
    that parse meshes and create engines (two creations side by side kept
    the p99 lower than one at a time, measured).  poll_s: pause between
    polls of the streams when nothing changed.
    """

    def __init__(self, budget_bytes: int, max_active: int = 4, max_inflight_blocks: int = 2,
                 block_steps: int = 64, workers: int = 2, poll_s: float = 2e-4):
        self.budget = int(budget_bytes)
        self.max_active = max(1, int(max_active))
        self.max_inflight = max(1, int(max_inflight_blocks))
        self.block_steps = block_steps
        self.workers = max(1, int(workers))
        self.poll_s = poll_s
        self.peak_bytes = 0
        self.peak_active = 0

    @staticmethod
    def _fail(r: Request, exc: BaseException, t0: float):
        r.error = f"{type(exc).__name__}: {exc}"
        r.completed = time.perf_counter() - t0

    def run(self, requests, keep_results: bool = True):
        """Serve the requests (sorted by arrival); returns them completed.
        A request whose mesh does not parse, or whose engine cannot be
        created or reports a device error, completes with `error` set; the
        others are not affected."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        pending = deque(reqs)
        waiting: deque = deque()      # arrived, not admitted: [request, parse future]
        creating = []                 # admitted: (request, mesh, path, create future)
        active = []                   # stepping: (request, mesh, run, path)
        used = 0
        tmp = tempfile.mkdtemp(prefix="vgpu_serve_")
        pool = _worker_pool(self.workers)      # mesh parsing and engine creation

        def parse(r):
            path = os.path.join(tmp, f"req{id(r)}.msh")
            with open(path, "w") as f:
                f.write(r.mesh_text)
            mesh = Mesh(path)
            return mesh, path, footprint_estimate(mesh, r.precision)

        t0 = time.perf_counter()
        try:
            while pending or waiting or creating or active:
                now = time.perf_counter() - t0
                while pending and pending[0].arrival <= now:
                    waiting.append([pending.popleft(), None])
                # Parse the first few waiting meshes ahead of admission.
                for w in list(waiting)[: self.workers]:
                    if w[1] is None:
                        w[1] = pool.submit(parse, w[0])
                # Admission, first come first served.  A mesh that fails to
                # parse fails its request only.
                while (waiting and waiting[0][1] is not None and waiting[0][1].done()
                       and len(active) + len(creating) < self.max_active):
                    r, fut = waiting[0]
                    if fut.exception() is not None:
                        waiting.popleft()
                        self._fail(r, fut.exception(), t0)
                        continue
                    mesh, path, est = fut.result()
                    if (active or creating) and used + est > self.budget:
                        break
                    waiting.popleft()
                    if len(waiting) >= self.workers and waiting[self.workers - 1][1] is None:
                        waiting[self.workers - 1][1] = pool.submit(parse, waiting[self.workers - 1][0])
                    r.estimate = est
                    r.admitted = time.perf_counter() - t0
                    used += est
                    creating.append((r, mesh, path, pool.submit(GpuRun, mesh, r.precision)))
                self.peak_bytes = max(self.peak_bytes, used)
                progressed = False
                still_creating = []
                for r, mesh, path, fut in creating:
                    if fut.done() and fut.exception() is not None:
                        # The engine could not be created (device memory, a
                        # problem the engine refuses): this request fails.
                        self._fail(r, fut.exception(), t0)
                        mesh.close()
                        os.unlink(path)
                        used -= r.estimate
                        progressed = True
                    elif fut.done():
                        run = fut.result()
                        r.device_bytes = int(run.stats().device_bytes)
                        r.started = time.perf_counter() - t0
                        active.append((r, mesh, run, path))
                        progressed = True
                    else:
                        still_creating.append((r, mesh, path, fut))
                creating = still_creating
                self.peak_active = max(self.peak_active, len(active))
                still = []
                for r, mesh, run, path in active:
                    try:
                        # A device error on the solve's stream ends the solve
                        # here, instead of reading as work still in flight.
                        finished = run.done()
                        if finished and run.step >= mesh.num_steps:
                            run.synchronize()
                            if keep_results:
                                r.td = run.td()
                                r.dft = run.dft()
                    except N.NativeError as exc:   # a device-side failure of this solve
                        self._fail(r, exc, t0)
                        run.close()
                        mesh.close()
                        os.unlink(path)
                        used -= r.estimate
                        progressed = True
                        continue
                    if not finished:
                        still.append((r, mesh, run, path))
                        continue
                    if run.step >= mesh.num_steps:
                        r.completed = time.perf_counter() - t0
                        r.cell_updates = mesh.num_cells * mesh.num_steps
                        run.close()
                        mesh.close()
                        os.unlink(path)
                        used -= r.estimate
                        progressed = True
                        continue
                    try:
                        for _ in range(self.max_inflight):
                            if not run.enqueue(self.block_steps):
                                break
                    except N.NativeError as exc:
                        self._fail(r, exc, t0)
                        run.close()
                        mesh.close()
                        os.unlink(path)
                        used -= r.estimate
                        progressed = True
                        continue
                    progressed = True
                    still.append((r, mesh, run, path))
                active = still
                if not progressed:
                    if not active and not creating and not waiting and pending:
                        time.sleep(max(0.0, min(pending[0].arrival - (time.perf_counter() - t0), 0.01)))
                    else:
                        time.sleep(self.poll_s)
        finally:
            pool.shutdown(wait=True)
            for r, mesh, run, path in active:
                run.close()
                mesh.close()
            for r, mesh, path, fut in creating:
                if fut.exception() is None:
                    fut.result().close()
                mesh.close()
            for r, fut in waiting:
                if fut is not None and fut.exception() is None:
                    fut.result()[0].close()
            try:
                for f in os.listdir(tmp):
                    os.unlink(os.path.join(tmp, f))
                os.rmdir(tmp)
            except OSError:
                pass
        return reqs


def solve_batch(meshes, precision: str = "fp32", budget_bytes: int | None = None, on_done=None,
                grouped: bool = False, tuning=None):
    """Solve independent meshes to their last step on the current device.

    The engines are created one after another, then advanced together.  By
    default vgpu_run_batch queues every engine's blocks round-robin on its
    own stream.  grouped=True: vgpu_run_grouped steps the engines that allow
    it as one group, one sweep launch per half step over every mesh's tiles,
    and the rest beside it.  On the 256-mesh batch of 32-160 cells per axis
    the streams step 11% faster: an engine's H sweep follows its own E sweep
    while that mesh's fields are still in L2, where a grouped half step
    sweeps every mesh before any H sweep starts.  Either way the call
    returns when all have finished.  tuning: (march depth, blocks per SM, group chunk)
    for the engines' sweep tiles and the group's launches, or "auto" to have
    autotune.tune() choose (timed on a sample of the meshes, cached).  Creation is neither spread over threads nor
    overlapped with stepping: both were measured, and engine creations that
    run beside other creations or beside stepping engines wait on each
    other's device allocations and copies (32 engines: 0.17 s one after
    another, 1.3-1.7 s on three threads).

    Without budget_bytes every mesh is solved in one wave and the finished
    GpuRun objects are returned in the meshes' order, their results ready to
    read; each carries batch_started (its wave's engines created) and
    batch_finished, seconds from the call, batch_report (vgpu_run_grouped's
    counts, None without grouping) and batch_tuning (the autotuner's record,
    None unless tuning="auto").  With budget_bytes, meshes are
    taken in order into waves whose footprint estimates fit the budget (a
    mesh larger than the budget forms a wave alone); on_done(index, run) is
    called for each finished solve of a wave, after which the engine is
    closed to make room for the next wave, and the call returns None."""
    t0 = time.perf_counter()
    tune_rec = None
    if tuning == "auto":
        if not grouped:
            raise ValueError('tuning="auto" tunes grouped launches: pass grouped=True')
        from . import autotune

        tuning, tune_rec = autotune.tune(meshes, precision)
    if budget_bytes is None:
        waves = [list(range(len(meshes)))]
    else:
        waves, cur, used = [], [], 0
        for q, m in enumerate(meshes):
            est = footprint_estimate(m, precision)
            if cur and used + est > budget_bytes:
                waves.append(cur)
                cur, used = [], 0
            cur.append(q)
            used += est
        if cur:
            waves.append(cur)
    result = [None] * len(meshes)
    for wave in waves:
        runs = []
        handed_over = False
        try:
            if tuning:
                set_sweep_tuning(*tuning)
            try:
                for q in wave:
                    runs.append(GpuRun(meshes[q], precision))
            finally:
                if tuning:
                    set_sweep_tuning(0, 0, 0)
            started = time.perf_counter() - t0
            if grouped:
                if tuning:
                    set_sweep_tuning(*tuning)
                try:
                    report = run_grouped(runs)
                finally:
                    if tuning:
                        set_sweep_tuning(0, 0, 0)
            else:
                run_batch(runs)
                report = None
            finished = time.perf_counter() - t0
            for r in runs:
                r.batch_report, r.batch_tuning = report, tune_rec
            for q, r in zip(wave, runs):
                r.batch_started, r.batch_finished = started, finished
            if budget_bytes is None:
                for q, r in zip(wave, runs):
                    result[q] = r
                handed_over = True
            elif on_done is not None:
                for q, r in zip(wave, runs):
                    on_done(q, r)
        finally:
            # Every engine of a budgeted wave is freed before the next wave,
            # and on any error (creation, stepping, a failing callback) no
            # engine of the wave outlives the call.
            if not handed_over:
                for r in runs:
                    r.close()
    return result if budget_bytes is None else None


def latency_summary(reqs):
    """p50 / p99 latency (arrival to completion), mean and solves/s over the
    requests that ran; failed requests are counted apart."""
    ok = [r for r in reqs if r.error is None]
    failed = len(reqs) - len(ok)
    if not ok:
        return {"p50_s": None, "p99_s": None, "mean_s": None, "solves_per_s": 0.0, "cell_updates": 0,
                "failed": failed}
    lat = np.array([r.latency for r in ok])
    span = max(r.completed for r in ok) - min(r.arrival for r in ok)
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()),
            "solves_per_s": len(ok) / span if span > 0 else float("inf"),
            "cell_updates": int(sum(r.cell_updates for r in ok)), "failed": failed}
