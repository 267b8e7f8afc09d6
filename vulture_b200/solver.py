"""Python front end of the drop-in solver path.

Mirrors the reference's flow (src/vulture.c:77-197): read a mesh and set up
(``Mesh``), advance the fields on the GPU (``GpuRun``), and write the same
observer files (``Mesh.write_outputs``).
"""
from __future__ import annotations

import ctypes as C
import os
from contextlib import contextmanager
from pathlib import Path

import numpy as np

from . import _native as N


@contextmanager
def _chdir(path):
    old = os.getcwd()
    os.chdir(path)
    try:
        yield
    finally:
        os.chdir(old)


class Mesh:
    """A parsed and set-up mesh: the reference's state before propagate()."""

    def __init__(self, path, log_path=None, verbose=False):
        self.path = str(Path(path).resolve())
        h = C.c_void_p()
        N.check_host(N.lib().vhost_load(self.path.encode(), log_path.encode() if log_path else None, int(verbose),
                                         C.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            N.lib().vhost_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def problem(self, precision: str = "fp64") -> C.c_void_p:
        p = C.c_void_p()
        prec = N.VGPU_FP64 if precision == "fp64" else N.VGPU_FP32
        N.check_host(N.lib().vhost_problem(self._h, prec, C.byref(p)))
        return p

    @property
    def num_steps(self) -> int:
        return int(N.lib().vhost_num_steps(self._h))

    @property
    def num_output_steps(self) -> int:
        return int(N.lib().vhost_num_output_steps(self._h))

    @property
    def num_td(self) -> int:
        return int(N.lib().vhost_num_td(self._h))

    @property
    def num_fd(self) -> int:
        return int(N.lib().vhost_num_fd(self._h))

    @property
    def num_bin(self) -> int:
        """Nodes over all TDOM_BINARY observers."""
        return int(N.lib().vhost_num_bin(self._h))

    @property
    def num_freq(self) -> int:
        return int(N.lib().vhost_num_freq(self._h))

    @property
    def dt(self) -> float:
        return float(N.lib().vhost_dt(self._h))

    @property
    def num_cells(self) -> int:
        """Outer-box cells, the reference's spi/cell denominator."""
        return int(N.lib().vhost_num_cells(self._h))

    def use_tags(self, use: bool = True):
        """Hand the engine the set-up's medium tags (the default), or leave
        them out so that it scans the coefficient volumes instead."""
        N.check_host(N.lib().vhost_use_tags(self._h, int(use)))

    def check_tags(self) -> int:
        """(cell, component) pairs whose medium tag disagrees with the
        coefficient volumes; -1 when the set-up kept no tags."""
        return int(N.lib().vhost_check_tags(self._h))

    def observer_name(self, fd: bool, slot: int) -> str:
        return N.lib().vhost_observer_name(self._h, int(fd), slot).decode()

    def empty_outputs(self):
        td = np.zeros((max(self.num_output_steps, 1), max(self.num_td, 1), 6))
        re = np.zeros((max(self.num_fd, 1), 6, max(self.num_freq, 1)))
        return td, re, np.zeros_like(re)

    def write_outputs(self, directory, td, re, im, full_precision=False):
        td = np.ascontiguousarray(td, dtype=np.float64)
        re = np.ascontiguousarray(re, dtype=np.float64)
        im = np.ascontiguousarray(im, dtype=np.float64)
        Path(directory).mkdir(parents=True, exist_ok=True)
        with _chdir(directory):
            N.check_host(N.lib().vhost_write_outputs(self._h, td.ctypes.data, self.num_output_steps,
                                                     re.ctypes.data, im.ctypes.data, int(full_precision)))


    def write_lines(self, directory):
        """xlines.dat / ylines.dat / zlines.dat, as the reference's set-up writes them."""
        Path(directory).mkdir(parents=True, exist_ok=True)
        with _chdir(directory):
            N.check_host(N.lib().vhost_write_lines(self._h))

    def bin_begin(self, directory, full_precision=False):
        """impulse.dat header, excite.dat and process.dat (no-op without binary observers)."""
        Path(directory).mkdir(parents=True, exist_ok=True)
        with _chdir(directory):
            N.check_host(N.lib().vhost_bin_begin(self._h, int(full_precision)))

    def bin_append(self, rows):
        """Append binary-observer rows [n][num_bin][6] (float32) to impulse.dat."""
        r = np.ascontiguousarray(rows, dtype=np.float32)
        if r.size:
            N.lib().vhost_bin_sink(self._h, 0, r.shape[0], self.num_bin, r.ctypes.data)

    def bin_end(self):
        N.check_host(N.lib().vhost_bin_end(self._h))

    def write_binary(self, directory, rows, full_precision=False):
        """All binary-observer files from rows sampled elsewhere."""
        self.bin_begin(directory, full_precision)
        self.bin_append(rows)
        self.bin_end()


class _HostBlock:
    """Owner of a page-locked host block from the library's cache, exposed to
    numpy: the array keeps this object alive and the block returns to the
    cache when the array goes."""

    def __init__(self, shape, dtype):
        nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
        self.ptr = N.lib().vgpu_host_alloc(nbytes)
        self.__array_interface__ = {"shape": tuple(shape), "typestr": np.dtype(dtype).str,
                                    "data": (self.ptr or 0, False), "version": 3}

    def __del__(self):
        try:
            if self.ptr:
                N.lib().vgpu_host_free(self.ptr)
        except Exception:
            pass


def _result_array(shape, dtype=np.float64):
    """An uninitialised array for a large read-back: page-locked, so the
    device writes it directly (a fresh pageable array costs a page fault per
    4 KB as the staged copy first touches it); small ones are plain numpy."""
    if int(np.prod(shape)) * np.dtype(dtype).itemsize >= (4 << 20):
        blk = _HostBlock(shape, dtype)
        if blk.ptr:
            return np.asarray(blk)
    return np.empty(shape, dtype)


class GpuRun:
    """An engine instance on the current CUDA device (vgpu_create/run)."""

    def __init__(self, mesh: Mesh, precision: str = "fp64"):
        self.mesh = mesh
        self.precision = precision
        e = C.c_void_p()
        N.check_gpu(N.lib().vgpu_create(mesh.problem(precision), C.byref(e)))
        self._e = e

    def run(self, nsteps=None):
        n = self.mesh.num_steps - self.step if nsteps is None else nsteps
        N.check_gpu(N.lib().vgpu_run(self._e, n))
        return self

    def collect_bin(self):
        """Keep every binary-observer row the engine delivers (see bin())."""
        self._bin_rows = []
        npts = self.mesh.num_bin

        def sink(user, first_row, num_rows, num_points, rows):
            a = np.ctypeslib.as_array(rows, shape=(num_rows * num_points * 6,))
            self._bin_rows.append((first_row, a.reshape(num_rows, num_points, 6).copy()))

        self._bin_cb = N.BIN_SINK(sink)
        N.check_gpu(N.lib().vgpu_set_bin_sink(self._e, C.cast(self._bin_cb, C.c_void_p), None))
        self._bin_npts = npts
        return self

    def stream_bin_to(self, mesh: Mesh):
        """Send binary-observer rows straight to the mesh's impulse.dat writer."""
        fn = C.cast(N.lib().vhost_bin_sink, C.c_void_p)
        N.check_gpu(N.lib().vgpu_set_bin_sink(self._e, fn, mesh._h))
        return self

    def bin(self):
        """Collected rows [rows][num_bin][6] float32, in delivery order."""
        if not getattr(self, "_bin_rows", None):
            return np.zeros((0, self.mesh.num_bin, 6), dtype=np.float32)
        return np.concatenate([r for _, r in self._bin_rows], axis=0)

    def bin_first_rows(self):
        return [f for f, _ in getattr(self, "_bin_rows", [])]

    @property
    def step(self) -> int:
        return int(N.lib().vgpu_current_step(self._e))

    @property
    def groupable(self) -> bool:
        """Whether the engine can step in a group (vgpu_groupable)."""
        rc = N.lib().vgpu_groupable(self._e)
        if rc < 0:
            N.check_gpu(rc)
        return rc == 1

    def enqueue(self, max_steps: int = 64) -> int:
        """Queue up to max_steps more steps (one 64-step block at most) without
        waiting; returns the steps queued, 0 once the problem is done."""
        q = C.c_uint64()
        N.check_gpu(N.lib().vgpu_enqueue(self._e, max_steps, C.byref(q)))
        return q.value

    def done(self) -> bool:
        """True when the queued steps have finished on the device; raises
        NativeError when the engine's stream reports a device error."""
        rc = N.lib().vgpu_query(self._e)
        if rc < 0:
            N.check_gpu(rc)
        return rc == 1

    def synchronize(self):
        N.check_gpu(N.lib().vgpu_synchronize(self._e))
        return self

    def stats(self) -> N.VgpuStats:
        st = N.VgpuStats()
        N.check_gpu(N.lib().vgpu_get_stats(self._e, C.byref(st)))
        return st

    def td(self, steps=None):
        m = self.mesh
        steps = m.num_output_steps if steps is None else steps
        out = np.zeros((max(steps, 1), max(m.num_td, 1), 6))
        if m.num_td:
            N.check_gpu(N.lib().vgpu_read_td(self._e, out.ctypes.data, steps))
        return out

    def dft(self):
        m = self.mesh
        if not m.num_fd or not m.num_freq:
            z = np.zeros((max(m.num_fd, 1), 6, max(m.num_freq, 1)))
            return z, z.copy()
        # Filled entirely by the read: no zero-fill of a buffer about to be overwritten.
        re = _result_array((m.num_fd, 6, max(m.num_freq, 1)))
        im = _result_array(re.shape)
        N.check_gpu(N.lib().vgpu_read_dft(self._e, re.ctypes.data, im.ctypes.data))
        return re, im

    def field(self, comp: int, shape):
        out = np.empty(shape)
        N.check_gpu(N.lib().vgpu_read_field(self._e, comp, out.ctypes.data))
        return out

    def write_field(self, comp: int, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        N.check_gpu(N.lib().vgpu_write_field(self._e, comp, v.ctypes.data))

    def time_kernel(self, kernel: int, warmup=3, iters=20):
        """Mean device ms per launch of one step kernel, and its field points."""
        ms = C.c_double()
        pts = C.c_uint64()
        N.check_gpu(N.lib().vgpu_time_kernel(self._e, kernel, warmup, iters, C.byref(ms), C.byref(pts)))
        return ms.value, pts.value

    def sweep_points(self, kernel: int):
        """(bulk, UPML) field points one sweep kernel updates per launch."""
        b, q = C.c_uint64(), C.c_uint64()
        N.check_gpu(N.lib().vgpu_sweep_points(self._e, kernel, C.byref(b), C.byref(q)))
        return b.value, q.value

    def check_finite(self):
        N.check_gpu(N.lib().vgpu_check_finite(self._e))

    def close(self):
        if self._e:
            N.lib().vgpu_destroy(self._e)
            self._e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_batch(runs, steps=None):
    """Advance several GpuRun engines of one device together (vgpu_run_batch):
    steps[i] more steps each (default: to the end of each problem)."""
    n = len(runs)
    if steps is None:
        steps = [r.mesh.num_steps - r.step for r in runs]
    arr = (C.c_void_p * n)(*[r._e.value for r in runs])
    st = (C.c_uint64 * n)(*steps)
    N.check_gpu(N.lib().vgpu_run_batch(arr, n, st))
    return runs


def run_grouped(runs, steps=None):
    """Advance several GpuRun engines of one device together with grouped
    launches (vgpu_run_grouped): the engines that allow it share one sweep
    launch per half step; steps[i] more steps each (default: to the end of
    each problem).  Returns the call's report as a dict."""
    n = len(runs)
    if steps is None:
        steps = [r.mesh.num_steps - r.step for r in runs]
    arr = (C.c_void_p * n)(*[r._e.value for r in runs])
    st = (C.c_uint64 * n)(*steps)
    rep = N.VgpuGroupReport()
    N.check_gpu(N.lib().vgpu_run_grouped(arr, n, st, C.byref(rep)))
    return {"launches": int(rep.launches), "grouped": int(rep.grouped), "rebuilds": int(rep.rebuilds),
            "tiles": int(rep.tiles), "group_ms": float(rep.group_ms)}


def set_sweep_tuning(march_depth: int = 0, blocks_per_sm: int = 0, group_chunk: int = 0) -> None:
    """Sweep tiling for engines this thread creates afterwards and groups it
    runs: planes per tile (0: the built-in rule), a cap on resident sweep
    blocks per SM (0: none) and the tiles a grouped sweep block takes at a
    time (0: 4).  Results do not depend on it."""
    N.check_gpu(N.lib().vgpu_set_sweep_tuning(int(march_depth), int(blocks_per_sm), int(group_chunk)))


def run_mesh(mesh_path, out_dir, precision="fp64", full_precision=False):
    """The reference's command-line flow on the GPU: set up, propagate, write outputs."""
    m = Mesh(mesh_path)
    m.write_lines(out_dir)
    m.bin_begin(out_dir, full_precision)
    g = GpuRun(m, precision)
    if m.num_bin:
        g.stream_bin_to(m)
    g.run()
    m.bin_end()
    re, im = g.dft()
    m.write_outputs(out_dir, g.td(), re, im, full_precision)
    g.close()
    return m
