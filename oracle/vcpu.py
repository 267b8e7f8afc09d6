"""ORACLE (test infrastructure only): ctypes binding of oracle/vcpu.c.

Runs the CPU restatement of the time loop on the same vgpu_problem the GPU
engine receives.  Imported only by tests/, the smoke check and bench.py's
CPU-baseline leg.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "_build" / "libvcpu.so"
_lib = {}


def _load():
    if "L" in _lib:
        return _lib["L"]
    if not LIB.exists():
        raise ImportError(f"oracle library not built: {LIB}")
    L = C.CDLL(str(LIB))
    for pre in ("vcpu64_", "vcpu32_"):
        getattr(L, pre + "create").restype = C.c_void_p
        getattr(L, pre + "create").argtypes = [C.c_void_p]
        getattr(L, pre + "destroy").argtypes = [C.c_void_p]
        getattr(L, pre + "run").argtypes = [C.c_void_p, C.c_uint64]
        getattr(L, pre + "read_td").argtypes = [C.c_void_p, C.c_void_p, C.c_uint64]
        getattr(L, pre + "read_bin").argtypes = [C.c_void_p, C.c_void_p, C.c_uint64]
        getattr(L, pre + "read_dft").argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        getattr(L, pre + "read_field").argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
        getattr(L, pre + "write_field").argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
    _lib["L"] = L
    return L


class CpuRun:
    """The oracle time loop on a problem from vulture_b200.Mesh.problem()."""

    def __init__(self, mesh, precision="fp64"):
        self.mesh = mesh
        self.pre = "vcpu64_" if precision == "fp64" else "vcpu32_"
        L = _load()
        self._h = getattr(L, self.pre + "create")(mesh.problem(precision))
        self.step = 0

    def _f(self, name):
        return getattr(_load(), self.pre + name)

    def run(self, nsteps=None):
        n = self.mesh.num_steps - self.step if nsteps is None else nsteps
        self._f("run")(self._h, n)
        self.step += n
        return self

    def td(self, steps=None):
        m = self.mesh
        steps = m.num_output_steps if steps is None else steps
        out = np.zeros((max(steps, 1), max(m.num_td, 1), 6))
        if m.num_td:
            self._f("read_td")(self._h, out.ctypes.data, steps)
        return out

    def bin(self, steps=None):
        """Binary-observer rows [steps][num_bin][6] as float32."""
        m = self.mesh
        steps = m.num_output_steps if steps is None else steps
        out = np.zeros((steps, m.num_bin, 6), dtype=np.float32)
        if m.num_bin and steps:
            self._f("read_bin")(self._h, out.ctypes.data, steps)
        return out

    def dft(self):
        m = self.mesh
        re = np.zeros((max(m.num_fd, 1), 6, max(m.num_freq, 1)))
        im = np.zeros_like(re)
        if m.num_fd:
            self._f("read_dft")(self._h, re.ctypes.data, im.ctypes.data)
        return re, im

    def field(self, comp, shape):
        out = np.zeros(shape)
        self._f("read_field")(self._h, comp, out.ctypes.data)
        return out

    def write_field(self, comp, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        self._f("write_field")(self._h, comp, v.ctypes.data)

    def close(self):
        if self._h:
            self._f("destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
