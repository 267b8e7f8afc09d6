"""ctypes bindings of the in-tree native library (include/vgpu.h, include/vhost.h).

The library is built in-tree by ``vulture_b200.build``; importing this module
fails loudly when it is missing -- there is no Python or CPU fallback for the
time loop.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libvulture_b200.so"

VGPU_FP64 = 0
VGPU_FP32 = 1

VGPU_OK = 0
VGPU_EINVAL = -1
VGPU_ENOMEM = -2
VGPU_ECUDA = -3
VGPU_ENODEV = -4
VGPU_ENONFINITE = -5
VGPU_ETIMEOUT = -6
VGPU_ECANCELLED = -7


class VgpuStats(C.Structure):
    _fields_ = [("run_ms", C.c_double), ("steps", C.c_uint64), ("kernel_launches", C.c_uint64),
                ("device_bytes", C.c_uint64), ("h2d_bytes", C.c_uint64), ("energy_e", C.c_double),
                ("energy_h", C.c_double), ("energy_step", C.c_uint64),
                ("merged_parts", C.c_uint32), ("reserved", C.c_uint32)]


class VgpuGroupReport(C.Structure):
    _fields_ = [("launches", C.c_uint64), ("grouped", C.c_int32), ("rebuilds", C.c_int32), ("tiles", C.c_int64),
                ("group_ms", C.c_double)]


# void sink(void *user, uint64_t first_row, uint32_t num_rows, int64_t num_points, const float *rows)
BIN_SINK = C.CFUNCTYPE(None, C.c_void_p, C.c_uint64, C.c_uint32, C.c_int64, C.POINTER(C.c_float))


class NativeError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"vulture_b200 native library not built: {LIB_PATH} (run python -m vulture_b200.build)")
    L = C.CDLL(str(LIB_PATH))
    P = C.c_void_p
    sig = {
        "vhost_load": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(P)]),
        "vhost_problem": (C.c_int, [P, C.c_int32, C.POINTER(P)]),
        "vhost_num_steps": (C.c_uint64, [P]),
        "vhost_num_output_steps": (C.c_uint64, [P]),
        "vhost_num_td": (C.c_int32, [P]),
        "vhost_num_fd": (C.c_int32, [P]),
        "vhost_num_freq": (C.c_int32, [P]),
        "vhost_dt": (C.c_double, [P]),
        "vhost_num_cells": (C.c_uint64, [P]),
        "vhost_use_tags": (C.c_int, [P, C.c_int32]),
        "vhost_check_tags": (C.c_int64, [P]),
        "vhost_write_outputs": (C.c_int, [P, P, C.c_uint64, P, P, C.c_int32]),
        "vhost_observer_name": (C.c_char_p, [P, C.c_int32, C.c_int32]),
        "vhost_num_bin": (C.c_int64, [P]),
        "vhost_bin_begin": (C.c_int, [P, C.c_int32]),
        "vhost_bin_sink": (None, [P, C.c_uint64, C.c_uint32, C.c_int64, P]),
        "vhost_bin_end": (C.c_int, [P]),
        "vhost_write_lines": (C.c_int, [P]),
        "vhost_free": (None, [P]),
        "vhost_last_error": (C.c_char_p, []),
        "vhost_main": (C.c_int, [C.c_int, C.POINTER(C.c_char_p)]),
        "vgpu_create": (C.c_int, [P, C.POINTER(P)]),
        "vgpu_run": (C.c_int, [P, C.c_uint64]),
        "vgpu_read_td": (C.c_int, [P, P, C.c_uint64]),
        "vgpu_read_dft": (C.c_int, [P, P, P]),
        "vgpu_read_field": (C.c_int, [P, C.c_int32, P]),
        "vgpu_write_field": (C.c_int, [P, C.c_int32, P]),
        "vgpu_check_finite": (C.c_int, [P]),
        "vgpu_current_step": (C.c_uint64, [P]),
        "vgpu_time_kernel": (C.c_int, [P, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_double),
                                       C.POINTER(C.c_uint64)]),
        "vgpu_get_stats": (C.c_int, [P, C.POINTER(VgpuStats)]),
        "vgpu_set_bin_sink": (C.c_int, [P, P, P]),
        "vgpu_sweep_points": (C.c_int, [P, C.c_int32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
        "vgpu_enqueue": (C.c_int, [P, C.c_uint64, C.POINTER(C.c_uint64)]),
        "vgpu_set_device": (C.c_int, [C.c_int32]),
        "vgpu_check_sweep_plan": (C.c_int, [P, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
        "vgpu_get_device": (C.c_int, [C.POINTER(C.c_int32)]),
        "vgpu_query": (C.c_int, [P]),
        "vgpu_synchronize": (C.c_int, [P]),
        "vgpu_run_batch": (C.c_int, [C.POINTER(P), C.c_int32, C.POINTER(C.c_uint64)]),
        "vgpu_set_sweep_wait_limit": (C.c_int, [C.c_int64]),
        "vgpu_run_grouped": (C.c_int, [C.POINTER(P), C.c_int32, C.POINTER(C.c_uint64),
                                       C.POINTER(VgpuGroupReport)]),
        "vgpu_groupable": (C.c_int, [P]),
        "vgpu_set_sweep_tuning": (C.c_int, [C.c_int32, C.c_int32, C.c_int32]),
        "vgpu_host_alloc": (C.c_void_p, [C.c_uint64]),
        "vgpu_host_free": (None, [C.c_void_p]),
        "vgpu_destroy": (None, [P]),
        "vgpu_last_error": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check_host(rc: int) -> None:
    if rc != 0:
        raise NativeError(rc, lib().vhost_last_error().decode(errors="replace"))


def check_gpu(rc: int) -> None:
    if rc != 0:
        raise NativeError(rc, lib().vgpu_last_error().decode(errors="replace"))


# Names of the C-ABI entry points, for export checks.
EXPORTS = ["vhost_load", "vhost_problem", "vhost_num_steps", "vhost_num_output_steps", "vhost_num_td",
           "vhost_num_fd", "vhost_num_freq", "vhost_dt", "vhost_num_cells", "vhost_write_outputs",
           "vhost_observer_name", "vhost_free", "vhost_last_error", "vhost_main", "vgpu_create", "vgpu_run",
           "vgpu_read_td", "vgpu_read_dft", "vgpu_read_field", "vgpu_write_field", "vgpu_check_finite",
           "vgpu_current_step", "vgpu_time_kernel", "vgpu_get_stats", "vgpu_destroy", "vgpu_last_error",
           "vgpu_set_bin_sink", "vgpu_dft_accumulate_static", "vhost_num_bin", "vhost_bin_begin", "vhost_bin_sink",
           "vhost_bin_end", "vhost_write_lines", "vgpu_sweep_points", "vgpu_enqueue", "vgpu_query",
           "vgpu_synchronize", "vgpu_run_batch", "vgpu_set_device", "vgpu_get_device",
           "vgpu_check_sweep_plan", "vgpu_set_sweep_wait_limit", "vgpu_run_grouped", "vgpu_groupable",
           "vgpu_set_sweep_tuning", "vgpu_host_alloc", "vgpu_host_free", "vhost_use_tags", "vhost_check_tags"]

VGPU_K_BULK_E, VGPU_K_BULK_H, VGPU_K_PML_E, VGPU_K_PML_H = 0, 1, 2, 3
# Other parts of a step and the 64-step DFT fold, for vgpu_time_kernel.
STEP_KERNELS = {
    "k_observe": 4, "k_bin_observe": 5, "k_mur_e": 6, "k_debye": 7, "k_sibc_e": 8, "k_source(E)": 9,
    "k_tfsf(E)": 10, "k_ghost(E)": 11, "k_mur_h": 12, "k_sibc_h": 13, "k_source(H)": 14, "k_tfsf(H)": 15,
    "k_ghost(H)": 16, "dft_fold_64": 17,
}
# Timing only: the scalar DFT fold the tensor-core fold replaced.
VGPU_K_DFT_BLOCK_SCALAR = 18
