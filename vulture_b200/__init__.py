"""vulture_b200: the Vulture FDTD time-stepping path on one NVIDIA B200.

The package holds the native library (host set-up in C99, CUDA engine for
sm_100a; C ABI in include/vgpu.h and include/vhost.h) and thin Python
front ends for it.
"""
import os as _os

# Many engines step side by side on their own streams; with the default 8
# hardware work queues, streams share queues and a set-up copy or kernel of
# one engine waits behind another's queued graphs.  32 queues (the most)
# avoid that; the setting only takes effect if the process has not yet
# created its CUDA context.
_os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

from .solver import GpuRun, Mesh, run_batch, run_grouped, run_mesh, set_sweep_tuning  # noqa: E402,F401

__all__ = ["Mesh", "GpuRun", "run_batch", "run_grouped", "run_mesh", "set_sweep_tuning"]
