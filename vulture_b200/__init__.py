"""vulture_b200: the Vulture FDTD time-stepping path on one NVIDIA B200.

The package holds the native library (host set-up in C99, CUDA engine for
sm_100a; C ABI in include/vgpu.h and include/vhost.h) and thin Python
front ends for it.
"""
from .solver import GpuRun, Mesh, run_batch, run_mesh  # noqa: F401

__all__ = ["Mesh", "GpuRun", "run_batch", "run_mesh"]
