"""The allocation-free DFT entry point (vgpu_dft_accumulate_static).

It serves callers that cannot allocate device memory: they own every
buffer, and the entry point keeps its own scratch in a fixed device array.
This file is named to be collected last, so a run that stops at the first
failure has run every other test before it.
"""
import ctypes
import math
import os

import numpy as np
import pytest

import vulture_b200 as vb
from vulture_b200 import _native as N
from helpers import stage_case

pytestmark = pytest.mark.gpu


def _fn():
    L = N.lib()
    f = L.vgpu_dft_accumulate_static
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_double,
                  ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p]
    return f


def test_static_dft_equals_engine_dft_over_two_calls():
    """Two calls in a row reproduce the engine's running DFT of the same
    observer point (hardsrc_ez: op1 and op2 sit on the same node)."""
    import torch

    mesh = stage_case("hardsrc_ez")
    old = os.getcwd()
    os.chdir(mesh.parent)
    try:
        m = vb.Mesh(mesh.name)
    finally:
        os.chdir(old)
    g = vb.GpuRun(m, "fp64").run()
    td = g.td()                    # [steps][num_td][6]
    re_e, im_e = g.dft()           # [num_fd][6][num_freq]
    g.close()
    nt, nf = m.num_steps, m.num_freq
    # Default frequencies of the reference (src/observer.c:433-441, 514-516).
    step_f = 1.0 / (nt * m.dt)
    omega = np.array([2.0 * math.pi * (0.0 + f * step_f) for f in range(nf)])

    dev = torch.device("cuda:0")
    samples = torch.tensor(np.ascontiguousarray(td[:, 0, :]), dtype=torch.float64, device=dev)
    om = torch.tensor(omega, dtype=torch.float64, device=dev)
    re = torch.zeros((6, nf), dtype=torch.float64, device=dev)
    im = torch.zeros((6, nf), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    f = _fn()
    half = nt // 2
    for first, rows in ((0, half), (half, nt - half)):
        ptr = samples.data_ptr() + first * 6 * 8
        rc = f(ptr, 6, rows, om.data_ptr(), nf, m.dt, first, re.data_ptr(), im.data_ptr())
        assert rc == 0, N.lib().vgpu_last_error().decode()
    torch.cuda.synchronize()
    peak = max(np.abs(re_e).max(), np.abs(im_e).max())
    assert np.abs(re.cpu().numpy() - re_e[0]).max() <= 1e-12 * peak
    assert np.abs(im.cpu().numpy() - im_e[0]).max() <= 1e-12 * peak


def test_static_dft_rejects_sizes_beyond_its_table():
    import torch

    dev = torch.device("cuda:0")
    buf = torch.zeros(8, dtype=torch.float64, device=dev)
    f = _fn()
    p = buf.data_ptr()
    assert f(p, 1, 300, p, 1, 1e-12, 0, p, p) == N.VGPU_EINVAL
    assert "maximum" in N.lib().vgpu_last_error().decode()
    assert f(p, 1, 256, p, 1000, 1e-12, 0, p, p) == N.VGPU_EINVAL
    assert "static twiddle table" in N.lib().vgpu_last_error().decode()
    # More series than the launch grid's 65535 block rows of 8 hold.
    assert f(p, 65535 * 8 + 1, 1, p, 1, 1e-12, 0, p, p) == N.VGPU_EINVAL
    assert "series" in N.lib().vgpu_last_error().decode()
