"""Failure paths of the engine on the GPU, made on the host or by a bounded
wait that is told to give up -- nothing here faults, traps or hangs a GPU.

- A non-finite field value, planted with vgpu_write_field, fails the run
  through the FP64 stability check and fails vgpu_check_finite.
- The stability check's FP64 sums of squares equal the fields read back.
- A sweep whose compute warps give up waiting for a stage's data (the wait
  limit lowered to zero polls through vgpu_set_sweep_wait_limit) makes
  vgpu_run return VGPU_ETIMEOUT; the producer warp keeps its full bound and
  waits for every load it issued, so the context stays usable: later runs of
  the same engine report the timeout again without stepping, and a new engine
  on the device runs normally.
"""
import ctypes
import os
import time

import numpy as np
import pytest

import vulture_b200 as vb
from vulture_b200 import _native as N
from vcpu import CpuRun
from helpers import stage_case

pytestmark = pytest.mark.gpu


def mesh_of(case):
    path = stage_case(case)
    old = os.getcwd()
    os.chdir(path.parent)
    try:
        return vb.Mesh(path.name)
    finally:
        os.chdir(old)


def shape_of(m):
    return tuple((ctypes.c_int32 * 3).from_address(m.problem().value + 8))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_planted_nan_fails_the_run_and_the_finiteness_check(precision):
    m = mesh_of("freespace_pml")
    shape = shape_of(m)
    g = vb.GpuRun(m, precision)
    g.run(10)
    ez = g.field(2, shape)
    ez[shape[0] // 2, shape[1] // 2, shape[2] // 2] = np.nan
    g.write_field(2, ez)
    with pytest.raises(N.NativeError) as err:
        g.run(64 - 10)
    assert err.value.code == N.VGPU_ENONFINITE
    with pytest.raises(N.NativeError) as err:
        g.check_finite()
    assert err.value.code == N.VGPU_ENONFINITE
    g.close()


def test_stability_check_equals_the_fields_sums_of_squares():
    m = mesh_of("hardsrc_ez")
    shape = shape_of(m)
    g = vb.GpuRun(m, "fp64").run(128)
    st = g.stats()
    assert st.energy_step == 128
    e = sum(float((g.field(c, shape) ** 2).sum()) for c in range(3))
    h = sum(float((g.field(c, shape) ** 2).sum()) for c in range(3, 6))
    assert e > 0 and h > 0
    assert abs(st.energy_e - e) <= 1e-12 * e and abs(st.energy_h - h) <= 1e-12 * h
    # The oracle's fields give the same sums: the engine's fields are its own.
    c = CpuRun(m, "fp64").run(128)
    e_cpu = sum(float((c.field(q, shape) ** 2).sum()) for q in range(3))
    assert abs(st.energy_e - e_cpu) <= 1e-12 * e_cpu
    g.close()


def test_sweep_wait_that_runs_out_is_reported_and_the_device_stays_usable():
    m = mesh_of("freespace_pml")
    g = vb.GpuRun(m, "fp32")
    N.check_gpu(N.lib().vgpu_set_sweep_wait_limit(0))
    try:
        with pytest.raises(N.NativeError) as err:
            g.run(16)
        assert err.value.code == N.VGPU_ETIMEOUT
    finally:
        N.check_gpu(N.lib().vgpu_set_sweep_wait_limit(-1))
    # The engine's run is lost: its later sweeps skip their work at once.
    t0 = time.perf_counter()
    with pytest.raises(N.NativeError) as err:
        g.run(16)
    assert err.value.code == N.VGPU_ETIMEOUT
    assert time.perf_counter() - t0 < 0.5
    g.close()
    # A new engine on the same device, with the default bound, runs and
    # equals the oracle.
    m2 = mesh_of("hardsrc_ez")
    g2 = vb.GpuRun(m2, "fp64").run()
    c2 = CpuRun(m2, "fp64").run()
    assert np.array_equal(g2.td(), c2.td())
    g2.close()
