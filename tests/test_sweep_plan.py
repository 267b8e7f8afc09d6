"""The sweeps' tiling, checked on the host (no GPU): for every reference test
mesh and the synthetic workloads, each point of every swept component's bulk
and UPML update boxes is claimed by exactly one tile, no other point is, and
the tiles keep the sweep kernel's limits (vgpu_check_sweep_plan)."""
import ctypes as C
import os
import random

import pytest

import vulture_b200 as vb
from vulture_b200 import _native as N
from vulture_b200 import meshgen
from helpers import case_names, stage_case, stage_text


def check(mesh, precision):
    bad, ntiles = C.c_int64(-1), C.c_int64(0)
    prec = N.VGPU_FP64 if precision == "fp64" else N.VGPU_FP32
    N.check_gpu(N.lib().vgpu_check_sweep_plan(mesh.problem(precision), prec, C.byref(bad), C.byref(ntiles)))
    return bad.value, ntiles.value


@pytest.mark.parametrize("case", case_names())
def test_reference_meshes_are_tiled_exactly_once(case):
    path = stage_case(case)
    old = os.getcwd()
    os.chdir(path.parent)
    try:
        m = vb.Mesh(path.name)
        for precision in ("fp32", "fp64"):
            bad, ntiles = check(m, precision)
            assert ntiles > 0
            assert bad == 0, f"{case} {precision}: {bad} violations"
    finally:
        os.chdir(old)


def synthetic():
    rng = random.Random(11)
    return {
        "graded_upml_small": meshgen.graded_upml(nt=10, dims=(60, 44, 37), plane=8, nfreq=4, npml=8, ntd=4),
        "shielded_enclosure_small": meshgen.shielded_enclosure(nt=10, dims=(70, 52, 45), plane=8, nfreq=4),
        **{f"batch_mesh_{q}": meshgen.batch_mesh(rng, q, nmin=32, nmax=80, ntmin=10, ntmax=20) for q in range(4)},
        **{f"serving_request_{q}": meshgen.serving_request(rng, q, nmin=48, nmax=70, ntmin=10, ntmax=20) for q in range(4)},
    }


@pytest.mark.parametrize("name", sorted(synthetic()))
def test_synthetic_meshes_are_tiled_exactly_once(name):
    m = vb.Mesh(stage_text(synthetic()[name], f"{name}.mesh"))
    for precision in ("fp32", "fp64"):
        bad, ntiles = check(m, precision)
        assert ntiles > 0 and bad == 0, f"{name} {precision}: {bad} violations"


@pytest.mark.parametrize("depth", [1, 2, 3, 7, 16, 32])
def test_tuned_march_depths_tile_exactly_once(depth):
    """vgpu_set_sweep_tuning's march depth changes the tiles, never the
    points they claim."""
    names = ["graded_upml_small", "batch_mesh_0", "serving_request_1"]
    meshes = [vb.Mesh(stage_text(synthetic()[n], f"{n}.mesh")) for n in names]
    base = [check(m, "fp32")[1] for m in meshes]
    vb.set_sweep_tuning(depth, 0, 0)
    try:
        for name, m, nb in zip(names, meshes, base):
            for precision in ("fp32", "fp64"):
                bad, ntiles = check(m, precision)
                assert ntiles > 0 and bad == 0, f"{name} {precision} depth {depth}: {bad} violations"
            if depth == 1:
                assert check(m, "fp32")[1] > nb
    finally:
        vb.set_sweep_tuning(0, 0, 0)


def test_sweep_tuning_rejects_out_of_range_values():
    for args in [(-1, 0, 0), (33, 0, 0), (4, -1, 0), (4, 0, -1), (4, 0, 4097)]:
        with pytest.raises(N.NativeError):
            vb.set_sweep_tuning(*args)
