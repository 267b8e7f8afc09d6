"""Grouped stepping: many meshes share one sweep launch per half step.

vgpu_run_grouped steps the groupable engines of a batch as one group -- a
tile list that spans every member mesh, one side launch for all members'
samples and sources, graphs of whole group steps -- and the other engines
beside it, as vgpu_run_batch would.  Members leave as their steps run out
and the group's launches shorten to the rest.  Each engine's time-domain samples,
running DFTs and final fields must equal its solo run's bit for bit, at
either precision, whatever the membership changes and the tile tuning
(march depth down to one plane per tile, block caps, chunks of one tile
to all of them).
"""
import os
import random
import time

import pytest

import vulture_b200 as vb
from vulture_b200 import _native as N
from vulture_b200 import meshgen
from vulture_b200.serve import solve_batch
from helpers import stage_text
from test_batch_serve import assert_same_run

pytestmark = pytest.mark.gpu


def with_fd_points(text, pts, nfreq):
    """A mesh text with frequency-domain point observers and their OF card."""
    lines = text.splitlines()
    ge = lines.index("GE")
    lines[ge:ge] = [f"OP {i} {i} {j} {j} {k} {k} fd{q} FDOM_ASCII" for q, (i, j, k) in enumerate(pts)]
    nt = next(q for q, line in enumerate(lines) if line.startswith("NT "))
    lines.insert(nt + 1, f"OF 1.0e8 1.0e10 {nfreq}")
    return "\n".join(lines) + "\n"


def free_space_mesh(n=(24, 20, 36), nt=140):
    """No UPML, Mur or ghost faces: the bulk sweep kernel's class."""
    out = ["VM 1.0.0", "CE free-space faces", "DM {} {} {}".format(*n), "GS"]
    out += [f"BT {f} FREE_SPACE" for f in ("XLO", "XHI", "YLO", "YHI", "ZLO", "ZHI")]
    out += ["MT diel SIMPLE 3.0 0.0 1.0", f"MB 2 {n[0] - 2} 3 9 4 {n[2] - 4} diel", "WF wf1 GAUSSIAN_PULSE 1.0",
            f"EX 8 8 7 7 10 11 src =EZ wf1 1.0", "OP 12 12 10 10 18 18 op1 TDOM_ASCII",
            "GE", f"NT {nt}", "MS 0.01", "EN"]
    return "\n".join(out) + "\n"


def group_paths():
    rng = random.Random(43)
    texts = [meshgen.batch_mesh(rng, q, nmin=20, nmax=48, ntmin=100, ntmax=300) for q in range(6)]
    texts[1] = with_fd_points(texts[1], [(7, 8, 9), (10, 9, 8), (9, 9, 9)], 9)
    texts.append(free_space_mesh())
    # A plane wave: not groupable, stepped beside the group.
    texts.append(meshgen.graded_upml(nt=90, dims=(40, 32, 24), plane=4, nfreq=6, npml=4, ntd=2))
    return [stage_text(t, f"g{q}.mesh") for q, t in enumerate(texts)]


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_grouped_equals_solo(precision):
    meshes = [vb.Mesh(p) for p in group_paths()]
    solo = [vb.GpuRun(m, precision).run() for m in meshes]
    runs = [vb.GpuRun(m, precision) for m in meshes]
    assert [r.groupable for r in runs] == [True] * 7 + [False]
    runs[2].run(17)                  # off a 64-step boundary: stepped beside the group
    rep = vb.run_grouped(runs)
    assert rep["grouped"] == 6
    # Members with different step counts leave at different steps.
    assert rep["rebuilds"] >= 3
    assert rep["tiles"] > 0 and rep["group_ms"] > 0
    for m, a, b in zip(meshes, runs, solo):
        assert a.step == m.num_steps
        assert_same_run(m, a, b)


@pytest.mark.parametrize("precision,depth,blocks,chunk", [
    ("fp32", 1, 1, 1), ("fp32", 2, 0, 3), ("fp32", 3, 2, 64), ("fp32", 32, 0, 1), ("fp32", 0, 0, 4096),
    ("fp64", 1, 0, 4), ("fp64", 2, 0, 4)])
def test_grouped_tuning_keeps_results(precision, depth, blocks, chunk):
    # One-plane tiles change mesh almost every tile: a buffer of mesh values
    # rewritten before every warp has stored its last plane would show here.
    meshes = [vb.Mesh(p) for p in group_paths()[:7]]
    solo = [vb.GpuRun(m, precision).run() for m in meshes]
    vb.set_sweep_tuning(depth, blocks, chunk)
    try:
        runs = [vb.GpuRun(m, precision) for m in meshes]
        rep = vb.run_grouped(runs)
    finally:
        vb.set_sweep_tuning(0, 0, 0)
    assert rep["grouped"] == 7
    for m, a, b in zip(meshes, runs, solo):
        assert_same_run(m, a, b)


def test_grouped_partial_steps_then_rest():
    meshes = [vb.Mesh(p) for p in group_paths()[:4]]
    solo = [vb.GpuRun(m, "fp64").run() for m in meshes]
    runs = [vb.GpuRun(m, "fp64") for m in meshes]
    vb.run_grouped(runs, [64, 128, 64, 64])
    assert [r.step for r in runs] == [64, 128, 64, 64]
    vb.run_grouped(runs)
    for m, a, b in zip(meshes, runs, solo):
        assert_same_run(m, a, b)


def test_grouped_rejects_overrun_and_duplicates():
    m = vb.Mesh(group_paths()[0])
    a, b = vb.GpuRun(m, "fp32"), vb.GpuRun(m, "fp32")
    with pytest.raises(N.NativeError):
        vb.run_grouped([a, b], [m.num_steps + 1, 1])
    with pytest.raises(N.NativeError):
        vb.run_grouped([a, a], [1, 1])
    assert a.step == 0 and b.step == 0


def test_grouped_wait_that_runs_out_fails_every_member():
    meshes = [vb.Mesh(p) for p in group_paths()[:3]]
    runs = [vb.GpuRun(m, "fp32") for m in meshes]
    N.check_gpu(N.lib().vgpu_set_sweep_wait_limit(0))
    try:
        with pytest.raises(N.NativeError) as err:
            vb.run_grouped(runs, [32, 32, 32])
        assert err.value.code == N.VGPU_ETIMEOUT
    finally:
        N.check_gpu(N.lib().vgpu_set_sweep_wait_limit(-1))
    # Every member's run is lost: a later run of each reports the timeout
    # at once without stepping.
    for r in runs:
        t0 = time.perf_counter()
        with pytest.raises(N.NativeError) as err:
            r.run(16)
        assert err.value.code == N.VGPU_ETIMEOUT
        assert time.perf_counter() - t0 < 0.5
        r.close()
    # A new group on the device runs and equals solo runs.
    fresh = [vb.GpuRun(m, "fp32") for m in meshes]
    vb.run_grouped(fresh)
    for m, r in zip(meshes, fresh):
        assert_same_run(m, r, vb.GpuRun(m, "fp32").run())


def test_solve_batch_autotuned_equals_solo(tmp_path):
    os.environ["VULTURE_B200_TUNE_CACHE"] = str(tmp_path / "tune.json")
    try:
        meshes = [vb.Mesh(p) for p in group_paths()]
        solo = [vb.GpuRun(m, "fp32").run() for m in meshes]
        runs = solve_batch(meshes, "fp32", grouped=True, tuning="auto")
        rec = runs[0].batch_tuning
        assert rec is not None and not rec["cached"] and len(rec["trials"]) >= 4
        assert runs[0].batch_report["grouped"] == 7
        for m, a, b in zip(meshes, runs, solo):
            assert_same_run(m, a, b)
        # The second batch of the same kind takes the cached choice.
        again = solve_batch(meshes[:7] + meshes[7:], "fp32", grouped=True, tuning="auto")
        assert again[0].batch_tuning["cached"]
    finally:
        os.environ.pop("VULTURE_B200_TUNE_CACHE", None)


def test_solve_batch_grouped_equals_solo():
    meshes = [vb.Mesh(p) for p in group_paths()[:5]]
    solo = [vb.GpuRun(m, "fp32").run() for m in meshes]
    runs = solve_batch(meshes, "fp32", grouped=True)
    assert runs[0].batch_report["grouped"] == 5 and runs[0].batch_tuning is None
    for m, a, b in zip(meshes, runs, solo):
        assert_same_run(m, a, b)
