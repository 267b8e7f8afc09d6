"""Batched and served solves: each result equals the same solve run alone.

The batch entry point (vgpu_run_batch) and the serving loop interleave
64-step blocks of several engines on one device; every engine keeps its own
stream and buffers, so its time-domain samples, running DFTs and final
fields must equal a solo run's bit for bit, at either precision.
"""
import random

import numpy as np
import pytest

import vulture_b200 as vb
from vulture_b200 import meshgen
from vulture_b200.serve import Request, Server, footprint_estimate, latency_summary, solve_batch
from helpers import stage_text

pytestmark = pytest.mark.gpu


def small_meshes():
    rng = random.Random(41)
    texts = [meshgen.batch_mesh(rng, q, nmin=20, nmax=40, ntmin=150, ntmax=260) for q in range(4)]
    texts.append(meshgen.graded_upml(nt=90, dims=(40, 32, 24), plane=8, nfreq=12, npml=4, ntd=4))
    return [stage_text(t, f"b{q}.mesh") for q, t in enumerate(texts)]


def shape_of(m):
    import ctypes

    p = m.problem()
    return tuple((ctypes.c_int32 * 3).from_address(p.value + 8))


def assert_same_run(m, a, b):
    assert np.array_equal(a.td(), b.td())
    if m.num_fd:
        (ar, ai), (br, bi) = a.dft(), b.dft()
        assert np.array_equal(ar, br) and np.array_equal(ai, bi)
    shape = shape_of(m)
    for comp in range(6):
        assert np.array_equal(a.field(comp, shape), b.field(comp, shape)), f"field {comp}"


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_batch_equals_solo(precision):
    paths = small_meshes()
    meshes = [vb.Mesh(p) for p in paths]
    solo = [vb.GpuRun(m, precision).run() for m in meshes]
    runs = [vb.GpuRun(m, precision) for m in meshes]
    runs[1].run(17)          # one engine starts mid-block
    vb.run_batch(runs)
    for m, a, b in zip(meshes, runs, solo):
        assert a.step == m.num_steps
        assert_same_run(m, a, b)


def test_solve_batch_equals_solo():
    meshes = [vb.Mesh(p) for p in small_meshes()]
    solo = [vb.GpuRun(m, "fp32").run() for m in meshes]
    runs = solve_batch(meshes, "fp32")
    for m, a, b in zip(meshes, runs, solo):
        assert a.step == m.num_steps
        assert_same_run(m, a, b)


def test_enqueue_steps_to_the_end():
    p = small_meshes()[4]
    m = vb.Mesh(p)
    solo = vb.GpuRun(m, "fp32").run()
    r = vb.GpuRun(m, "fp32")
    queued = []
    while True:
        q = r.enqueue(64)
        if not q:
            break
        queued.append(q)
    r.synchronize()
    assert r.done()
    assert sum(queued) == m.num_steps and all(q <= 64 for q in queued)
    assert_same_run(m, r, solo)
    # Past the end: a batch that asks for more steps is refused.
    with pytest.raises(vb._native.NativeError):
        vb.run_batch([r], [1])


def test_batch_rejects_overrun_of_a_listed_twice_engine():
    p = small_meshes()[0]
    m = vb.Mesh(p)
    r = vb.GpuRun(m, "fp32")
    n = m.num_steps
    with pytest.raises(vb._native.NativeError):
        vb.run_batch([r, r], [n - 10, n - 10])
    r.synchronize()


def test_served_results_equal_solo_and_budget_queues():
    rng = random.Random(5)
    texts = [meshgen.serving_request(rng, q, nmin=24, nmax=40, ntmin=120, ntmax=200) for q in range(6)]
    meshes = [vb.Mesh(stage_text(t, f"s{q}.mesh")) for q, t in enumerate(texts)]
    ests = [footprint_estimate(m, "fp32") for m in meshes]
    reqs = [Request(t, arrival=0.002 * q, precision="fp32", tag=str(q)) for q, t in enumerate(texts)]
    srv = Server(budget_bytes=2 * max(ests))
    done = srv.run(reqs)
    assert srv.peak_bytes <= srv.budget
    assert srv.peak_active <= 2 and srv.peak_active >= 1
    for r, m in zip(done, meshes):
        assert r.completed is not None and r.completed >= r.admitted >= r.arrival
        assert r.device_bytes <= r.estimate
        solo = vb.GpuRun(m, "fp32").run()
        assert np.array_equal(r.td, solo.td())
        (ar, ai), (br, bi) = r.dft, solo.dft()
        assert np.array_equal(ar, br) and np.array_equal(ai, bi)
    s = latency_summary(done)
    assert s["p99_s"] >= s["p50_s"] > 0
