"""Host-side parts of the serving layer (no GPU): footprint estimates and
latency summaries."""
import random

import pytest

import vulture_b200 as vb
from vulture_b200 import meshgen
from vulture_b200.serve import Request, footprint_estimate, latency_summary
from helpers import stage_text


def test_footprint_grows_with_cells_and_word_size():
    rng = random.Random(3)
    small = vb.Mesh(stage_text(meshgen.serving_request(rng, 0, nmin=24, nmax=24, ntmin=100, ntmax=100), "a.mesh"))
    big = vb.Mesh(stage_text(meshgen.serving_request(rng, 1, nmin=48, nmax=48, ntmin=100, ntmax=100), "b.mesh"))
    for m in (small, big):
        # At least the six field volumes and the engine's fixed blocks.
        assert footprint_estimate(m, "fp32") > m.num_cells * 6 * 4 + (64 << 20)
        assert footprint_estimate(m, "fp64") > footprint_estimate(m, "fp32")
    assert footprint_estimate(big, "fp32") > footprint_estimate(small, "fp32")


def test_latency_summary_percentiles_and_rate():
    reqs = []
    for q in range(100):
        r = Request("", arrival=0.01 * q)
        r.completed = r.arrival + 0.5 + 0.01 * q
        r.cell_updates = 10
        reqs.append(r)
    s = latency_summary(reqs)
    assert s["p50_s"] == pytest.approx(0.995, abs=1e-9)
    assert s["p99_s"] == pytest.approx(1.4801, abs=1e-9)
    assert s["solves_per_s"] == pytest.approx(100 / (reqs[-1].completed - reqs[0].arrival))
    assert s["cell_updates"] == 1000


class FakeRun:
    """Stands in for GpuRun on the host: each enqueue advances up to 64
    steps at once and the stream always reads as drained."""
    live = 0
    peak = 0

    def __init__(self, mesh, precision):
        self.mesh, self.precision, self.step = mesh, precision, 0
        FakeRun.live += 1
        FakeRun.peak = max(FakeRun.peak, FakeRun.live)

    def stats(self):
        class S:
            device_bytes = 1
        return S()

    def done(self):
        return True

    def enqueue(self, n=64):
        q = min(n, self.mesh.num_steps - self.step)
        self.step += q
        return q

    def synchronize(self):
        return self

    def td(self):
        return None

    def dft(self):
        return None

    def close(self):
        FakeRun.live -= 1


def test_server_admits_by_slots_and_budget(monkeypatch):
    import vulture_b200.serve as serve

    monkeypatch.setattr(serve, "GpuRun", FakeRun)
    FakeRun.live = FakeRun.peak = 0
    rng = random.Random(9)
    texts = [meshgen.serving_request(rng, q, nmin=24, nmax=32, ntmin=100, ntmax=300) for q in range(8)]
    est = max(footprint_estimate(vb.Mesh(stage_text(t, f"e{q}.mesh")), "fp32") for q, t in enumerate(texts))
    reqs = [Request(t, arrival=0.0, precision="fp32", tag=str(q)) for q, t in enumerate(texts)]
    srv = serve.Server(budget_bytes=int(2.5 * est), max_active=4)
    done = srv.run(reqs)
    assert [r.tag for r in done] == [str(q) for q in range(8)]
    assert all(r.completed >= r.admitted >= r.arrival for r in done)
    assert srv.peak_bytes <= srv.budget and srv.peak_active <= 2 and FakeRun.peak <= 2
    assert FakeRun.live == 0
    # First come, first served: admissions follow arrival order.
    assert [r.admitted for r in done] == sorted(r.admitted for r in done)
    srv = serve.Server(budget_bytes=10 ** 15, max_active=3)
    FakeRun.peak = 0
    srv.run([Request(t, arrival=0.0) for t in texts])
    assert FakeRun.peak <= 3 and srv.peak_active <= 3


def test_server_fails_a_bad_request_and_serves_the_rest(monkeypatch):
    import vulture_b200.serve as serve

    monkeypatch.setattr(serve, "GpuRun", FakeRun)
    FakeRun.live = FakeRun.peak = 0
    rng = random.Random(12)
    good = [meshgen.serving_request(rng, q, nmin=24, nmax=28, ntmin=100, ntmax=150) for q in range(3)]
    bad = "VM 1.0.0\nDM 8 8 8\nNOT A CARD\nEN\n"
    reqs = [Request(good[0], 0.0, tag="a"), Request(bad, 0.0, tag="bad"), Request(good[1], 0.0, tag="b"),
            Request(good[2], 0.0, tag="c")]
    done = serve.Server(budget_bytes=10 ** 15, max_active=2).run(reqs)
    errors = {r.tag: r.error for r in done}
    assert errors["bad"] is not None and all(errors[t] is None for t in "abc")
    assert FakeRun.live == 0
    s = latency_summary(done)
    assert s["failed"] == 1 and s["cell_updates"] > 0


def test_solve_batch_waves_fit_the_budget(monkeypatch):
    import vulture_b200.serve as serve

    monkeypatch.setattr(serve, "GpuRun", FakeRun)

    def fake_run_batch(runs):
        for r in runs:
            while r.enqueue(64):
                pass
    monkeypatch.setattr(serve, "run_batch", fake_run_batch)
    FakeRun.live = FakeRun.peak = 0
    rng = random.Random(13)
    meshes = [vb.Mesh(stage_text(meshgen.batch_mesh(rng, q, nmin=16, nmax=24, ntmin=50, ntmax=90), f"w{q}.mesh"))
              for q in range(7)]
    est = [footprint_estimate(m, "fp32") for m in meshes]
    seen = []
    out = serve.solve_batch(meshes, "fp32", budget_bytes=int(2.5 * max(est)),
                            on_done=lambda q, r: seen.append((q, r.step == meshes[q].num_steps)))
    assert out is None
    assert sorted(q for q, _ in seen) == list(range(7)) and all(ok for _, ok in seen)
    assert FakeRun.peak <= 2 and FakeRun.live == 0
    FakeRun.peak = 0
    runs = serve.solve_batch(meshes, "fp32")
    assert len(runs) == 7 and FakeRun.peak == 7
    for r in runs:
        r.close()


class FaultyRun(FakeRun):
    """A FakeRun whose stream reports a device error once it has stepped: the
    fault of a real engine surfaces from vgpu_query as VGPU_ECUDA."""

    def done(self):
        from vulture_b200 import _native as N

        if self.step > 0:
            raise N.NativeError(N.VGPU_ECUDA, "stream query: an illegal memory access was encountered")
        return True


def test_server_ends_a_solve_whose_stream_reports_a_device_error(monkeypatch):
    import vulture_b200.serve as serve

    created = []

    def make(mesh, precision):
        # The second request's engine fails on the device; the others run.
        r = (FaultyRun if len(created) == 1 else FakeRun)(mesh, precision)
        created.append(r)
        return r

    monkeypatch.setattr(serve, "GpuRun", make)
    FakeRun.live = FakeRun.peak = 0
    rng = random.Random(21)
    texts = [meshgen.serving_request(rng, q, nmin=24, nmax=28, ntmin=100, ntmax=150) for q in range(3)]
    reqs = [Request(t, 0.0, tag=str(q)) for q, t in enumerate(texts)]
    done = serve.Server(budget_bytes=10 ** 15, max_active=1).run(reqs)
    errors = {r.tag: r.error for r in done}
    assert errors["1"] is not None and "illegal memory access" in errors["1"]
    assert errors["0"] is None and errors["2"] is None
    assert all(r.completed is not None for r in done)
    assert FakeRun.live == 0


def test_solve_batch_closes_every_engine_when_the_batch_or_callback_fails(monkeypatch):
    import vulture_b200.serve as serve

    monkeypatch.setattr(serve, "GpuRun", FakeRun)
    rng = random.Random(22)
    meshes = [vb.Mesh(stage_text(meshgen.batch_mesh(rng, q, nmin=16, nmax=20, ntmin=50, ntmax=60), f"f{q}.mesh"))
              for q in range(4)]

    def failing_batch(runs):
        raise RuntimeError("device error while stepping")

    monkeypatch.setattr(serve, "run_batch", failing_batch)
    FakeRun.live = 0
    with pytest.raises(RuntimeError):
        serve.solve_batch(meshes, "fp32")
    assert FakeRun.live == 0
    with pytest.raises(RuntimeError):
        serve.solve_batch(meshes, "fp32", budget_bytes=10 ** 15)
    assert FakeRun.live == 0

    def fake_run_batch(runs):
        for r in runs:
            while r.enqueue(64):
                pass

    monkeypatch.setattr(serve, "run_batch", fake_run_batch)

    def bad_callback(q, r):
        if q == 1:
            raise ValueError("callback failed")

    with pytest.raises(ValueError):
        serve.solve_batch(meshes, "fp32", budget_bytes=10 ** 15, on_done=bad_callback)
    assert FakeRun.live == 0
