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
    small = vb.Mesh(stage_text(meshgen.config5_request(rng, 0, nmin=24, nmax=24, ntmin=100, ntmax=100), "a.mesh"))
    big = vb.Mesh(stage_text(meshgen.config5_request(rng, 1, nmin=48, nmax=48, ntmin=100, ntmax=100), "b.mesh"))
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
