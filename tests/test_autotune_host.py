"""The autotuner's host logic (no GPU): size classes, the sample spread over
a batch's sizes, the cache key and the JSON cache round trip; and the
grouped entry point's argument checks, which run before any device use."""
import ctypes as C
import json

import pytest

from vulture_b200 import _native as N
from vulture_b200 import autotune


class FakeMesh:
    def __init__(self, cells):
        self.num_cells = cells
        self.num_steps = 100


def test_size_classes_are_powers_of_four_in_cells():
    assert autotune.size_class(4 ** 8) == autotune.size_class(4 ** 8 * 3) == 8
    assert autotune.size_class(4 ** 8 * 4) == 9
    assert autotune.size_class(32 ** 3) < autotune.size_class(160 ** 3)


def test_sample_spreads_over_sizes():
    meshes = [FakeMesh(c) for c in (50, 10, 40, 30, 20, 60, 70, 80, 90, 100)]
    s = autotune._sample(meshes, 4)
    cells = [m.num_cells for m in s]
    assert cells == sorted(cells) and cells[0] == 10 and cells[-1] == 100 and len(set(cells)) == 4
    assert len(autotune._sample(meshes[:3], 4)) == 3


def test_signature_depends_on_precision_and_mix():
    a = [FakeMesh(32 ** 3)] * 4
    b = [FakeMesh(32 ** 3)] * 2 + [FakeMesh(160 ** 3)] * 2
    assert autotune.signature(a, "fp32") != autotune.signature(a, "fp64")
    assert autotune.signature(a, "fp32") != autotune.signature(b, "fp32")
    assert autotune.signature(a, "fp32") == autotune.signature(a * 2, "fp32")


def test_cached_choice_is_returned_without_timing(tmp_path, monkeypatch):
    path = tmp_path / "tune.json"
    monkeypatch.setenv("VULTURE_B200_TUNE_CACHE", str(path))
    meshes = [FakeMesh(64 ** 3)] * 3
    key = autotune.signature(meshes, "fp32")
    path.write_text(json.dumps({key: {"depth": 16, "blocks_per_sm": 2, "chunk": 8, "trials": []}}))

    def no_timing(*a, **k):
        raise AssertionError("timed although cached")

    monkeypatch.setattr(autotune, "time_setting", no_timing)
    (depth, blocks, chunk), rec = autotune.tune(meshes, "fp32")
    assert (depth, blocks, chunk) == (16, 2, 8) and rec["cached"]


def test_tune_picks_the_fastest_trial_and_caches_it(tmp_path, monkeypatch):
    path = tmp_path / "tune.json"
    monkeypatch.setenv("VULTURE_B200_TUNE_CACHE", str(path))
    speed = {(0, 0, 4): 1.0, (8, 0, 16): 3.0, (16, 0, 4): 2.0, (32, 0, 2): 0.5, (16, 2, 4): 2.5}

    def fake(sample, precision, depth, blocks, chunk, steps):
        return {"depth": depth, "blocks_per_sm": blocks, "chunk": chunk, "group_ms": 1.0,
                "mcell_per_s": speed.get((depth, blocks, chunk), 0), "tiles": 1}

    monkeypatch.setattr(autotune, "time_setting", fake)
    meshes = [FakeMesh(c) for c in (40 ** 3, 90 ** 3, 150 ** 3)]
    (depth, blocks, chunk), rec = autotune.tune(meshes, "fp32")
    assert (depth, blocks, chunk) == (8, 0, 16) and not rec["cached"]
    assert json.loads(path.read_text())[rec["key"]]["depth"] == 8


def test_grouped_entry_checks_arguments_before_the_device():
    L = N.lib()
    rep = N.VgpuGroupReport()
    assert L.vgpu_run_grouped(None, 0, None, C.byref(rep)) == 0
    assert rep.launches == 0 and rep.grouped == 0
    assert L.vgpu_run_grouped(None, 2, None, None) == N.VGPU_EINVAL
    arr = (C.c_void_p * 1)(None)
    st = (C.c_uint64 * 1)(1)
    assert L.vgpu_run_grouped(arr, 1, st, None) == N.VGPU_EINVAL
    assert L.vgpu_groupable(None) == N.VGPU_EINVAL
