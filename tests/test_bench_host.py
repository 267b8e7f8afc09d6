"""Host logic of bench.py (no GPU): the FP32 error report and the shared
workload description of both arms."""
import gzip
import json

import numpy as np

import bench


def test_both_arms_describe_the_same_workload():
    # 216 x 176 x 136 outer cells: 200 x 160 x 120 plus 8 UPML cells per side.
    assert bench.N_OUT == 216 * 176 * 136 == 5170176
    assert bench.CONFIG["n_out_cells"] == bench.N_OUT
    assert bench.CONFIG["precision"] == "fp32"


def test_error_report_per_result_and_against_the_reference(tmp_path, monkeypatch):
    rng = np.random.default_rng(3)
    steps, npts, nfd, nf = 50, 4, 3, 16
    td64 = rng.normal(size=(steps, npts, 6))
    td64[:, 3, :] = 1e-40            # a point the pulse has not reached
    td = td64 * (1 + 1e-6)
    re64 = rng.uniform(0.5, 1.0, size=(nfd, 6, nf))
    im64 = np.zeros_like(re64)
    # Result (q, c) scaled by 10^(e/20): a known dB error e on every frequency.
    err_db = np.full((nfd, 6), 1e-5)
    err_db[1, 2] = 5e-3
    err_db[2, 4] = 0.05
    re = re64 * 10 ** (err_db[:, :, None] / 20)
    im = im64.copy()
    names = [f"p{q}" for q in range(nfd)]
    ref = {"mesh": {"nt": steps}, "td": {"a": {"rel_l2": 1e-3, "norm": 1.0}},
           "fd_db": {n: [1e-2] * 6 for n in names}}
    fix = tmp_path / "ref.json.gz"
    with gzip.open(fix, "wt") as fh:
        json.dump(ref, fh)
    monkeypatch.setattr(bench, "FP32_REFERENCE_ERROR", fix)
    rep = bench.error_report(td, re, im, td64, re64, im64, steps, names)
    assert rep["td_points"] == 3 and rep["td_points_below_1e-3_of_peak"] == 1
    assert abs(rep["td_rel_l2_max"] - 1e-6) < 1e-9
    assert rep["fd_results"] == nfd * 6
    assert abs(rep["fd_db_max"] - 0.05) < 1e-9
    assert sum(rep["fd_db_histogram"].values()) == nfd * 6
    assert rep["fd_share_within_1e-3_db"] == (nfd * 6 - 2) / (nfd * 6)
    v = rep["vs_reference_fp32"]
    assert v["results_compared"] == nfd * 6
    # Every result but the 0.05 dB one is at or below the reference's 1e-2 dB.
    assert v["share_engine_le_reference"] == (nfd * 6 - 1) / (nfd * 6)
    assert v["reference_td_rel_l2_max"] == 1e-3


def test_error_report_without_a_matching_reference_run(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "FP32_REFERENCE_ERROR", tmp_path / "missing.json.gz")
    td = np.ones((4, 1, 6))
    re = np.ones((1, 6, 3))
    rep = bench.error_report(td, re, re * 0, td, re, re * 0, 4, ["p0"])
    assert "vs_reference_fp32" not in rep and rep["fd_db_max"] == 0.0


def test_traffic_records_scale_by_cells(tmp_path, monkeypatch):
    # A record captured on a smaller case scales with the cells a launch
    # updates; a plain number is already per launch at full size.
    prof = tmp_path / "profiles"
    prof.mkdir()
    (prof / "traffic.json").write_text(json.dumps({"k<E,bulk>:fp32": {"bytes": 200, "cells": 10},
                                                   "k<E,UPML>:fp32": 1234}))
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.scaled_traffic("k<E,bulk>", "fp32", 25.0) == 500.0
    assert bench.scaled_traffic("k<E,UPML>", "fp32", 99.0) == 1234
    assert bench.scaled_traffic("k<H,bulk>", "fp32", 1.0) is None
