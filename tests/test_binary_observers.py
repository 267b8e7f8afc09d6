"""TDOM_BINARY observers: impulse.dat, excite.dat and process.dat
(src/observer.c:1016-1212), and the mesh-line files of the set-up
(src/grid.c:942-944).

CPU tests: the oracle's float rows written through the host writer equal the
files the reference's FP64 build writes on the same mesh, byte for byte --
except impulse.dat bytes 4-7, where the FP64 reference writes four bytes of
its double dt (sizeof(float) of a `real`, src/observer.c:1147); those hold
(float)dt here, as in the shipped real=float build.
GPU tests: the engine's streamed rows equal the oracle's rows bit for bit,
and the CLI writes the same files.
"""
import os
import shutil
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

import vulture_b200 as vb
from vulture_b200._native import NativeError
from vcpu import CpuRun
from helpers import ROOT, have_reference_binaries, run_reference, stage_case, stage_text

# A small box with a graded PML side, a hard source and two binary observers:
# a strided plane and a single node, inside a restricted output window.
PLANE_MESH = """VM 1.0.0
CE Binary observers: a strided plane and a node in an OT window, with a comment longer than the process.dat limit
DM 24 20 18
GS
BT XLO PML 4
BT YHI PML 4
WF wf1 GAUSSIAN_PULSE 1.0
EX 12 12 10 10 9 10 source =EZ wf1 -4439809.322 0.0
OP 2 22 3 17 9 9 bplane TDOM_BINARY 3 2 1
OP 12 12 10 10 9 9 bnode TDOM_BINARY 1 1 1
OP 12 12 10 10 9 9 op1 TDOM_ASCII
GE
NT 150
OT 20 129
MS 0.01
EN
"""


def _oracle_files(mesh_path: Path, out: Path, precision="fp64"):
    old = os.getcwd()
    os.chdir(mesh_path.parent)
    try:
        m = vb.Mesh(mesh_path.name)
    finally:
        os.chdir(old)
    c = CpuRun(m, precision).run()
    rows = c.bin()
    m.write_lines(out)
    m.write_binary(out, rows)
    return m, rows


def _compare_to_reference(mesh_path: Path, tmp_path: Path):
    m, rows = _oracle_files(mesh_path, tmp_path)
    ref = run_reference(mesh_path, binary="vulture_oracle_f64")
    mine = (tmp_path / "impulse.dat").read_bytes()
    theirs = (ref / "impulse.dat").read_bytes()
    assert len(mine) == len(theirs)
    assert mine[:4] == theirs[:4]
    assert struct.unpack("<f", mine[4:8])[0] == np.float32(m.dt)
    assert mine[8:] == theirs[8:]
    for f in ("excite.dat", "process.dat", "xlines.dat", "ylines.dat", "zlines.dat"):
        assert (tmp_path / f).read_text() == (ref / f).read_text(), f
    return m, rows


needs_ref = pytest.mark.skipif(not have_reference_binaries(), reason="reference builds under oracle/_ref absent")


# Reference test meshes with a binary observer, less the long-running ones.
SLOW = {"dgref_ref", "dgrefmb_ref", "sgref_mur", "sgref_pml6", "sgref_pml12", "dgref_mur", "dgref_pml6",
        "dgref_pml12", "dgrefmb_pml6"}
BINARY_CASES = sorted(p.parent.name for p in (ROOT / "tests" / "golden" / "cases").glob("*/*.mesh")
                      if "TDOM_BINARY" in p.read_text() and p.parent.name not in SLOW)
# One of each family for the GPU runs.
GPU_CASES = ["closedbox_spar", "freespace_mur", "freespace_pml", "parplate1D_debyepml_xyz", "parplate1D_planewave_zxy",
             "parplate1D_sibcgo04_yxz", "planewave_pec_yzx", "waveform_ext"]


@needs_ref
@pytest.mark.parametrize("case", BINARY_CASES)
def test_reference_case_binary_files_match(case, tmp_path):
    """Every reference test mesh with a binary observer."""
    m, rows = _compare_to_reference(stage_case(case), tmp_path)
    assert rows.shape == (m.num_output_steps, m.num_bin, 6)


@needs_ref
def test_strided_plane_binary_files_match(tmp_path):
    m, rows = _compare_to_reference(stage_text(PLANE_MESH), tmp_path)
    # 1 + 20//3 = 7 in x, 1 + 14//2 = 8 in y, one k plane; plus the node.
    assert m.num_bin == 7 * 8 + 1
    assert rows.shape == (110, 57, 6)
    assert np.abs(rows).max() > 0


def test_node_order_is_k_then_j_then_i(tmp_path):
    mp = stage_text(PLANE_MESH)
    m, rows = _oracle_files(mp, tmp_path)
    b = (tmp_path / "impulse.dat").read_bytes()
    rec = np.frombuffer(b[8:], dtype=np.dtype([("ijk", "<i4", 3), ("f", "<f4", 6)]))
    assert rec.size == 110 * 57
    ijk = rec["ijk"][:57]
    assert [tuple(v) for v in ijk[:3]] == [(2, 3, 9), (5, 3, 9), (8, 3, 9)]
    assert tuple(ijk[7]) == (2, 5, 9)
    assert tuple(ijk[56]) == (12, 10, 9)
    assert np.array_equal(rec["f"].reshape(110, 57, 6), rows)


def test_zero_step_is_refused(tmp_path):
    bad = PLANE_MESH.replace("bplane TDOM_BINARY 3 2 1", "bplane TDOM_BINARY 3 0 1")
    mp = stage_text(bad)
    old = os.getcwd()
    os.chdir(mp.parent)
    try:
        with pytest.raises(NativeError, match="zero step"):
            vb.Mesh(mp.name)
    finally:
        os.chdir(old)


def test_no_binary_observers_writes_no_binary_files(tmp_path):
    mp = stage_case("hardsrc_ez")
    old = os.getcwd()
    os.chdir(mp.parent)
    try:
        m = vb.Mesh(mp.name)
    finally:
        os.chdir(old)
    assert m.num_bin == 0
    m.bin_begin(tmp_path)
    m.bin_end()
    assert not (tmp_path / "impulse.dat").exists() and not (tmp_path / "process.dat").exists()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("case", ["plane"] + GPU_CASES)
def test_engine_rows_equal_oracle_rows(case, precision):
    mp = stage_text(PLANE_MESH) if case == "plane" else stage_case(case)
    old = os.getcwd()
    os.chdir(mp.parent)
    try:
        m = vb.Mesh(mp.name)
    finally:
        os.chdir(old)
    g = vb.GpuRun(m, precision).collect_bin()
    # Uneven runs: a partial first block, then the rest.
    g.run(37)
    g.run()
    a = g.bin()
    b = CpuRun(m, precision).run().bin()
    assert a.shape == b.shape
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    firsts = g.bin_first_rows()
    assert firsts == sorted(firsts) and firsts[0] == 0


@pytest.mark.gpu
def test_cli_writes_reference_binary_files(tmp_path):
    mp = stage_text(PLANE_MESH)
    exe = ROOT / "vulture_b200" / "bin" / "vulture-b200"
    r = subprocess.run([str(exe), mp.name], cwd=mp.parent, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    _oracle_files(mp, tmp_path)
    for f in ("impulse.dat", "excite.dat", "process.dat", "xlines.dat", "ylines.dat", "zlines.dat"):
        assert (mp.parent / f).read_bytes() == (tmp_path / f).read_bytes(), f
