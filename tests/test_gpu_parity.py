"""GPU parity: the CUDA engine against the oracle on identical inputs.

FP64: every time-domain sample and every final field value equal the oracle's
bit for bit (the engine is built with --fmad=false and restates each update's
expression order); running DFTs agree to 1e-12 of their peak (the engine's
cos/sin are CUDA's, the oracle's glibc's).
FP32 storage: equal to the oracle's FP32 variant bit for bit, and within
1e-4 relative L2 of the FP64 oracle on every time-domain file.
"""
import os
import random

import numpy as np
import pytest

import vulture_b200 as vb
from vulture_b200 import meshgen
from vcpu import CpuRun
from helpers import case_names, max_rel, stage_case, stage_text

pytestmark = pytest.mark.gpu

SLOW = {"dgref_ref", "dgrefmb_ref", "sgref_mur", "sgref_pml6", "sgref_pml12"}


def solve_both(mesh_path, precision):
    old = os.getcwd()
    os.chdir(mesh_path.parent)
    try:
        m = vb.Mesh(mesh_path.name)
        g = vb.GpuRun(m, precision).run()
        c = CpuRun(m, precision).run()
        return m, g, c
    finally:
        os.chdir(old)


def shape_of(m):
    p = m.problem()
    import ctypes

    n = (ctypes.c_int32 * 3).from_address(p.value + 8)
    return tuple(n)


def assert_same(m, g, c, dft_tol=1e-12):
    assert np.array_equal(g.td(), c.td()), f"TD max diff {np.abs(g.td() - c.td()).max()}"
    shape = shape_of(m)
    for comp in range(6):
        a, b = g.field(comp, shape), c.field(comp, shape)
        assert np.array_equal(a, b), f"field {comp} max diff {np.abs(a - b).max()}"
    if m.num_fd:
        (gr, gi), (cr, ci) = g.dft(), c.dft()
        peak = max(np.abs(cr).max(), np.abs(ci).max(), 1e-300)
        assert np.abs(gr - cr).max() <= dft_tol * peak
        assert np.abs(gi - ci).max() <= dft_tol * peak


@pytest.mark.parametrize("case", [c for c in case_names() if c not in SLOW])
def test_fp64_engine_equals_oracle(case):
    m, g, c = solve_both(stage_case(case), "fp64")
    assert_same(m, g, c)


@pytest.mark.parametrize("case", [c for c in case_names() if c not in SLOW])
def test_fp32_engine_equals_fp32_oracle(case):
    m, g, c = solve_both(stage_case(case), "fp32")
    assert_same(m, g, c, dft_tol=1e-10)


def rel_l2(a, b):
    den = np.sqrt((b ** 2).sum())
    return float(np.sqrt(((a - b) ** 2).sum()) / den) if den > 0 else 0.0


@pytest.mark.parametrize("case", ["hardsrc_ez", "freespace_pml", "freespace_mur", "parplate1D_debyepml_xyz",
                                  "planewave_pec_xyz", "closedbox_spar", "dipole_vrz", "dgref_pml6"])
def test_fp32_within_1e4_of_fp64(case):
    mesh = stage_case(case)
    old = os.getcwd()
    os.chdir(mesh.parent)
    try:
        m = vb.Mesh(mesh.name)
        a = vb.GpuRun(m, "fp32").run().td()
        b = vb.GpuRun(m, "fp64").run().td()
    finally:
        os.chdir(old)
    for p in range(m.num_td):
        assert rel_l2(a[:, p, :], b[:, p, :]) <= 1e-4, f"observer {p}"


def many_media_mesh(nmedia=300, seed=5):
    """A mesh with more distinct coefficient tuples than the one-byte index
    holds, so the sweeps read the full coefficient volumes: single-cell
    blocks of seeded dielectrics and conductors inside a UPML box."""
    rng = random.Random(seed)
    out = ["VM 1.0.0", "CE many media", "DM 24 22 20", "GS",
           "BT XLO PML 4", "BT XHI PML 4", "BT YLO PML 4", "BT YHI PML 4", "BT ZLO PML 4", "BT ZHI PML 4"]
    for m in range(nmedia):
        out.append(f"MT m{m} SIMPLE {1.0 + 9.0 * rng.random():.6f} {0.05 * rng.random():.6f} 1.0")
    cells = set()
    while len(cells) < nmedia:
        cells.add((rng.randrange(3, 21), rng.randrange(3, 19), rng.randrange(3, 17)))
    for m, (i, j, k) in enumerate(sorted(cells)):
        out.append(f"MB {i} {i + 1} {j} {j + 1} {k} {k + 1} m{m}")
    out += ["WF wf1 GAUSSIAN_PULSE 1.0", "EX 12 12 11 11 10 11 src =EZ wf1 1.0",
            "OP 8 8 8 8 8 8 op1 TDOM_ASCII", "OP 15 15 14 14 12 12 op2 TDOM_ASCII", "GE", "NT 120", "MS 0.01", "EN"]
    return "\n".join(out) + "\n"


def debye_tfsf_cubic_mesh(nt=200):
    """A cubic grid (so the plane wave uses the 1-D auxiliary grid and every
    value is bit-exact) with a Debye block and a TFSF plane wave inside a
    UPML box, and observers off the Huygens faces: the engine merges the
    Debye update with the E corrections, and the H corrections with the next
    step's samples, into single launches (vgpu_stats.merged_parts = 3)."""
    return "\n".join([
        "VM 1.0.0", "CE Debye block and plane wave on a cubic grid", "DM 40 36 32", "GS",
        "BT XLO PML 6", "BT XHI PML 6", "BT YLO PML 6", "BT YHI PML 6", "BT ZLO PML 6", "BT ZHI PML 6",
        "MT deb DEBYE 2.0 0.0 1.0 1.000000e+10 -1.000000e+10", "MB 12 24 10 20 11 19 deb",
        "WF wf1 GAUSSIAN_PULSE 1.0",
        "PW 4 36 4 32 4 28 pw1 wf1 0.0 0.0 0.0 111111",
        "OP 20 20 18 18 15 15 op1 TDOM_ASCII", "OP 14 14 12 12 13 13 op2 TDOM_ASCII",
        "OP 25 25 22 22 17 17 op3 FDOM_ASCII", "OP 2 2 2 2 2 2 op4 TDOM_ASCII",
        "GE", f"NT {nt}", "MS 0.005", "EN"]) + "\n"


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_merged_side_launches_equal_oracle(precision):
    m, g, c = solve_both(stage_text(debye_tfsf_cubic_mesh()), precision)
    assert g.stats().merged_parts == 3
    assert np.abs(c.td()).max() > 0
    assert_same(m, g, c, dft_tol=1e-12 if precision == "fp64" else 1e-10)


def synthetic():
    rng = random.Random(11)
    return {
        "pec_cube_full": meshgen.pec_cube(),
        "graded_upml_short": meshgen.graded_upml(nt=130, dims=(200, 160, 120), plane=16, nfreq=20),
        "shielded_enclosure_small": meshgen.shielded_enclosure(nt=150, dims=(80, 64, 56), plane=8, nfreq=20),
        "batch_mesh": meshgen.batch_mesh(rng, 0, nmin=32, nmax=64, ntmin=200, ntmax=300),
        "serving_request": meshgen.serving_request(rng, 0, nmin=48, nmax=64, ntmin=200, ntmax=300),
        "many_media": many_media_mesh(),
    }


@pytest.mark.parametrize("name", list(synthetic()))
def test_synthetic_workloads_fp64_equal_oracle(name):
    m, g, c = solve_both(stage_text(synthetic()[name]), "fp64")
    # The analytic plane-wave incident field uses CUDA's exp/sin/cos on the
    # device and glibc's in the oracle: values agree to 1e-12 relative.
    if name in ("graded_upml_short", "shielded_enclosure_small") or ("PW " in synthetic()[name]):
        assert max_rel(g.td().reshape(-1, 6), c.td().reshape(-1, 6)) <= 1e-12
    else:
        assert_same(m, g, c)
