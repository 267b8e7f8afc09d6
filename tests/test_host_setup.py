"""Host side: mesh parsing and set-up, restating src/mesh.c and the init*
functions.  Values are checked against the reference's own formulas."""
import math

import numpy as np
import pytest

import vulture_b200 as vb
from vulture_b200 import meshgen
from vulture_b200._native import NativeError
from helpers import GOLDEN, case_names, stage_case, stage_text


@pytest.mark.parametrize("case", case_names())
def test_every_reference_mesh_sets_up(case):
    m = vb.Mesh(stage_case(case))
    assert m.num_steps > 0 and m.dt > 0 and m.num_cells > 0


@pytest.mark.parametrize("name", ["eof", "no_vm"])
def test_reference_parser_negative_cases_fail(name):
    """The reference's tests/parser cases are expected to fail (WILL_FAIL)."""
    with pytest.raises(NativeError):
        vb.Mesh(GOLDEN / "parser" / f"{name}.mesh")


def test_time_step_formula():
    """dt = CN / c0 / sqrt(sum 1/dmin^2) over primary and secondary edges (src/grid.c:673-675)."""
    n = 16
    m = vb.Mesh(stage_text(meshgen.pec_cube(nt=10, n=n)))
    c0 = 299792458.0
    lines = [i * 0.01 for i in range(n + 1)]
    de = [lines[i + 1] - lines[i] for i in range(n)]
    dh = [0.5 * (de[i] + de[i - 1]) for i in range(1, n)]
    d = min(de + dh)
    assert m.dt == 0.99 / c0 / math.sqrt((1.0 / d) * (1.0 / d) + (1.0 / d) * (1.0 / d) + (1.0 / d) * (1.0 / d))


def test_outer_cell_count_includes_pml():
    m = vb.Mesh(stage_text(meshgen.graded_upml(nt=10, dims=(20, 16, 12), plane=2, nfreq=4, ntd=1)))
    assert m.num_cells == (20 + 16) * (16 + 16) * (12 + 16)


@pytest.mark.parametrize("bad,needle", [
    ("DM 0 4 4", "DM"),
    ("NT x", "NT"),
    ("EX 1 1 1 1 1 2 s =EQ wf1 1.0", "EX"),
    ("OP 1 2 1 1 1 1 o1 TDOM_ASCII", "OP"),
    ("MT m SIMPLE 0.5", "MT"),
    ("CN 1.5", "CN"),
])
def test_invalid_cards_are_rejected(bad, needle):
    base = ["VM 1.0.0", "CE t", "DM 4 4 4", "GS", "WF wf1 GAUSSIAN_PULSE", "EX 1 1 1 1 1 2 s =EZ wf1 1.0",
            "OP 2 2 2 2 2 2 o TDOM_ASCII", "GE", "NT 5", "MS 0.01", "EN"]
    key = bad.split()[0]
    idx = next(i for i, l in enumerate(base) if l.startswith(key)) if any(l.startswith(key) for l in base) else None
    lines = list(base)
    if idx is None:
        lines.insert(lines.index("GE") if key in ("MT", "OP", "EX", "WF", "PW", "MB", "TB") else lines.index("EN"), bad)
    else:
        lines[idx] = bad
    with pytest.raises(NativeError) as e:
        vb.Mesh(stage_text("\n".join(lines) + "\n"))
    assert needle in str(e.value)


def test_missing_source_is_an_error():
    text = "VM 1.0.0\nDM 4 4 4\nGS\nWF wf1 GAUSSIAN_PULSE\nOP 2 2 2 2 2 2 o TDOM_ASCII\nGE\nNT 5\nMS 0.01\nEN\n"
    with pytest.raises(NativeError, match="No source"):
        vb.Mesh(stage_text(text))


def test_observer_slots_follow_card_order():
    m = vb.Mesh(stage_case("dgref_pml6"))
    names = [m.observer_name(False, s) for s in range(m.num_td)]
    assert len(names) == m.num_td and len(set(names)) == len(names)


def test_default_frequencies_when_no_of_card():
    """numFreq = max(NT/10, 1) (src/observer.c:433-441)."""
    m = vb.Mesh(stage_case("hardsrc_ez"))
    assert m.num_freq == m.num_steps // 10


def test_sheet_sparams_are_passive():
    s11, s21 = meshgen.sheet_sparams()
    assert -1 < s11 < 0 and 0 <= s21 < 1e-6
    assert 1 - (s11 * s11 + s21 * s21) >= 0
