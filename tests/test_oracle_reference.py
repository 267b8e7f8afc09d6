"""Pin the oracle to the reference itself: the reference compiled from its own
sources with real=double (oracle/build_ref.sh) and the oracle give identical
17-digit observer values on every reference test mesh and on small versions
of the five synthetic workloads."""
import os
import random

import numpy as np
import pytest

import vulture_b200 as vb
from vulture_b200 import meshgen
from vcpu import CpuRun
from helpers import case_names, have_reference_binaries, load_asc, outputs_in, run_reference, stage_case, stage_text

pytestmark = pytest.mark.skipif(not have_reference_binaries(), reason="reference binaries not built")


def oracle_outputs(mesh):
    old = os.getcwd()
    os.chdir(mesh.parent)
    try:
        m = vb.Mesh(mesh.name)
        c = CpuRun(m, "fp64").run()
        re, im = c.dft()
        m.write_outputs(mesh.parent, c.td(), re, im, full_precision=True)
    finally:
        os.chdir(old)
    return mesh.parent


def assert_identical(ref_dir, mine_dir):
    names = outputs_in(ref_dir)
    assert names
    for f in names:
        a = load_asc(ref_dir / f)
        b = load_asc(mine_dir / f)
        assert a.shape == b.shape, f
        assert np.array_equal(a, b), f"{f}: max diff {np.abs(a - b).max()}"


SLOW = {"dgref_ref", "dgrefmb_ref", "sgref_mur", "sgref_pml6", "sgref_pml12"}


@pytest.mark.parametrize("case", [c for c in case_names() if c not in SLOW])
def test_oracle_equals_reference_fp64(case):
    mesh = stage_case(case)
    ref = run_reference(mesh)
    assert_identical(ref, oracle_outputs(mesh))


def synthetic_small():
    rng = random.Random(7)
    return {
        "pec_cube": meshgen.pec_cube(nt=60, n=20),
        "graded_upml": meshgen.graded_upml(nt=80, dims=(30, 24, 20), plane=4, nfreq=12, ntd=3),
        "shielded_enclosure": meshgen.shielded_enclosure(nt=60, dims=(40, 32, 28), plane=4, nfreq=10),
        "batch_mesh": meshgen.batch_mesh(rng, 0, nmin=16, nmax=28, ntmin=50, ntmax=80),
        "serving_request": meshgen.serving_request(rng, 1, nmin=20, nmax=28, ntmin=50, ntmax=80),
    }


@pytest.mark.parametrize("name", list(synthetic_small()))
def test_oracle_equals_reference_on_synthetic_workloads(name):
    mesh = stage_text(synthetic_small()[name])
    ref = run_reference(mesh)
    assert_identical(ref, oracle_outputs(mesh))
