"""FP64 parity on the shielded enclosure at its full extent.

The mesh is the enclosure workload's own: 400x300x250 graded cells, Mur outer
boundary, a thin-walled SIBC box with a seeded aperture, 4 PEC thin wires,
TFSF illumination and the 128x128 plane of FD points plus 8 more -- at 8
frequencies instead of 500 and a few dozen steps, so the single-threaded CPU
oracle finishes in about a minute.  Every field starts from the same seeded
random state on both sides (vgpu_write_field / the oracle's write), so from
the first step every update path -- bulk sweeps over 30 M cells, Mur faces,
SIBC walls, wires, Huygens faces -- moves non-zero values.

Expected agreement: the analytic TFSF incident field uses CUDA's exp on the
device and glibc's in the oracle, so values agree to 1e-12 of each
component's peak rather than bit for bit; points farther from every Huygens
face than the pulse of differences can travel in the run's steps are equal
bit for bit.
"""
import os

import numpy as np
import pytest

import vulture_b200 as vb
from vulture_b200 import meshgen
from vcpu import CpuRun
from helpers import stage_text

pytestmark = pytest.mark.gpu

STEPS = 40


def test_enclosure_full_extent_fp64_equals_oracle():
    text = meshgen.shielded_enclosure(seed=3, nt=STEPS, dims=(400, 300, 250), plane=128, nfreq=8)
    path = stage_text(text, "enclosure.mesh")
    old = os.getcwd()
    os.chdir(path.parent)
    try:
        m = vb.Mesh(path.name)
    finally:
        os.chdir(old)
    assert m.num_cells == 400 * 300 * 250 and m.num_fd == 128 * 128 + 8
    import ctypes

    shape = tuple((ctypes.c_int32 * 3).from_address(m.problem().value + 8))
    g = vb.GpuRun(m, "fp64")
    c = CpuRun(m, "fp64")
    rng = np.random.default_rng(17)
    for comp in range(6):
        v = rng.uniform(-1.0, 1.0, size=shape)
        g.write_field(comp, v)
        c.write_field(comp, v)
    del v
    g.run()
    c.run()
    (gr, gi), (cr, ci) = g.dft(), c.dft()
    peak = max(np.abs(cr).max(), np.abs(ci).max())
    assert peak > 0
    assert np.abs(gr - cr).max() <= 1e-12 * peak
    assert np.abs(gi - ci).max() <= 1e-12 * peak
    # Huygens box: 6 cells in from every outer face.  Points more than
    # STEPS + 2 cells inside it have not been reached by any difference.
    lo, hi = 6 + STEPS + 2, np.array([400, 300, 250]) - 6 - STEPS - 2
    for comp in range(6):
        a, b = g.field(comp, shape), c.field(comp, shape)
        top = np.abs(b).max()
        assert top > 0
        assert np.abs(a - b).max() <= 1e-12 * top, f"field {comp}: {np.abs(a - b).max() / top:.3g} of peak"
        inner = (slice(lo + 1, hi[0] + 1), slice(lo + 1, hi[1] + 1), slice(lo + 1, hi[2] + 1))
        assert np.array_equal(a[inner], b[inner]), f"field {comp} differs far from the Huygens faces"
        del a, b
    g.close()
