"""The drop-in command line on the GPU.

`vulture-b200 <mesh>` must write the observer text files the reference's
`vulture <mesh>` writes (src/observer.c:726-798 time domain, 819-854 waveform,
949-995 frequency domain), from the GPU engine:
  - FP64 with --full-precision against the reference's FP64 build printing
    17 significant digits (oracle/_ref/vulture_oracle_f64_dump): the same
    files, every time-domain and waveform file byte for byte; the observer
    DFT files agree to 1e-12 of their peak, since the engine's cos/sin are
    CUDA's and the reference's glibc's;
  - --fp32 (the shipped `real=float` precision) against the reference's own
    golden files with its util/pydiff.py bands, as the reference's CTest
    harness compares them (tests/CMakeLists.txt:55-62).
"""
import shutil
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

from helpers import (EXPECTED, ROOT, golden_cases, have_reference_binaries, load_asc, outputs_in, pydiff_ok,
                     run_reference, stage_case)

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not have_reference_binaries(), reason="reference builds under oracle/_ref absent")
EXE = ROOT / "vulture_b200" / "bin" / "vulture-b200"

# The reference meshes whose FP32 goldens its own build reproduces bit for
# bit, and which hold no analytic plane wave (whose incident field uses
# CUDA's exp, so their time-domain text agrees to 1e-12, not byte for byte).
BYTE_EXACT = ["hardsrc_ex", "hardsrc_ey", "hardsrc_ez", "freespace_mur", "freespace_pml", "parplate_empty_xyz",
              "parplate_empty_zxy", "parplate1D_diel", "softsrc_idz", "dipole_vrx", "closedbox_pec"]


def run_cli(mesh: Path, *opts) -> Path:
    d = Path(tempfile.mkdtemp(prefix="vb_cli_"))
    for f in mesh.parent.iterdir():
        if f.is_file() and not f.name.startswith(("eh_", "wf_", "vulture.log")):
            shutil.copy(f, d / f.name)
    r = subprocess.run([str(EXE), *opts, mesh.name], cwd=d, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-500:] + r.stderr[-500:]
    return d


@needs_ref
@pytest.mark.parametrize("case", BYTE_EXACT)
def test_cli_fp64_files_equal_the_reference_build(case):
    mesh = stage_case(case)
    ours = run_cli(mesh, "--full-precision")
    ref = run_reference(mesh, "vulture_oracle_f64_dump")
    names = outputs_in(ref)
    assert names and outputs_in(ours) == names
    for n in names:
        if n.startswith("eh_") and n.endswith("_fd.asc"):
            a, b = load_asc(ours / n), load_asc(ref / n)
            assert a.shape == b.shape and np.array_equal(a[:, 0], b[:, 0]), n
            peak = np.abs(b[:, 1:]).max()
            assert np.abs(a[:, 1:] - b[:, 1:]).max() <= 1e-12 * max(peak, 1e-300), n
        else:
            assert (ours / n).read_bytes() == (ref / n).read_bytes(), n
    shutil.rmtree(ours, ignore_errors=True)
    shutil.rmtree(ref, ignore_errors=True)


@pytest.mark.parametrize("case", golden_cases())
def test_cli_fp32_files_match_the_reference_goldens(case):
    """Time-domain goldens in the reference's pydiff bands: strict (rtol
    1e-5, atol 1e-2), marginal (1e-4, 1e-1) for the lossless PEC cavities and
    parplate1D_debye_xyz, whose goldens the FP32 set-up in double drifts from
    by a few float ulps (the oracle's golden pin uses the same bands)."""
    mesh = stage_case(case)
    ours = run_cli(mesh, "--fp32")
    files = sorted(p.name[:-3] for p in (EXPECTED / case).glob("*_td.asc.gz"))
    assert files
    marginal = case.startswith(("hardsrc_", "softsrc_")) or case == "parplate1D_debye_xyz"
    band = (1e-4, 1e-1) if marginal else (1e-5, 1e-2)
    for f in files:
        valid, test = load_asc(EXPECTED / case / (f + ".gz")), load_asc(ours / f)
        assert valid.shape == test.shape, f
        assert pydiff_ok(valid, test, *band), f"{case}/{f}: max abs diff {np.abs(valid - test).max()}"
    shutil.rmtree(ours, ignore_errors=True)
