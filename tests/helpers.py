"""Shared helpers of the test suite: fixture paths, the reference's pydiff
tolerance, and running the reference binaries built under oracle/_ref."""
from __future__ import annotations

import gzip
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
CASES = GOLDEN / "cases"
EXPECTED = GOLDEN / "expected"
REF_BIN = ROOT / "oracle" / "_ref"

sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def case_names():
    return sorted(p.name for p in CASES.iterdir() if p.is_dir())


def golden_cases():
    return sorted(p.name for p in EXPECTED.iterdir() if p.is_dir())


def mesh_of(case: str) -> Path:
    return next((CASES / case).glob("*.mesh"))


def stage_case(case: str) -> Path:
    """Copy a case's inputs into a fresh directory; returns the mesh path."""
    d = Path(tempfile.mkdtemp(prefix=f"vb_{case}_"))
    for f in (CASES / case).iterdir():
        shutil.copy(f, d / f.name)
    return d / mesh_of(case).name


def stage_text(text: str, name="m.mesh") -> Path:
    d = Path(tempfile.mkdtemp(prefix="vb_syn_"))
    p = d / name
    p.write_text(text)
    return p


def load_asc(path) -> np.ndarray:
    opener = gzip.open if str(path).endswith(".gz") else open
    with opener(path, "rt") as f:
        return np.loadtxt(f, comments="#", ndmin=2)


def pydiff_ok(valid: np.ndarray, test: np.ndarray, rtol=1e-5, atol=1e-2) -> bool:
    """The reference's test criterion (util/pydiff.py:58-68)."""
    return valid.shape == test.shape and bool(np.allclose(valid, test, rtol=rtol, atol=atol))


def max_rel(a: np.ndarray, b: np.ndarray) -> float:
    """max|a-b| / max|b| per column, the error metric for time series."""
    scale = np.abs(b).max(axis=0)
    scale[scale == 0] = 1.0
    return float((np.abs(a - b) / scale).max()) if a.size else 0.0


def have_reference_binaries() -> bool:
    return (REF_BIN / "vulture_oracle_f64_dump").exists()


def run_reference(mesh: Path, binary="vulture_oracle_f64_dump", timeout=600) -> Path:
    """Run a reference build on a staged mesh in its own directory."""
    d = Path(tempfile.mkdtemp(prefix="vb_ref_"))
    for f in mesh.parent.iterdir():
        if f.is_file() and not f.name.startswith(("eh_", "wf_", "vulture.log")):
            shutil.copy(f, d / f.name)
    r = subprocess.run([str(REF_BIN / binary), mesh.name], cwd=d, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"reference run failed ({r.returncode}): {r.stderr[-500:]}")
    return d


def outputs_in(d: Path):
    return sorted(p.name for p in Path(d).glob("*.asc") if p.name.startswith(("eh_", "wf_")))
