"""Copy the reference's own test inputs and a subset of its golden outputs
into tests/golden/ so the suite runs where the reference tree is absent.

  cases/<case>/     the .mesh file and any input files it reads
                    (pole-residue, Debye and external-waveform files)
  expected/<case>/  the reference's golden eh_*/wf_* .asc files, gzipped,
                    for the cases listed in GOLDEN_CASES (FP32 results of
                    the reference as shipped; tolerance rtol 1e-5, atol 1e-2
                    as its util/pydiff.py)
  parser/           the reference's parser negative tests

Run from the repository root: python tests/golden/make_fixtures.py
"""
from __future__ import annotations

import gzip
import os
import shutil
import sys
from pathlib import Path

REF = Path(os.environ.get("VULTURE_REF", str(Path(__file__).resolve().parents[3] / "reference"))) / "tests"
HERE = Path(__file__).resolve().parent

GOLDEN_CASES = [
    "hardsrc_ex", "hardsrc_ey", "hardsrc_ez", "softsrc_idx", "softsrc_imdz",
    "freespace_mur", "freespace_pml", "waveform_ext", "planewave_empty_xyz", "planewave_pec_yzx",
    "dipole_vry", "closedbox_go04", "closedbox_spar", "dgref_pml6", "parplate_empty_zxy",
    "parplate1D_debye_xyz", "parplate1D_diel", "parplate1D_sibcspar_yxz", "parplate1D_planewave_zyx",
]


def main():
    if not REF.is_dir():
        sys.exit(f"reference tests not found at {REF}")
    cases = HERE / "cases"
    expected = HERE / "expected"
    for d in (cases, expected, HERE / "parser"):
        if d.exists():
            shutil.rmtree(d)
        d.mkdir(parents=True)
    for case in sorted(p.name for p in REF.iterdir() if p.is_dir()):
        src = REF / case
        meshes = list(src.glob("*.mesh"))
        if case == "parser":
            for m in meshes:
                shutil.copy(m, HERE / "parser" / m.name)
            continue
        if not meshes:
            continue
        dst = cases / case
        dst.mkdir()
        for f in src.iterdir():
            if f.suffix == ".mesh" or f.suffix in (".pfe", ".prm", ".dat") or (
                    f.suffix == ".asc" and not f.name.startswith(("eh_", "wf_"))):
                if f.name.startswith(("analytic", "impulse", "excite", "process")):
                    continue
                shutil.copy(f, dst / f.name)
        if case in GOLDEN_CASES:
            edst = expected / case
            edst.mkdir()
            for f in sorted(src.glob("*.asc")):
                if f.name.startswith(("eh_", "wf_")):
                    with open(f, "rb") as fi, gzip.open(edst / (f.name + ".gz"), "wb", compresslevel=9) as fo:
                        fo.write(fi.read())
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
