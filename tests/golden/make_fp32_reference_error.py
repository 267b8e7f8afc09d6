"""Generate tests/golden/fp32_reference_error.json.gz: the error of the
reference's own FP32 build against its FP64 build on the graded
200x160x120 UPML mesh (Debye block, TFSF, 16 time-domain points and a
64x64 plane of frequency-domain points over 200 frequencies, 4000 steps).

Both runs are the reference's own binaries, compiled from its sources by
oracle/build_ref.sh: vulture_ref_f32_omp (typedef float real, as shipped)
and vulture_oracle_f64_omp (real = double).  Their observer files
(src/observer.c:760-798 time domain, src/observer.c:949-995 frequency domain,
both "%16.8e") are compared with the error measures the engine's FP32 mode is
held to:
  - time domain, per point observer: relative L2 of the six components'
    samples over all steps, ||a - b|| / ||b||;
  - frequency domain, per result (point observer x component): the largest
    |20 log10 |X32| - 20 log10 |X64|| over the frequencies where |X64| is
    within 60 dB of that result's peak.
The reference normalises every DFT by its waveform's DFT (observer.c:972-981);
the ratio of magnitudes is what is compared.

Run from the repository root (takes tens of minutes on 8 cores):
    python tests/golden/make_fp32_reference_error.py [threads]
"""
from __future__ import annotations

import gzip
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

OUT = Path(__file__).resolve().parent / "fp32_reference_error.json.gz"
MESH = dict(seed=2, nt=4000, dims=(200, 160, 120), plane=64, nfreq=200, npml=8, ntd=16)


def run(binary: Path, directory: Path, threads: int) -> float:
    t0 = time.perf_counter()
    r = subprocess.run([str(binary), "-n", str(threads), "graded_upml.mesh"], cwd=directory,
                       env=dict(os.environ, OMP_NUM_THREADS=str(threads)), capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{binary.name} failed: {r.stderr[-400:]}")
    return time.perf_counter() - t0


def read_cols(path: Path) -> np.ndarray:
    return np.loadtxt(path, ndmin=2)


def td_rel_l2(a: np.ndarray, b: np.ndarray) -> tuple[float, float]:
    """Columns: step, then six components (observer.c:791-793)."""
    a, b = a[:, 1:7], b[:, 1:7]
    den = float(np.sqrt((b ** 2).sum()))
    return (float(np.sqrt(((a - b) ** 2).sum())) / den if den > 0 else 0.0), den


def fd_db(a: np.ndarray, b: np.ndarray) -> list[float]:
    """Columns: frequency, then (re, im) per component (observer.c:972-984).
    Per component: the largest dB difference over the frequencies within 60 dB
    of the FP64 result's peak (NaN for a result that is zero throughout)."""
    out = []
    for c in range(6):
        m32 = np.hypot(a[:, 1 + 2 * c], a[:, 2 + 2 * c])
        m64 = np.hypot(b[:, 1 + 2 * c], b[:, 2 + 2 * c])
        peak = m64.max()
        if peak <= 0:
            out.append(float("nan"))
            continue
        sel = m64 > peak * 1e-3
        d = np.abs(20 * np.log10(np.maximum(m32[sel], 1e-300)) - 20 * np.log10(m64[sel]))
        out.append(float(d.max()))
    return out


def main():
    from vulture_b200 import meshgen

    threads = int(sys.argv[1]) if len(sys.argv) > 1 else (os.cpu_count() or 1)
    ref = ROOT / "oracle" / "_ref"
    text = meshgen.graded_upml(**MESH)
    work = Path(tempfile.mkdtemp(prefix="vb_fp32ref_"))
    dirs = {}
    walls = {}
    for name in ("vulture_ref_f32_omp", "vulture_oracle_f64_omp"):
        d = work / name
        d.mkdir()
        (d / "graded_upml.mesh").write_text(text)
        walls[name] = run(ref / name, d, threads)
        dirs[name] = d
        print(f"{name}: {walls[name]:.1f} s", flush=True)
    d32, d64 = dirs["vulture_ref_f32_omp"], dirs["vulture_oracle_f64_omp"]
    td, fd = {}, {}
    for f in sorted(d64.glob("eh_*_td.asc")):
        e, n = td_rel_l2(read_cols(d32 / f.name), read_cols(f))
        td[f.name[3:-7]] = {"rel_l2": e, "norm": n}
    for f in sorted(d64.glob("eh_*_fd.asc")):
        fd[f.name[3:-7]] = fd_db(read_cols(d32 / f.name), read_cols(f))
    # Four significant digits are kept: the fixture serves as a per-result bound.
    td = {k: {"rel_l2": float(f"{v['rel_l2']:.4g}"), "norm": float(f"{v['norm']:.4g}")} for k, v in td.items()}
    fd = {k: [float(f"{x:.4g}") if x == x else None for x in v] for k, v in fd.items()}
    out = {"mesh": {k: list(v) if isinstance(v, tuple) else v for k, v in MESH.items()},
           "builds": ["vulture_ref_f32_omp", "vulture_oracle_f64_omp"], "threads": threads,
           "wall_s": walls, "window_db": 60.0, "td": td, "fd_db": fd}
    with gzip.open(OUT, "wt") as fh:
        json.dump(out, fh)
    v = np.array([x for r in fd.values() for x in r if x is not None])
    print(f"wrote {OUT}: {len(td)} TD points, {v.size} FD results; FD dB median {np.median(v):.3g}, "
          f"p99 {np.percentile(v, 99):.3g}, max {v.max():.3g}")
    subprocess.run(["rm", "-rf", str(work)], check=False)


if __name__ == "__main__":
    main()
