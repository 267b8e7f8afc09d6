"""The FP32 storage mode's accuracy, on the CPU: the oracle's FP32 variant
(which the FP32 engine equals bit for bit, tests/test_gpu_parity.py) against
its FP64 variant on the synthetic workload shapes, held to the bounds the
engine states:

- time domain: relative L2 per observer point at most 1e-4, over the points
  the pulse has reached (norm at least 1e-3 of the largest; the others hold
  only round-off);
- frequency domain, per result (point x component): the largest magnitude
  error in dB over the frequencies within 60 dB of that result's peak is at
  most 1e-3 dB, or at most the reference's own FP32 error on that result
  where the reference's FP32 build misses 1e-3 dB itself.

The reference's FP32 error comes from its own builds run on the same mesh
(oracle/_ref: vulture_ref_f32, the shipped `real=float`, against
vulture_oracle_f64), compared by the same measure on its observer files
(src/observer.c:949-995, normalised by the waveform's DFT).  The engine keeps
the DFT accumulators in FP64 where the reference keeps them in `real`.
"""
import random

import numpy as np
import pytest

import vulture_b200 as vb
from vulture_b200 import meshgen
from vcpu import CpuRun
from helpers import have_reference_binaries, load_asc, run_reference, stage_text

TD_BOUND = 1e-4
FD_BOUND_DB = 1e-3


def td_errors(a, b):
    norms = np.sqrt((b ** 2).sum(axis=(0, 2)))
    top = norms.max() if norms.size else 0.0
    errs = []
    for p, n in enumerate(norms):
        if n > 0 and n >= 1e-3 * top:
            errs.append(float(np.sqrt(((a[:, p, :] - b[:, p, :]) ** 2).sum()) / n))
    return errs


def db_error(m32, m64):
    """Largest |dB| difference over the frequencies within 60 dB of the FP64
    result's peak; None for a result that is zero throughout."""
    if m64.max() <= 0:
        return None
    sel = m64 > m64.max() * 1e-3
    return float(np.abs(20 * np.log10(np.maximum(m32[sel], 1e-300) / m64[sel])).max())


def cases():
    rng = random.Random(21)
    return {
        "graded_upml": meshgen.graded_upml(nt=300, dims=(36, 30, 24), plane=4, nfreq=16, npml=6, ntd=6),
        "shielded_enclosure": meshgen.shielded_enclosure(nt=300, dims=(56, 48, 40), plane=3, nfreq=16),
        "batch_mesh": meshgen.batch_mesh(rng, 0, nmin=24, nmax=32, ntmin=300, ntmax=300),
        "serving_request": meshgen.serving_request(rng, 1, nmin=24, nmax=32, ntmin=300, ntmax=300),
        "pec_cube": meshgen.pec_cube(nt=300, n=24),
    }


@pytest.mark.parametrize("name", sorted(cases()))
def test_fp32_storage_tracks_fp64(name):
    path = stage_text(cases()[name], f"{name}.mesh")
    m = vb.Mesh(path)
    r32, r64 = CpuRun(m, "fp32").run(), CpuRun(m, "fp64").run()
    errs = td_errors(r32.td(), r64.td())
    if m.num_td:
        assert errs and max(errs) <= TD_BOUND, errs
    if not m.num_fd:
        return
    (a, b), (c, d) = r32.dft(), r64.dft()
    ref32 = ref64 = None
    if have_reference_binaries():
        ref32, ref64 = run_reference(path, "vulture_ref_f32"), run_reference(path, "vulture_oracle_f64")
    checked = 0
    for q in range(m.num_fd):
        name_q = m.observer_name(True, q)
        if ref32 is not None:
            A, B = load_asc(ref32 / f"eh_{name_q}_fd.asc"), load_asc(ref64 / f"eh_{name_q}_fd.asc")
        for comp in range(6):
            mine = db_error(np.hypot(a[q, comp], b[q, comp]), np.hypot(c[q, comp], d[q, comp]))
            if mine is None:
                continue
            bound = FD_BOUND_DB
            if ref32 is not None:
                theirs = db_error(np.hypot(A[:, 1 + 2 * comp], A[:, 2 + 2 * comp]),
                                  np.hypot(B[:, 1 + 2 * comp], B[:, 2 + 2 * comp]))
                if theirs is not None:
                    bound = max(bound, theirs)
            assert mine <= bound, f"{name_q} component {comp}: {mine:.3g} dB > {bound:.3g} dB"
            checked += 1
    assert checked > 0
