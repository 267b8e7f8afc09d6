"""The FP32 storage mode's accuracy, on the CPU: the oracle's FP32 variant
(which the FP32 engine equals bit for bit, tests/test_gpu_parity.py) against
its FP64 variant on the synthetic workload shapes.  Time domain: relative L2
per observer point at most 1e-4, over the points the pulse has reached
(norm at least 1e-3 of the largest; the others hold only round-off).
Frequency domain: the magnitude error in dB per result (point x component)
over frequencies within 60 dB of that result's peak, reported and bounded
loosely (the 1e-3 dB figure is a per-result report, which the reference's
own FP32 build does not meet on every result)."""
import random

import numpy as np
import pytest

import vulture_b200 as vb
from vulture_b200 import meshgen
from vcpu import CpuRun
from helpers import stage_text


def td_errors(a, b):
    norms = np.sqrt((b ** 2).sum(axis=(0, 2)))
    top = norms.max() if norms.size else 0.0
    errs = []
    for p, n in enumerate(norms):
        if n > 0 and n >= 1e-3 * top:
            errs.append(float(np.sqrt(((a[:, p, :] - b[:, p, :]) ** 2).sum()) / n))
    return errs


def fd_db(re32, im32, re64, im64):
    m32, m64 = np.hypot(re32, im32), np.hypot(re64, im64)
    worst = []
    for q in range(m64.shape[0]):
        for c in range(6):
            ref = m64[q, c]
            if ref.max() <= 0:
                continue
            sel = ref > ref.max() * 1e-3
            worst.append(float(np.abs(20 * np.log10(np.maximum(m32[q, c][sel], 1e-300) / ref[sel])).max()))
    return worst


def cases():
    rng = random.Random(21)
    return {
        "graded_upml": meshgen.graded_upml(nt=300, dims=(36, 30, 24), plane=4, nfreq=16, npml=6, ntd=6),
        "batch_mesh": meshgen.batch_mesh(rng, 0, nmin=24, nmax=32, ntmin=300, ntmax=300),
        "serving_request": meshgen.serving_request(rng, 1, nmin=24, nmax=32, ntmin=300, ntmax=300),
        "pec_cube": meshgen.pec_cube(nt=300, n=24),
    }


@pytest.mark.parametrize("name", sorted(cases()))
def test_fp32_storage_tracks_fp64(name):
    m = vb.Mesh(stage_text(cases()[name], f"{name}.mesh"))
    r32, r64 = CpuRun(m, "fp32").run(), CpuRun(m, "fp64").run()
    errs = td_errors(r32.td(), r64.td())
    assert errs and max(errs) <= 1e-4, errs
    if m.num_fd:
        (a, b), (c, d) = r32.dft(), r64.dft()
        db = fd_db(a, b, c, d)
        assert db and float(np.median(db)) <= 1e-3 and max(db) <= 0.1, db
