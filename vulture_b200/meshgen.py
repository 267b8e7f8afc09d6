"""Seeded synthetic meshes in the reference's .mesh format for the five
workloads the engine is measured on.

Each generator returns the mesh text; the cards and their meanings follow the
reference's parser (src/mesh.c:58-191).  No public dataset is involved: these
are synthetic shapes of the stated sizes.
"""
from __future__ import annotations

import math
import random


def _graded_lines(rng: random.Random, ncells: int, dmin=1e-3, dmax=8e-3, ratio=1.3):
    """Mesh lines from a graded walk: steps in [dmin, dmax], neighbour ratio
    <= ratio, with both growing and shrinking steps."""
    d = rng.uniform(dmin, dmax)
    lines = [0.0]
    for _ in range(ncells):
        lines.append(lines[-1] + d)
        r = rng.uniform(1.0 / ratio, ratio)
        d = min(max(d * r, dmin), dmax)
    return lines


def _lines_card(tag: str, lines) -> str:
    out = [tag]
    for q in range(0, len(lines), 6):
        out.append(" ".join(f"{v:.9e}" for v in lines[q:q + 6]))
    return "\n".join(out)


def pec_cube(seed: int = 1, nt: int = 1000, n: int = 64) -> str:
    """Free-space cube of n^3 10 mm cells, PEC walls, CN 0.99, hard Ez source
    at the centre (one z-edge), Gaussian pulse (delay 1.5 ns, width 0.5 ns),
    8 time-domain point observers at seeded interior nodes."""
    rng = random.Random(seed)
    c = n // 2
    lines = ["VM 1.0.0", f"CE Synthetic free-space cube {n}^3, PEC walls (seed {seed})", f"DM {n} {n} {n}", "GS"]
    for f in ("XLO", "XHI", "YLO", "YHI", "ZLO", "ZHI"):
        lines.append(f"BT {f} PEC")
    lines.append("WF wf1 GAUSSIAN_PULSE 1.0 1.5e-9 0.5e-9")
    lines.append(f"EX {c} {c} {c} {c} {c} {c + 1} src =EZ wf1 1.0")
    for q in range(8):
        i, j, k = (rng.randint(1, n - 1) for _ in range(3))
        lines.append(f"OP {i} {i} {j} {j} {k} {k} op{q + 1} TDOM_ASCII")
    lines += ["GE", f"NT {nt}", "CN 0.99", "MS 0.01", "EN"]
    return "\n".join(lines) + "\n"


def graded_upml(seed: int = 2, nt: int = 4000, dims=(200, 160, 120), plane=64, nfreq=200, npml=8,
            ntd: int = 16) -> str:
    """Non-uniform graded mesh with 8-cell UPML, one Debye block (eps_s=4,
    eps_inf=2, tau=1e-10 s as one real pole pair), a TFSF plane wave with
    seeded angles and polarisation, 16 time-domain points and a plane x plane
    frequency-domain observer grid on a k-plane."""
    rng = random.Random(seed)
    nx, ny, nz = dims
    out = ["VM 1.0.0", f"CE Synthetic graded mesh {nx}x{ny}x{nz}, UPML, Debye, TFSF (seed {seed})",
           f"DM {nx} {ny} {nz}", "GS"]
    for f in ("XLO", "XHI", "YLO", "YHI", "ZLO", "ZHI"):
        out.append(f"BT {f} PML {npml}")
    # Debye: eps_inf=2, delta eps=2, tau=1e-10 -> residue delta/(2 tau), pole -1/tau.
    tau = 1e-10
    out.append(f"MT deb DEBYE 2.0 0.0 1.0 {2.0 / (2 * tau):.6e} {-1.0 / tau:.6e}")
    inset = 3
    pw = [inset, nx - inset, inset, ny - inset, inset, nz - inset]
    blk = []
    for a, n in enumerate(dims):
        lo = rng.randint(pw[2 * a] + 2, n // 2)
        hi = rng.randint(lo + 2, pw[2 * a + 1] - 2)
        blk += [lo, hi]
    out.append("MB {} {} {} {} {} {} deb".format(*blk))
    out.append("WF wf1 GAUSSIAN_PULSE 1.0")
    theta, phi, eta = rng.uniform(0, 180), rng.uniform(0, 359.9), rng.uniform(0, 359.9)
    out.append("PW {} {} {} {} {} {} pw1 wf1 {:.4f} {:.4f} {:.4f} 111111".format(*pw, theta, phi, eta))
    for q in range(ntd):
        i, j, k = rng.randint(1, nx - 1), rng.randint(1, ny - 1), rng.randint(1, nz - 1)
        out.append(f"OP {i} {i} {j} {j} {k} {k} td{q + 1} TDOM_ASCII")
    kp = rng.randint(nz // 4, 3 * nz // 4)
    i0, j0 = (nx - plane) // 2, (ny - plane) // 2
    for a in range(plane):
        for b in range(plane):
            i, j = i0 + a, j0 + b
            out.append(f"OP {i} {i} {j} {j} {kp} {kp} fd_{a}_{b} FDOM_ASCII")
    out += ["GE", f"NT {nt}", f"OF 1.0e8 1.0e10 {nfreq}"]
    out.append(_lines_card("XL", _graded_lines(rng, nx)))
    out.append(_lines_card("YL", _graded_lines(rng, ny)))
    out.append(_lines_card("ZL", _graded_lines(rng, nz)))
    out.append("EN")
    return "\n".join(out) + "\n"


def sheet_sparams(sigma=1e7, thickness=1e-3, f0=1e9):
    """Real two-port S-parameters of a conducting sheet at f0 from its
    surface resistance: S11 = (Rs - eta0)/(Rs + eta0) and a transmission
    attenuated by the sheet's skin depths.  Used as a zero-pole SIBC model
    (BT name SIBC S11 S12 S21 S22)."""
    mu0 = 4e-7 * math.pi
    eta0 = 376.730313668
    delta = math.sqrt(2.0 / (2 * math.pi * f0 * mu0 * sigma))
    rs = 1.0 / (sigma * delta)
    s11 = (rs - eta0) / (rs + eta0)
    s21 = 4 * rs / eta0 * math.exp(-thickness / delta)
    return s11, s21


def shielded_enclosure(seed: int = 3, nt: int = 20000, dims=(400, 300, 250), plane=128, nfreq=500) -> str:
    """Shielded enclosure: graded mesh, first-order Mur outer boundary, a
    thin-walled box of SIBC walls (sigma=1e7 S/m, 1 mm) with a seeded
    rectangular aperture, 4 PEC thin wires, TFSF illumination, 8 FD points and
    a plane x plane FD observer grid."""
    rng = random.Random(seed)
    nx, ny, nz = dims
    out = ["VM 1.0.0", f"CE Synthetic shielded enclosure {nx}x{ny}x{nz}, SIBC walls (seed {seed})",
           f"DM {nx} {ny} {nz}", "GS"]
    for f in ("XLO", "XHI", "YLO", "YHI", "ZLO", "ZHI"):
        out.append(f"BT {f} MUR")
    s11, s21 = sheet_sparams()
    out.append(f"BT wall SIBC {s11:.9e} {s21:.9e} {s21:.9e} {s11:.9e}")
    out.append("WT wire PEC")
    b = [nx // 4, 3 * nx // 4, ny // 4, 3 * ny // 4, nz // 4, 3 * nz // 4]
    # Aperture in the XLO wall.
    aj0 = rng.randint(b[2] + 2, (b[2] + b[3]) // 2 - 2)
    aj1 = rng.randint(aj0 + 2, b[3] - 2)
    ak0 = rng.randint(b[4] + 2, (b[4] + b[5]) // 2 - 2)
    ak1 = rng.randint(ak0 + 2, b[5] - 2)
    x0 = b[0]
    out.append(f"TB {x0} {x0} {b[2]} {aj0} {b[4]} {b[5]} wall")
    out.append(f"TB {x0} {x0} {aj1} {b[3]} {b[4]} {b[5]} wall")
    out.append(f"TB {x0} {x0} {aj0} {aj1} {b[4]} {ak0} wall")
    out.append(f"TB {x0} {x0} {aj0} {aj1} {ak1} {b[5]} wall")
    out.append(f"TB {b[1]} {b[1]} {b[2]} {b[3]} {b[4]} {b[5]} wall")
    out.append(f"TB {b[0]} {b[1]} {b[2]} {b[2]} {b[4]} {b[5]} wall")
    out.append(f"TB {b[0]} {b[1]} {b[3]} {b[3]} {b[4]} {b[5]} wall")
    out.append(f"TB {b[0]} {b[1]} {b[2]} {b[3]} {b[4]} {b[4]} wall")
    out.append(f"TB {b[0]} {b[1]} {b[2]} {b[3]} {b[5]} {b[5]} wall")
    for w in range(4):
        i = rng.randint(b[0] + 4, b[1] - 4)
        j = rng.randint(b[2] + 4, b[3] - 4)
        k0 = rng.randint(b[4] + 2, (b[4] + b[5]) // 2)
        k1 = rng.randint(k0 + 2, b[5] - 2)
        out.append(f"TW {i} {i} {j} {j} {k0} {k1} wire")
    out.append("WF wf1 GAUSSIAN_PULSE 1.0")
    pw = [6, nx - 6, 6, ny - 6, 6, nz - 6]
    out.append("PW {} {} {} {} {} {} pw1 wf1 {:.4f} {:.4f} {:.4f} 111111".format(
        *pw, rng.uniform(60, 120), rng.uniform(150, 210), rng.uniform(0, 359.9)))
    for q in range(8):
        i = rng.randint(b[0] + 2, b[1] - 2)
        j = rng.randint(b[2] + 2, b[3] - 2)
        k = rng.randint(b[4] + 2, b[5] - 2)
        out.append(f"OP {i} {i} {j} {j} {k} {k} pt{q + 1} FDOM_ASCII")
    kp = (b[4] + b[5]) // 2
    i0, j0 = (nx - plane) // 2, (ny - plane) // 2
    for a in range(plane):
        for c in range(plane):
            out.append(f"OP {i0 + a} {i0 + a} {j0 + c} {j0 + c} {kp} {kp} fd_{a}_{c} FDOM_ASCII")
    out += ["GE", f"NT {nt}", f"OF 1.0e8 3.0e9 {nfreq}"]
    out.append(_lines_card("XL", _graded_lines(rng, nx)))
    out.append(_lines_card("YL", _graded_lines(rng, ny)))
    out.append(_lines_card("ZL", _graded_lines(rng, nz)))
    out.append("EN")
    return "\n".join(out) + "\n"


def batch_mesh(rng: random.Random, index: int, nmin=32, nmax=160, ntmin=2000, ntmax=8000, npml=6) -> str:
    """One batched-workload mesh: per-axis size uniform in [nmin, nmax],
    6-cell UPML, seeded dielectric and PEC slabs, a hard or soft z dipole."""
    n = [rng.randint(nmin, nmax) for _ in range(3)]
    nt = rng.randint(ntmin, ntmax)
    out = ["VM 1.0.0", f"CE Batched mesh {index}", "DM {} {} {}".format(*n), "GS"]
    for f in ("XLO", "XHI", "YLO", "YHI", "ZLO", "ZHI"):
        out.append(f"BT {f} PML {npml}")
    out.append(f"MT diel SIMPLE {rng.uniform(1.0, 10.0):.4f} 0.0 1.0")
    for _ in range(rng.randint(1, 3)):
        a = rng.randrange(3)
        lo = rng.randint(1, n[a] - 3)
        hi = rng.randint(lo + 1, min(n[a] - 1, lo + max(2, n[a] // 4)))
        bb = [1, n[0] - 1, 1, n[1] - 1, 1, n[2] - 1]
        bb[2 * a], bb[2 * a + 1] = lo, hi
        med = "diel" if rng.random() < 0.7 else "PEC"
        out.append("MB {} {} {} {} {} {} {}".format(*bb, med))
    out.append("WF wf1 GAUSSIAN_PULSE 1.0")
    i, j, k = n[0] // 3, n[1] // 3, n[2] // 3
    tag = "=EZ" if rng.random() < 0.5 else "EZ"
    out.append(f"EX {i} {i} {j} {j} {k} {k + 1} src {tag} wf1 1.0")
    out.append(f"OP {n[0] // 2} {n[0] // 2} {n[1] // 2} {n[1] // 2} {n[2] // 2} {n[2] // 2} op1 TDOM_ASCII")
    out += ["GE", f"NT {nt}", "MS 0.01", "EN"]
    return "\n".join(out) + "\n"


def batch_meshes(seed: int = 4, count: int = 256, **kw):
    rng = random.Random(seed)
    return [batch_mesh(rng, q, **kw) for q in range(count)]


def serving_request(rng: random.Random, index: int, nmin=48, nmax=256, ntmin=2000, ntmax=20000) -> str:
    """One serving request: lognormal size clipped to [nmin, nmax] per axis,
    UPML or Mur by coin flip, optional Debye block and TFSF source."""
    mu = math.log(math.sqrt(nmin * nmax))
    n = [int(min(max(rng.lognormvariate(mu, 0.4), nmin), nmax)) for _ in range(3)]
    nt = int(min(max(rng.lognormvariate(math.log(6000), 0.6), ntmin), ntmax))
    out = ["VM 1.0.0", f"CE Serving request {index}", "DM {} {} {}".format(*n), "GS"]
    bnd = "PML 6" if rng.random() < 0.5 else "MUR"
    for f in ("XLO", "XHI", "YLO", "YHI", "ZLO", "ZHI"):
        out.append(f"BT {f} {bnd}")
    if rng.random() < 0.5:
        tau = 1e-10
        out.append(f"MT deb DEBYE 2.0 0.0 1.0 {1.0 / tau:.6e} {-1.0 / tau:.6e}")
        out.append("MB {} {} {} {} {} {} deb".format(n[0] // 2, n[0] - 4, 4, n[1] - 4, 4, n[2] - 4))
    out.append("WF wf1 GAUSSIAN_PULSE 1.0")
    if rng.random() < 0.5:
        out.append("PW 3 {} 3 {} 3 {} pw1 wf1 {:.3f} {:.3f} {:.3f} 111111".format(
            n[0] - 3, n[1] - 3, n[2] - 3, rng.uniform(0, 180), rng.uniform(0, 359.9), rng.uniform(0, 359.9)))
    else:
        i, j, k = n[0] // 2, n[1] // 2, n[2] // 2
        out.append(f"EX {i} {i} {j} {j} {k} {k + 1} src =EZ wf1 1.0")
    out.append(f"OP {n[0] // 3} {n[0] // 3} {n[1] // 3} {n[1] // 3} {n[2] // 3} {n[2] // 3} op1 TDOM_ASCII")
    out.append(f"OP {n[0] // 3} {n[0] // 3} {n[1] // 3} {n[1] // 3} {n[2] // 3} {n[2] // 3} op2 FDOM_ASCII")
    out += ["GE", f"NT {nt}", "OF 1.0e8 5.0e9 100", "MS 0.005", "EN"]
    return "\n".join(out) + "\n"


def write(text: str, path) -> str:
    with open(path, "w") as f:
        f.write(text)
    return str(path)
