"""Build the vulture_b200 native code in-tree.

Produces
  vulture_b200/lib/libvulture_b200.so   host set-up (C99) + CUDA engine (sm_100a)
  vulture_b200/bin/vulture-b200         the vulture command line on the engine
  oracle/_build/libvcpu.so              CPU oracle (test infrastructure only)

The engine is compiled with ``--fmad=false`` so FP64 results equal the
reference's real=double solver bit for bit (the reference's gcc -O2 build on
x86-64 does not contract multiply-adds).
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "vulture_b200"
HOST_SRC = sorted((PKG / "csrc" / "host").glob("*.c"))
ENGINE_SRC = [PKG / "csrc" / "engine" / "engine.cu"]
ENGINE_HDR = sorted((PKG / "csrc" / "engine").glob("*.cuh")) + sorted((ROOT / "include").glob("*.h"))
OBJ = PKG / "_build"
LIB = PKG / "lib" / "libvulture_b200.so"
CLI = PKG / "bin" / "vulture-b200"
ORACLE_SRC = ROOT / "oracle" / "vcpu.c"
ORACLE_LIB = ROOT / "oracle" / "_build" / "libvcpu.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-std=gnu11", "-O2", "-fPIC", "-Wall", "-Wno-unused-parameter", "-Wno-format-truncation",
          "-Wno-alloc-size-larger-than", f"-I{ROOT / 'include'}", f"-I{PKG / 'csrc' / 'host'}"]
NVFLAGS = GENCODE + ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC",
                     f"-I{ROOT / 'include'}", f"-I{PKG / 'csrc' / 'engine'}", "-Xptxas", "-v"]


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd, quiet=True):
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(map(str, cmd))}")
    return r.stdout + r.stderr


def build_engine(verbose: bool = False) -> Path:
    OBJ.mkdir(parents=True, exist_ok=True)
    LIB.parent.mkdir(parents=True, exist_ok=True)
    objs = []
    for src in HOST_SRC:
        o = OBJ / (src.stem + ".o")
        if _stale(o, [src, *sorted((PKG / "csrc" / "host").glob("*.h")), *sorted((ROOT / "include").glob("*.h"))]):
            _run(["gcc", *CFLAGS, "-c", src, "-o", o])
        objs.append(o)
    for src in ENGINE_SRC:
        o = OBJ / (src.stem + ".o")
        if _stale(o, [src, *ENGINE_HDR]):
            out = _run([NVCC, *NVFLAGS, "-c", src, "-o", o])
            (OBJ / "ptxas.log").write_text(out)
            if verbose:
                print(out)
        objs.append(o)
    if _stale(LIB, objs):
        _run([NVCC, *GENCODE, "-shared", "-o", LIB, *objs, "-lm", "-lpthread"])
    if _stale(CLI, [LIB, PKG / "csrc" / "cli_main.c"]):
        CLI.parent.mkdir(parents=True, exist_ok=True)
        _run(["gcc", "-O2", f"-I{ROOT / 'include'}", PKG / "csrc" / "cli_main.c", "-o", CLI,
              f"-L{LIB.parent}", "-lvulture_b200", "-Wl,-rpath,$ORIGIN/../lib"])
    return LIB


def build_oracle() -> Path:
    """CPU oracle: vcpu64_* (double) and vcpu32_* (float storage)."""
    ORACLE_LIB.parent.mkdir(parents=True, exist_ok=True)
    if _stale(ORACLE_LIB, [ORACLE_SRC, ROOT / "include" / "vgpu.h"]):
        o64 = ORACLE_LIB.parent / "vcpu64.o"
        o32 = ORACLE_LIB.parent / "vcpu32.o"
        # -ffp-contract=off keeps a*b+c as two roundings, like the reference build.
        base = ["gcc", "-std=gnu11", "-O2", "-fPIC", "-ffp-contract=off", f"-I{ROOT / 'include'}"]
        _run([*base, "-DVCPU_REAL=double", "-DVCPU_PREFIX=vcpu64_", "-c", ORACLE_SRC, "-o", o64])
        _run([*base, "-DVCPU_REAL=float", "-DVCPU_PREFIX=vcpu32_", "-c", ORACLE_SRC, "-o", o32])
        _run(["gcc", "-shared", "-o", ORACLE_LIB, o64, o32, "-lm"])
    return ORACLE_LIB


def build_reference() -> bool:
    """Compile the reference solver into oracle/_ref when its sources exist:
    VULTURE_REF, else a checkout named `reference` beside the repository."""
    ref = Path(os.environ.get("VULTURE_REF", str(ROOT.parent / "reference")))
    if not (ref / "src").is_dir():
        return False
    out = ROOT / "oracle" / "_ref"
    env = dict(os.environ, VULTURE_REF=str(ref))
    if not (out / "vulture_oracle_f64_dump").exists():
        subprocess.run(["bash", str(ROOT / "oracle" / "build_ref.sh")], check=True, capture_output=True, env=env)
        return True
    # The propagate() replacements compile against include/vgpu.h and the
    # oracle: rebuild them when those change.
    deps = [ROOT / "include" / "vgpu.h", ORACLE_SRC, *sorted((ROOT / "oracle" / "propagate_gpu").glob("*.c"))]
    for name in ("vulture_ref_oracle_shim", "vulture_ref_gpu"):
        if _stale(out / name, deps):
            subprocess.run(["bash", str(ROOT / "oracle" / "build_ref.sh"), name], check=True, capture_output=True,
                           env=env)
    return True


def build_all(verbose: bool = False):
    build_engine(verbose)
    build_oracle()
    build_reference()


if __name__ == "__main__":
    build_all(verbose="-v" in sys.argv)
    print(f"built {LIB}")
