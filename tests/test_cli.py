"""The command-line driver's contract with the caller, without a GPU: the
reference's help/version options, its exit codes (1 for a bad option, 6 for
an input error, src/message.c:104-105), and a plain error, not a fallback,
when no device is present."""
import shutil
import subprocess
from pathlib import Path

import pytest

from conftest import gpu_available
from helpers import CASES

ROOT = Path(__file__).resolve().parent.parent
EXE = ROOT / "vulture_b200" / "bin" / "vulture-b200"


def cli(*args, cwd=None):
    return subprocess.run([str(EXE), *args], cwd=cwd, capture_output=True, text=True, timeout=120)


def test_help_and_version_exit_zero(tmp_path):
    r = cli("-h", cwd=tmp_path)
    assert r.returncode == 0 and "Usage" in r.stdout + r.stderr
    r = cli("-V", cwd=tmp_path)
    assert r.returncode == 0 and "0.7.1" in r.stdout + r.stderr


def test_bad_option_exits_one(tmp_path):
    r = cli("-Z", cwd=tmp_path)
    assert r.returncode == 1 and "invalid option" in r.stdout + r.stderr


def test_missing_mesh_exits_six(tmp_path):
    r = cli(str(tmp_path / "absent.mesh"), cwd=tmp_path)
    assert r.returncode == 6 and "Cannot open input mesh file" in r.stdout + r.stderr


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_no_device_is_an_error_not_a_fallback(tmp_path):
    for f in (CASES / "hardsrc_ez").iterdir():
        shutil.copy(f, tmp_path / f.name)
    r = cli("hardsrc_ez.mesh", cwd=tmp_path)
    assert r.returncode == 6 and "no CUDA device" in r.stdout + r.stderr
    assert not list(tmp_path.glob("eh_*_td.asc"))   # no observer output without the engine
