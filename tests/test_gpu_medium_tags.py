"""The engine's coefficient index from medium tags equals the one from the
volumes: the same run with the set-up's tags handed to vgpu_create and with
them left out (vhost_use_tags) gives the same samples, DFTs and fields bit
for bit, at both precisions, on meshes with UPML, Debye, lumped sources,
PEC wires, SIBC and Mur, and on one whose triples overflow the tags.
"""
import ctypes
import os
import subprocess
from pathlib import Path

import pytest

import vulture_b200 as vb
from vulture_b200 import _native as N
from vulture_b200 import meshgen
from helpers import stage_case, stage_text
from test_batch_serve import assert_same_run
from test_gpu_parity import many_media_mesh

pytestmark = pytest.mark.gpu


def meshes():
    yield "dipole_vrz", stage_case("dipole_vrz")
    yield "parplate1D_sibcspar_xyz", stage_case("parplate1D_sibcspar_xyz")
    yield "graded_upml", stage_text(meshgen.graded_upml(nt=120, dims=(60, 48, 40), plane=8, nfreq=5, npml=6),
                                    "graded.mesh")
    yield "enclosure", stage_text(meshgen.shielded_enclosure(nt=120, dims=(80, 64, 56), plane=8, nfreq=5),
                                  "enclosure.mesh")
    yield "many_media", stage_text(many_media_mesh(), "many_media.mesh")


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("name,path", list(meshes()))
def test_tagged_index_equals_scanned(name, path, precision):
    m = vb.Mesh(path)
    tagged = vb.GpuRun(m, precision).run()
    m.use_tags(False)
    scanned = vb.GpuRun(m, precision).run()
    m.use_tags(True)
    assert_same_run(m, tagged, scanned)


def test_creation_reports_the_tag_path(capfd):
    m = vb.Mesh(stage_case("dipole_vrz"))
    os.environ["VGPU_TRACE"] = "1"
    try:
        vb.GpuRun(m, "fp32").close()
        m.use_tags(False)
        vb.GpuRun(m, "fp32").close()
        m.use_tags(True)
    finally:
        os.environ.pop("VGPU_TRACE", None)
    lines = [ln for ln in capfd.readouterr().err.splitlines() if ln.startswith("vgpu create")]
    assert len(lines) == 2
    assert " coef-from-tags " in lines[0] and " coef " in lines[1]


def tag_offsets(tmp_path):
    """Offsets of coef_tag and num_tags in vgpu_problem, from the header."""
    root = Path(__file__).resolve().parents[1]
    src = tmp_path / "off.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "vgpu.h"\n'
                   'int main(void) { printf("%zu %zu\\n", offsetof(vgpu_problem, coef_tag), '
                   'offsetof(vgpu_problem, num_tags)); return 0; }\n')
    exe = tmp_path / "off"
    subprocess.run(["gcc", "-I", str(root / "include"), str(src), "-o", str(exe)], check=True)
    a, b = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    return int(a), int(b)


def test_tag_past_the_table_is_rejected(tmp_path):
    m = vb.Mesh(stage_case("dipole_vrz"))
    p = m.problem("fp32")
    off_tag, off_num = tag_offsets(tmp_path)
    tags = ctypes.c_void_p.from_address(p.value + off_tag).value
    num = ctypes.c_int32.from_address(p.value + off_num).value
    assert tags and 0 < num < 255
    q = m.num_cells // 2
    cell = ctypes.c_uint8.from_address(tags + q)
    old = cell.value
    cell.value = num + 1
    try:
        with pytest.raises(N.NativeError) as err:
            vb.GpuRun(m, "fp32")
        assert err.value.code == N.VGPU_EINVAL and "medium tag" in str(err.value)
    finally:
        cell.value = old
    a = vb.GpuRun(m, "fp32").run()
    m.use_tags(False)
    b = vb.GpuRun(m, "fp32").run()
    m.use_tags(True)
    assert_same_run(m, a, b)
