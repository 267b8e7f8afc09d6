"""The engine's coefficient index from medium tags equals the one from the
volumes: the same run with the set-up's tags handed to vgpu_create and with
them left out (vhost_use_tags) gives the same samples, DFTs and fields bit
for bit, at both precisions, on meshes with UPML, Debye, lumped sources,
PEC wires, SIBC and Mur, and on one whose triples overflow the tags.
"""
import os

import pytest

import vulture_b200 as vb
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
