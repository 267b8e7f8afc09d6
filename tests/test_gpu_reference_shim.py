"""The drop-in boundary from the reference's side, on the GPU.

oracle/propagate_gpu/propagate_gpu.c is the reference's own propagate()
(src/simulation.c:136-231) rewritten on the C ABI of include/vgpu.h: built
into the reference (variant vulture_ref_gpu, linked against
vulture_b200/lib/libvulture_b200.so), it fills a vgpu_problem from the
reference's state, runs every step on the GPU engine and hands the samples
back to the reference's own observer code.  On every reference mesh it maps
(no plane wave, SIBC surface or Debye medium), that binary must write the
files the reference's FP64 build writes with its CPU loop -- every text and
binary observer file equal byte for byte, frequency-domain files included,
since the reference accumulates those itself from the engine's bit-exact
samples."""
import pytest

from helpers import REF_BIN, run_reference, stage_case

pytestmark = pytest.mark.gpu
needs = pytest.mark.skipif(not (REF_BIN / "vulture_ref_gpu").exists(), reason="reference builds under oracle/_ref absent")

CASES = ["hardsrc_ex", "hardsrc_ey", "hardsrc_ez", "hardsrc_jmsxy", "softsrc_idx", "softsrc_imdz", "freespace_mur",
         "freespace_pml", "dipole_vrx", "dipole_vry", "parplate_empty_xyz", "parplate_empty_zyx", "parplate1D_diel",
         "parplate1D_simplepml_xyz", "parplate1D_simpleslab_yzx", "closedbox_pec", "waveform_ext", "dgref_pml6"]


def files_of(d):
    return sorted(p.name for p in d.iterdir() if p.suffix in (".asc", ".dat"))


@needs
@pytest.mark.parametrize("case", CASES)
def test_reference_with_the_gpu_propagate_writes_its_own_files(case):
    mesh = stage_case(case)
    ours = run_reference(mesh, "vulture_ref_gpu")
    ref = run_reference(mesh, "vulture_oracle_f64_dump")
    names = files_of(ref)
    assert names and files_of(ours) == names
    for n in names:
        assert (ours / n).read_bytes() == (ref / n).read_bytes(), n
    log = (ours / "vulture.log").read_text()
    assert "GPU engine" in log
