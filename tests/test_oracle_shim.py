"""The reference-side propagate() replacement (oracle/propagate_gpu/), checked
on the CPU: built into the reference with its five vgpu calls served by the
CPU oracle instead of the GPU (variant vulture_ref_oracle_shim), it must make
the reference write exactly the files its own time loop writes -- every
observer text file and binary file equal, byte for byte, to those of the
reference's FP64 build.  This pins the replacement's reading of the
reference's state (grid, coefficients, UPML, Mur, ghost faces, sources,
observers) without a GPU; tests/test_gpu_reference_shim.py runs the same
replacement on the GPU engine."""
import pytest

from helpers import REF_BIN, run_reference, stage_case

needs = pytest.mark.skipif(not (REF_BIN / "vulture_ref_oracle_shim").exists(),
                           reason="reference builds under oracle/_ref absent")

CASES = ["hardsrc_ex", "softsrc_imdz", "hardsrc_jmsxy", "freespace_mur", "freespace_pml", "dipole_vry",
         "parplate_empty_xyz", "parplate1D_diel", "parplate1D_simplepml_zyx", "closedbox_pec", "waveform_ext"]


def files_of(d):
    return sorted(p.name for p in d.iterdir() if p.suffix in (".asc", ".dat"))


@needs
@pytest.mark.parametrize("case", CASES)
def test_replacement_on_the_oracle_writes_the_references_files(case):
    mesh = stage_case(case)
    ours = run_reference(mesh, "vulture_ref_oracle_shim")
    ref = run_reference(mesh, "vulture_oracle_f64_dump")
    names = files_of(ref)
    assert names and files_of(ours) == names
    for n in names:
        assert (ours / n).read_bytes() == (ref / n).read_bytes(), n
