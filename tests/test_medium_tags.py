"""Medium tags: the set-up's one-byte tag per cell and component.

The host set-up paints, beside the nine coefficient volumes, one byte per
cell and component naming the (alpha, beta, gamma) triple it painted there
(the idea of the reference's USE_INDEXED_MEDIA option, src/grid.h:108-136),
and carries the tags through the UPML carry-in (src/pml.c:445-629).  The
engine builds its coefficient index from the tags instead of scanning the
doubles, so the tags must describe the volumes exactly: every (cell,
component) pair is checked bit for bit on every reference test mesh and on
the synthetic workloads.  A mesh with more than 255 distinct triples keeps
no tags, and the engine then scans the volumes.
"""
import random

import pytest

import vulture_b200 as vb
from vulture_b200 import meshgen
from helpers import case_names, stage_case, stage_text
from test_gpu_parity import many_media_mesh


@pytest.mark.parametrize("case", case_names())
def test_tags_describe_volumes(case):
    m = vb.Mesh(stage_case(case))
    assert m.check_tags() == 0
    m.close()


def synthetic_texts():
    rng = random.Random(4)
    out = {"pec_cube": meshgen.pec_cube(n=48, nt=10),
           "graded_upml": meshgen.graded_upml(nt=10, dims=(80, 64, 48), plane=16, nfreq=4),
           "enclosure": meshgen.shielded_enclosure(nt=10, dims=(120, 90, 75), plane=16, nfreq=4)}
    for q in range(6):
        out[f"batch{q}"] = meshgen.batch_mesh(rng, q, nmin=20, nmax=48, ntmin=10, ntmax=20)
    for q in range(4):
        out[f"serve{q}"] = meshgen.serving_request(rng, q, nmin=24, nmax=48, ntmin=10, ntmax=20)
    return out


@pytest.mark.parametrize("name", list(synthetic_texts()))
def test_tags_describe_synthetic_volumes(name):
    m = vb.Mesh(stage_text(synthetic_texts()[name], name + ".mesh"))
    assert m.check_tags() == 0
    m.close()


def test_too_many_triples_keep_no_tags():
    m = vb.Mesh(stage_text(many_media_mesh(), "many_media.mesh"))
    assert m.check_tags() == -1
    m.use_tags(False)
    m.use_tags(True)      # nothing to put back: still none
    assert m.check_tags() == -1
    m.close()


@pytest.mark.parametrize("seed", range(6))
def test_tags_describe_volumes_of_random_meshes(seed):
    # Batch and serving meshes from other seeds: random media, slabs, sizes,
    # UPML or Mur, Debye blocks and plane waves.
    rng = random.Random(100 + seed)
    for q in range(4):
        text = (meshgen.batch_mesh(rng, q, nmin=16, nmax=40, ntmin=5, ntmax=10) if q % 2 == 0 else
                meshgen.serving_request(rng, q, nmin=20, nmax=44, ntmin=5, ntmax=10))
        m = vb.Mesh(stage_text(text, f"r{seed}_{q}.mesh"))
        assert m.check_tags() == 0
        m.close()
