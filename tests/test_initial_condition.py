"""The host initial-condition generator (vlasiator_b200/projects.py,
maxwellian_cell) against the reference's own initial condition:
Project::setVelocitySpace (projects/project.cpp:239-260) filling every block
with MaxwellianPhaseSpaceDensity / TriMaxwellianPhaseSpaceDensity
(projects/project.h:45-73) at the cell centres, then the first
adjust_velocity_blocks (spatial_cells/spatial_cell_cpu.cpp:179-273).

The committed digests (tests/golden/initial_sp.json, made by
tests/golden/make_golden_initial.py from the reference build) pin the block
IDs and values bit for bit without the reference; with the reference build
present the same comparison runs against it directly, for the whole mesh and
for a box three blocks beyond the content."""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle.oracle import ReferenceBuild, reference_available
from vlasiator_b200.mesh import MASS_PROTON
from vlasiator_b200.projects import maxwellian_cell

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "initial_sp.json")
with open(PATH) as _f:
    FIXTURE = json.load(_f)
CASES = FIXTURE["cases"]


def _generate(mesh, case):
    ta = case["T_aniso"]
    return maxwellian_cell(mesh, case["n"], case["T"], case["V"], min_value=FIXTURE["min_value"],
                           add_width=FIXTURE["add_width"], T_aniso=None if ta is None else (*ta, np.eye(3)))


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_generator_matches_reference_digests(mesh, case):
    c = _generate(mesh, case)
    assert c.n_blocks == case["n_blocks"]
    assert hashlib.sha256(c.gids.astype("<u4").tobytes()).hexdigest() == case["gids_sha256"]
    assert hashlib.sha256(np.ascontiguousarray(c.data, "<f4").tobytes()).hexdigest() == case["data_sha256"]


@pytest.mark.skipif(not reference_available("sp"), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_generator_matches_reference_fill_and_adjust(mesh, case):
    ref = ReferenceBuild("sp")
    ref.init(mesh)
    c = _generate(mesh, case)
    ta = case["T_aniso"]
    # the fill alone, on the generator's blocks
    np.testing.assert_array_equal(ref.fill_blocks(c.gids, case["V"], case["T"], case["n"], MASS_PROTON, ta), c.data)
    # fill and first adjustment over a box three blocks beyond the content
    L = np.array(mesh.length)
    i, j, k = mesh.indices(c.gids)
    lo = np.maximum(np.array([i.min(), j.min(), k.min()]) - 3, 0)
    hi = np.minimum(np.array([i.max(), j.max(), k.max()]) + 3, L - 1)
    ii, jj, kk = np.meshgrid(*[np.arange(lo[d], hi[d] + 1) for d in range(3)], indexing="ij")
    box = mesh.gid(ii.ravel(), jj.ravel(), kk.ravel()).astype(np.uint32)
    h = ref.create([box], [ref.fill_blocks(box, case["V"], case["T"], case["n"], MASS_PROTON, ta)],
                   [FIXTURE["min_value"]])
    try:
        ref.adjust(h, 1, FIXTURE["min_value"], add_width=FIXTURE["add_width"])
        g, d = ref.extract(h, 0)
    finally:
        ref.destroy(h)
    np.testing.assert_array_equal(g, c.gids)
    np.testing.assert_array_equal(d, c.data)
