"""Generates tests/golden/initial_sp.json from the reference's own code (FP32
build, oracle/build_ref.sh into oracle/_ref/): the initial condition of one
population as Project::setVelocitySpace builds it (projects/project.cpp:
239-260): every block of the mesh (findBlocksToInitialize, project.cpp:
179-218) filled at the cell centres with MaxwellianPhaseSpaceDensity or
TriMaxwellianPhaseSpaceDensity (projects/project.h:45-73), then the first
block adjustment (SpatialCell::adjust_velocity_blocks,
spatial_cells/spatial_cell_cpu.cpp:179-273; minValue 1e-15, addWidthV 1).

The fixture keeps, per case, the block count and SHA-256 digests of the
kept block IDs (uint32) and values (float32, little-endian), sorted by block
ID, so the generator is pinned bit for bit in a few hundred bytes.

    python tests/golden/make_golden_initial.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import ReferenceBuild  # noqa: E402
from vlasiator_b200.mesh import MASS_PROTON, VelocityMesh  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

# (name, n [m^-3], T [K], V [m/s], (Tx, Ty, Tz) [K] or None)
CASES = [
    ("larmor", 1e6, 5e5, (0.0, 0.0, 0.0), None),
    ("drifting", 3e6, 2e6, (3e5, -2e5, 1e5), None),
    ("dense_cold", 1e7, 1e5, (-6e5, 4e5, 0.0), None),
    ("trimaxwellian", 1e6, 1e6, (1e5, 0.0, -2e5), (5e5, 2e6, 1e6)),
]


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def reference_initial_cell(ref: ReferenceBuild, mesh: VelocityMesh, n, T, V, T_aniso):
    """Every block of the mesh filled by the reference, then its first adjustment."""
    gids = np.arange(int(np.prod(mesh.length)), dtype=np.uint32)
    data = ref.fill_blocks(gids, V, T, n, MASS_PROTON, T_aniso)
    h = ref.create([gids], [data], [1e-15])
    try:
        ref.adjust(h, 1, 1e-15, add_width=1)
        return ref.extract(h, 0)
    finally:
        ref.destroy(h)


def make() -> str:
    mesh = VelocityMesh()
    ref = ReferenceBuild("sp")
    ref.init(mesh)
    out = []
    for name, n, T, V, ta in CASES:
        g, d = reference_initial_cell(ref, mesh, n, T, V, ta)
        out.append({"name": name, "n": n, "T": T, "V": list(V), "T_aniso": None if ta is None else list(ta),
                    "n_blocks": int(len(g)), "gids_sha256": digest(g.astype("<u4")),
                    "data_sha256": digest(d.astype("<f4"))})
    path = os.path.join(HERE, "initial_sp.json")
    with open(path, "w") as f:
        json.dump({"min_value": 1e-15, "add_width": 1, "mass": MASS_PROTON, "cases": out}, f, indent=1)
    return path


if __name__ == "__main__":
    print(make())
