"""Generates the golden fixtures in this folder from the reference's own code.

Runs the reference's map_1d (vlasovsolver/cpu_acc_map.cpp:121-636, built by
oracle/build_ref.sh into oracle/_ref/) on small seeded Maxwellian cells and
stores inputs, intersections and outputs as compressed .npz files: PPM in
FP32 and FP64 (map1d_sp, map1d_dp) and the PQM and PLM reconstructions in
FP32 (map1d_sp_pqm, map1d_sp_plm).  The
fixtures let the parity tests pin the oracle and the CUDA path on machines
where the reference tree is not available.

    python tests/golden/make_golden.py [--all]   (default: only missing files)
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import ReferenceBuild, Restatement  # noqa: E402
from vlasiator_b200.mesh import CHARGE, MASS_PROTON, MU_0, VelocityMesh  # noqa: E402
from vlasiator_b200.projects import larmor_cell, maxwellian_cell  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
ORDERS = [[0, 1, 2], [1, 2, 0], [2, 0, 1]]


def _geometry(orc, c, dt_frac, map_order, mesh):
    Bm = float(np.linalg.norm(c.B))
    Tg = 2 * np.pi * MASS_PROTON / (CHARGE * Bm)
    L, t = orc.acceleration_transform(c.B, np.zeros(3), 0.0, c.V, np.zeros(3), CHARGE, MASS_PROTON, dt_frac * Tg,
                                      CHARGE, 0, MU_0)
    return orc.cell_intersections(L, t, mesh, map_order)


def make(precision: str = "sp") -> str:
    mesh = VelocityMesh()
    ref = ReferenceBuild(precision)
    ref.init(mesh)
    orc = Restatement(precision[:2])
    cases = []
    c0 = larmor_cell()
    cases.append(("larmor", c0, 0.01, 0))
    rng = np.random.default_rng(20261203)
    for k in range(3):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        c = maxwellian_cell(mesh, 10 ** rng.uniform(5.5, 6.5), 10 ** rng.uniform(5.0, 5.6), d * rng.uniform(0, 6e5))
        b = rng.normal(size=3)
        c.B = b / np.linalg.norm(b) * rng.uniform(5e-9, 5e-8)
        cases.append((f"drift{k}", c, float(rng.uniform(0.01, 0.07)), k % 3))
    out = {}
    for name, c, frac, mo in cases:
        isect = _geometry(orc, c, frac, mo, mesh)
        out[f"{name}/gids_in"] = c.gids
        out[f"{name}/data_in"] = c.data.astype(ref.realf)
        out[f"{name}/isect"] = isect
        out[f"{name}/map_order"] = np.array(mo)
        h = ref.create([c.gids], [c.data.astype(ref.realf)], [1e-15])
        for s, dim in enumerate(ORDERS[mo]):
            ref.map_1d(h, isect[4 * dim:4 * dim + 4][None, :], dim)
            g, dd = ref.extract(h, 0)
            out[f"{name}/sweep{s}_gids"] = g
            out[f"{name}/sweep{s}_data"] = dd
        ref.destroy(h)
    path = os.path.join(HERE, f"map1d_{precision}.npz")
    np.savez_compressed(path, **out)
    return path


if __name__ == "__main__":
    for p in ("sp", "dp", "sp_pqm", "sp_plm"):
        if "--all" in sys.argv or not os.path.exists(os.path.join(HERE, f"map1d_{p}.npz")):
            print(make(p))
