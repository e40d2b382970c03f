"""Pins the C restatement of map_1d to the reference's own code.

Against the committed fixtures (made by tests/golden/make_golden.py from the
reference's map_1d) the restatement must be bit-exact, in both the FP32 and
the all-FP64 build.  Where the reference build exists locally, random cells
are also compared directly.
"""
import os

import numpy as np
import pytest

from oracle.oracle import ReferenceBuild, Restatement, reference_available
from vlasiator_b200.mesh import CHARGE, MASS_PROTON, MU_0
from vlasiator_b200.projects import random_drifting_cells

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
ORDERS = [[0, 1, 2], [1, 2, 0], [2, 0, 1]]


@pytest.mark.parametrize("precision", ["sp", "dp"])
def test_restatement_matches_reference_fixtures(precision, mesh):
    orc = Restatement(precision)
    z = np.load(os.path.join(GOLDEN, f"map1d_{precision}.npz"))
    names = sorted({k.split("/")[0] for k in z.files})
    assert names
    for name in names:
        g, d = z[f"{name}/gids_in"], z[f"{name}/data_in"]
        isect = z[f"{name}/isect"]
        mo = int(z[f"{name}/map_order"])
        for s, dim in enumerate(ORDERS[mo]):
            g, d, flags = orc.map_1d(mesh, g, d, isect[4 * dim:4 * dim + 4], dim, 1e-15)
            assert flags == 0
            np.testing.assert_array_equal(g, z[f"{name}/sweep{s}_gids"], err_msg=f"{name} sweep {s} block set")
            assert np.array_equal(d, z[f"{name}/sweep{s}_data"]), f"{name} sweep {s} values not bit-exact"


@pytest.mark.skipif(not reference_available("sp"), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("precision", ["sp", "dp"])
def test_restatement_matches_reference_build_random(precision, mesh):
    if not reference_available(precision):
        pytest.skip("reference build missing")
    orc = Restatement(precision)
    ref = ReferenceBuild(precision)
    ref.init(mesh)
    cells = random_drifting_cells(12, seed=11)
    for ci, c in enumerate(cells):
        Bm = np.linalg.norm(c.B)
        Tg = 2 * np.pi * MASS_PROTON / (CHARGE * Bm)
        L, t = orc.acceleration_transform(c.B, np.zeros(3), 0.0, c.V, np.zeros(3), CHARGE, MASS_PROTON, 0.04 * Tg,
                                          CHARGE, 0, MU_0)
        mo = ci % 3
        isect = orc.cell_intersections(L, t, mesh, mo)
        g, d = c.gids, c.data.astype(orc.realf)
        h = ref.create([g], [d], [1e-15])
        try:
            for dim in ORDERS[mo]:
                g, d, _ = orc.map_1d(mesh, g, d, isect[4 * dim:4 * dim + 4], dim, 1e-15)
                ref.map_1d(h, isect[4 * dim:4 * dim + 4][None, :], dim)
                g2, d2 = ref.extract(h, 0)
                np.testing.assert_array_equal(g, g2)
                assert np.array_equal(d, d2)
        finally:
            ref.destroy(h)
