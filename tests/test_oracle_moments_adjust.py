"""Oracle moments and block adjustment: pinned against the reference's own
moment templates (where the reference build exists) and against their
defining properties."""
import numpy as np
import pytest

from oracle.oracle import ReferenceBuild, reference_available
from vlasiator_b200.mesh import CHARGE, K_B, MASS_PROTON, WID3
from vlasiator_b200.projects import maxwellian_cell, random_drifting_cells


def test_moments_of_a_maxwellian(mesh, orc_dp):
    n, T, V = 2e6, 1e6, np.array([1.5e5, -2e5, 3e4])
    c = maxwellian_cell(mesh, n, T, V, dtype=np.float64)
    m = orc_dp.moments(mesh, c.gids, c.data, MASS_PROTON, CHARGE)
    assert abs(m[0] / n - 1) < 2e-3                  # density
    np.testing.assert_allclose(m[5:8], V, atol=2e3)  # bulk velocity (m/s)
    P = n * K_B * T
    np.testing.assert_allclose(m[9:12] / P, 1.0, atol=1e-2)  # isotropic pressure
    assert np.all(np.abs(m[12:15]) < 1e-6 * P)               # no shear
    assert m[4] == m[0] * MASS_PROTON and m[8] == m[0] * CHARGE


@pytest.mark.skipif(not reference_available("sp"), reason="reference build (oracle/_ref) not present")
def test_moments_match_reference_templates(mesh, orc_sp):
    ref = ReferenceBuild("sp")
    ref.init(mesh)
    cells = random_drifting_cells(6, seed=4)
    h = ref.create([c.gids for c in cells], [c.data for c in cells], [1e-15] * len(cells))
    try:
        for ci, c in enumerate(cells):
            m = orc_sp.moments(mesh, c.gids, c.data, MASS_PROTON, CHARGE)
            first, second = ref.moments(h, ci, m[5:8])
            np.testing.assert_allclose(m[0:4], first, rtol=1e-12, atol=0)
            # off-diagonal terms are sums that cancel: compare against the trace
            scale = np.abs(m[9:12]).max()
            np.testing.assert_allclose(m[9:15], MASS_PROTON * second, rtol=1e-10, atol=1e-11 * scale)
    finally:
        ref.destroy(h)


def test_adjust_properties(mesh, orc_sp):
    c = maxwellian_cell(mesh, 1e6, 5e5, (1e5, 0, 0))
    # an arbitrary superset of the pruned mesh: all blocks of a box around it
    g0, d0 = c.gids, c.data
    i, j, k = mesh.indices(g0)
    box = [mesh.gid(x, y, z) for x in range(i.min() - 2, i.max() + 3) for y in range(j.min() - 2, j.max() + 3)
           for z in range(k.min() - 2, k.max() + 3)]
    box = np.array(sorted(set(box) - set(g0.tolist())), np.uint32)
    g = np.concatenate([g0, box])
    d = np.concatenate([d0, np.full((len(box), WID3), 1e-17, np.float32)])
    ga, da, loss = orc_sp.adjust(mesh, g, d, 1e-15)
    # adjusting an already adjusted mesh returns it unchanged
    np.testing.assert_array_equal(ga, g0)
    np.testing.assert_array_equal(da, d0)
    assert loss == pytest.approx(len(box) * 64 * 1e-17 * (3e4 ** 3), rel=1e-6)
    gb, db, loss2 = orc_sp.adjust(mesh, ga, da, 1e-15)
    np.testing.assert_array_equal(gb, ga)
    assert loss2 == 0.0


def test_adjust_adds_zero_neighbours(mesh, orc_sp):
    g = np.array([mesh.gid(10, 20, 30)], np.uint32)
    d = np.zeros((1, WID3), np.float32)
    d[0, 5] = 2e-15
    ga, da, loss = orc_sp.adjust(mesh, g, d, 1e-15)
    assert len(ga) == 27 and loss == 0.0
    assert np.array_equal(da[ga == g[0]][0], d[0])
    assert da.sum() == d.sum()
    # at the mesh corner the neighbourhood is clipped
    g = np.array([mesh.gid(0, 0, 0)], np.uint32)
    ga, _, _ = orc_sp.adjust(mesh, g, d, 1e-15)
    assert len(ga) == 8
