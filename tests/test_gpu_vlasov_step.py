"""Parity of the grid operations with the oracle: block adjustment with
spatial neighbours (adjustVelocityBlocks, grid.cpp:775-817), the time-step
limits (reduce_vlasov_dt, arch_dt.cpp:34-97; updateAccelerationMaxdt,
cpu_acc_transform.cpp:41-55) and one full Vlasov step (translation z, x, y,
"_R" moments, acceleration, adjustment, "_V" moments) on small periodic grids.

Tolerances: adjustment and the time-step limits are exact (integer sets, the
same IEEE operations).  The Vlasov step in the exact remap mode is bit-exact
wherever the device and host FP64 geometry round to the same Realf
intersections in the cell and its neighbourhood; elsewhere, and in the fused
mode, values agree to 1e-5 of the cell's peak and block sets to 1%.
"""
import numpy as np
import pytest

from oracle.oracle import ReferenceBuild, reference_available
from vlasiator_b200.grid import grid_neighbors
from vlasiator_b200.mesh import CHARGE, MASS_PROTON, WID3
from tests.grid_cases import r_dt_restated, varied_grid
from vlasiator_b200.projects import maxwellian_cell, sinewave_grid

pytestmark = pytest.mark.gpu

DX = 3e5


@pytest.fixture(scope="module")
def vl():
    from vlasiator_b200 import vlgpu
    vlgpu.load()
    return vlgpu


def test_spatial_adjust_matches_oracle(vl, mesh, orc_sp):
    dims = (4, 3, 2)
    cells = varied_grid(mesh, dims, seed=5)
    total = sum(c.n_blocks for c in cells)
    with vl.Batch(mesh, len(cells), 8 * total + 65536) as b:
        b.upload([c.gids for c in cells], [c.data for c in cells])
        b.set_grid(dims, DX)
        b.adjust()
        got = b.cells()
        loss = b.rho_loss()
        b.sync()
        assert not b.status().any()
    ref, ref_loss = orc_sp.adjust_grid(mesh, dims, [(c.gids, c.data) for c in cells], 1e-15)
    grown = 0
    for ci in range(len(cells)):
        np.testing.assert_array_equal(got[ci][0], ref[ci][0], err_msg=f"cell {ci}")
        assert np.array_equal(got[ci][1], ref[ci][1]), f"cell {ci}"
        assert loss[ci] == pytest.approx(ref_loss[ci], rel=1e-12, abs=1e-300)
        grown += len(ref[ci][0]) > len(cells[ci].gids)
    assert grown > len(cells) // 2  # the neighbours' content did add blocks
    # no spatial neighbours: the same cells adjusted alone keep fewer blocks
    with vl.Batch(mesh, len(cells), 8 * total + 65536) as b:
        b.upload([c.gids for c in cells], [c.data for c in cells])
        b.adjust()
        alone = b.cells()
    assert sum(len(g) for g, _ in alone) < sum(len(g) for g, _ in got)


def test_max_dt_matches_restatement(vl, mesh):
    dims = (3, 2, 2)
    dx = (3e5, 2e5, 4e5)
    cells = varied_grid(mesh, dims, seed=11)
    B = np.array([[1e-9 * (c + 1), -2e-9, 3e-9] for c in range(len(cells))])
    with vl.Batch(mesh, len(cells), 4 * sum(c.n_blocks for c in cells)) as b:
        b.upload([c.gids for c in cells], [c.data for c in cells])
        b.set_grid(dims, dx)
        b.compute_intersections(B, 0.01, 0)  # stages the fields
        r, v = b.max_dt(22.0)
    np.testing.assert_array_equal(r, r_dt_restated(mesh, cells, dx))
    if reference_available("sp"):
        # and the reference's own reduce_vlasov_dt (arch_dt.cpp:33-97)
        ref = ReferenceBuild("sp")
        ref.init(mesh)
        h = ref.create([c.gids for c in cells], [c.data for c in cells], [1e-15] * len(cells))
        try:
            r_ref, total = ref.max_r_dt(h, dx)
        finally:
            ref.destroy(h)
        np.testing.assert_array_equal(r, r_ref)
        assert total == r.min()
    Bm = np.sqrt((B ** 2).sum(1)) + 1e-30
    np.testing.assert_allclose(v, np.abs(2 * np.pi * MASS_PROTON / (CHARGE * Bm)) * (22.0 / 360.0), rtol=1e-15)


def _run_step(vl, mesh, dims, cells, dt, mo, exact):
    total = sum(c.n_blocks for c in cells)
    with vl.Batch(mesh, len(cells), 6 * total + 65536, exact=exact) as b:
        b.upload([c.gids for c in cells], [c.data for c in cells])
        b.set_grid(dims, DX)
        b.vlasov_step(np.stack([c.B for c in cells]), dt, mo)
        out = dict(cells=b.cells(), isect=b.intersections(), loss=b.rho_loss(), mom_r=b.moments_r(),
                   mom_v=b.moments(second=True), status=b.status())
        b.sync()
    return out


@pytest.mark.parametrize("exact", [True, False])
def test_vlasov_step_matches_oracle(vl, mesh, orc_sp, exact):
    dims = (6, 2, 2)
    cells = sinewave_grid(dims, mesh)
    dt = 0.8 * float(r_dt_restated(mesh, cells, (DX, DX, DX)).min())
    mo = 1
    got = _run_step(vl, mesh, dims, cells, dt, mo, exact)
    assert not got["status"].any()
    ref, ref_loss, mom_r, mom_v, isect = orc_sp.vlasov_step(mesh, dims, [(c.gids, c.data) for c in cells],
                                                            np.stack([c.B for c in cells]), dt, mo, (DX, DX, DX),
                                                            MASS_PROTON, CHARGE)
    # exact mode: the translation is bit-exact, so the "_R" moments agree to
    # FP64 rounding; fused mode: within the fused translation's tolerance
    np.testing.assert_allclose(got["mom_r"][:, [0, 4, 8, 15]], mom_r[:, [0, 4, 8, 15]],
                               rtol=1e-12 if exact else 1e-6)
    if exact:
        np.testing.assert_allclose(got["isect"], isect, rtol=1e-12, atol=1e-9)
    else:  # the pivot comes from the fused translation's moments
        np.testing.assert_allclose(got["isect"], isect, rtol=1e-6, atol=1e-2)
    same32 = np.all(got["isect"].astype(np.float32) == isect.astype(np.float32), axis=1)
    nbrs = grid_neighbors(dims)
    exact_cells = 0
    for ci in range(len(cells)):
        g1, d1 = got["cells"][ci]
        g2, d2 = ref[ci]
        hood = [ci] + [n for n in nbrs[ci] if n >= 0]
        if exact and all(same32[h] for h in hood):
            np.testing.assert_array_equal(g1, g2, err_msg=f"cell {ci}")
            assert np.array_equal(d1, d2), f"cell {ci}: VDF not bit-exact"
            exact_cells += 1
        else:
            common = np.intersect1d(g1, g2)
            assert len(common) >= 0.99 * max(len(g1), len(g2))
            i1, i2 = np.searchsorted(g1, common), np.searchsorted(g2, common)
            assert np.abs(d1[i1] - d2[i2]).max() <= 1e-5 * float(np.abs(d2).max())
        tol = 1e-9 if exact else 1e-6
        np.testing.assert_allclose(got["mom_v"][ci, [0, 4, 8, 15]], mom_v[ci, [0, 4, 8, 15]], rtol=tol)
    if exact:
        assert exact_cells >= len(cells) // 2
    # mass: translation conserves it up to what enters missing blocks, the
    # adjustment's loss is accounted
    m0 = sum(float(c.data.astype(np.float64).sum()) for c in cells)
    m1 = sum(float(d.astype(np.float64).sum()) for _, d in got["cells"])
    assert abs(m1 / m0 - 1.0) < 1e-3


def test_spatial_adjust_with_a_wide_cell(vl, mesh, orc_sp):
    """One hot cell whose content box (about 48 x 48 rows of y, z) exceeds
    the adjustment's shared-memory mask and the content-mask limit: that cell
    is adjusted with global scratch masks and its neighbours read its block
    list instead of its mask."""
    dims = (3, 2, 2)
    cells = varied_grid(mesh, dims, seed=9)
    cells[4] = maxwellian_cell(mesh, 1e6, 1e8, (1e5, 0.0, -1e5))
    box = np.unique(cells[4].gids // mesh.length[0])  # (y, z) rows of the hot cell
    assert len(box) > 1600
    # every cell of this small periodic grid neighbours the hot one and
    # takes its content blocks
    total = sum(c.n_blocks for c in cells)
    with vl.Batch(mesh, len(cells), len(cells) * cells[4].n_blocks + 4 * total + 65536) as b:
        b.upload([c.gids for c in cells], [c.data for c in cells])
        b.set_grid(dims, DX)
        b.adjust()
        got = b.cells()
        loss = b.rho_loss()
        b.sync()
        assert not b.status().any()
    ref, ref_loss = orc_sp.adjust_grid(mesh, dims, [(c.gids, c.data) for c in cells], 1e-15)
    for ci in range(len(cells)):
        np.testing.assert_array_equal(got[ci][0], ref[ci][0], err_msg=f"cell {ci}")
        assert np.array_equal(got[ci][1], ref[ci][1]), f"cell {ci}"
        assert loss[ci] == pytest.approx(ref_loss[ci], rel=1e-12, abs=1e-300)
