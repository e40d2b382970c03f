"""The oracle's block adjustment pinned against the reference's own code.

The reference build (oracle/_ref) compiles SpatialCell::adjust_velocity_blocks,
compute_block_has_content, update_velocity_block_content_lists and
updateSparseMinValue (spatial_cells/spatial_cell_cpu.cpp:179-273, 290-316,
675-727) and the grid drivers update_velocity_block_content_lists /
adjust_velocity_blocks_in_cells (spatial_cells/block_adjust_cpu.cpp:33-117)
from the reference tree.  The restatement (orc_adjust, orc_adjust_with,
orc_content_gids) must give the same block sets, the same data and the same
RHOLOSSADJUST, with and without spatial neighbours.
"""
import numpy as np
import pytest

from oracle.oracle import ReferenceBuild, grid_neighbors, reference_available
from vlasiator_b200.mesh import WID3
from vlasiator_b200.projects import random_drifting_cells

pytestmark = pytest.mark.skipif(not reference_available("sp"), reason="reference build (oracle/_ref) not present")


def _perturbed_cells(mesh, n, seed):
    """Drifting Maxwellians with blocks removed and empty or faint blocks added,
    so that adjustment both adds and removes blocks."""
    rng = np.random.default_rng(seed)
    cells = random_drifting_cells(n, seed=seed, mesh=mesh)
    out = []
    for c in cells:
        g, d = c.gids.copy(), c.data.copy()
        keep = rng.random(len(g)) > 0.15
        g, d = g[keep], d[keep]
        i, j, k = mesh.indices(g)
        extra = set()
        for _ in range(max(4, len(g) // 8)):
            q = rng.integers(0, len(g))
            off = rng.integers(-3, 4, size=3)
            x, y, z = i[q] + off[0], j[q] + off[1], k[q] + off[2]
            if 0 <= x < mesh.length[0] and 0 <= y < mesh.length[1] and 0 <= z < mesh.length[2]:
                extra.add(int(mesh.gid(x, y, z)))
        extra = np.array(sorted(extra - set(g.tolist())), np.uint32)
        de = np.zeros((len(extra), WID3), np.float32)
        faint = rng.random(len(extra)) < 0.5
        de[faint] = rng.uniform(0, 2e-15, size=(faint.sum(), WID3)).astype(np.float32)
        g = np.concatenate([g, extra])
        d = np.concatenate([d, de])
        o = rng.permutation(len(g))
        out.append((g[o], d[o]))
    return out


def test_content_flags_match_reference(mesh, orc_sp):
    ref = ReferenceBuild("sp")
    ref.init(mesh)
    cells = _perturbed_cells(mesh, 5, seed=31)
    h = ref.create([g for g, _ in cells], [d for _, d in cells], [1e-15] * len(cells))
    try:
        for c, (g, d) in enumerate(cells):
            gr, _ = ref.extract(h, c, sort=False)
            flags = ref.content(h, c)
            want = np.sort(gr[flags])
            np.testing.assert_array_equal(np.sort(orc_sp.content_gids(g, d, 1e-15)), want)
    finally:
        ref.destroy(h)


@pytest.mark.parametrize("add_width", [1, 2])
def test_single_cell_adjust_matches_reference(mesh, orc_sp, add_width):
    ref = ReferenceBuild("sp")
    ref.init(mesh)
    cells = _perturbed_cells(mesh, 6, seed=7 + add_width)
    h = ref.create([g for g, _ in cells], [d for _, d in cells], [1e-15] * len(cells))
    try:
        loss_ref = ref.adjust(h, len(cells), 1e-15, add_width=add_width)
        for c, (g, d) in enumerate(cells):
            go, do, loss = orc_sp.adjust(mesh, g, d, 1e-15, add_width=add_width)
            gr, dr = ref.extract(h, c)
            np.testing.assert_array_equal(go, gr)
            np.testing.assert_array_equal(do, dr)
            assert loss == pytest.approx(loss_ref[c], rel=1e-12, abs=0)
    finally:
        ref.destroy(h)


def test_grid_adjust_matches_reference(mesh, orc_sp):
    grid = (3, 3, 2)
    n = grid[0] * grid[1] * grid[2]
    cells = _perturbed_cells(mesh, n, seed=101)
    nbrs = grid_neighbors(grid)
    ref = ReferenceBuild("sp")
    ref.init(mesh)
    h = ref.create([g for g, _ in cells], [d for _, d in cells], [1e-15] * n)
    try:
        loss_ref = ref.adjust(h, n, 1e-15, add_width=1, neighbors=nbrs)
        out, loss = orc_sp.adjust_grid(mesh, grid, cells, 1e-15)
        for c in range(n):
            gr, dr = ref.extract(h, c)
            np.testing.assert_array_equal(out[c][0], gr)
            np.testing.assert_array_equal(out[c][1], dr)
        np.testing.assert_allclose(loss, loss_ref, rtol=1e-12, atol=0)
    finally:
        ref.destroy(h)



def test_reference_full_step_matches_restatement(mesh, orc_sp):
    """The reference arm's full acceleration step (pivot moments, geometry,
    map_1d x3, adjust, moments) gives the restated step's cells and moments."""
    from vlasiator_b200.mesh import CHARGE, MASS_PROTON
    cells = random_drifting_cells(6, seed=12, mesh=mesh)
    B = np.stack([c.B for c in cells])
    dt = 0.01 * 2 * np.pi * MASS_PROTON / (CHARGE * np.linalg.norm(B, axis=1))
    ref = ReferenceBuild("sp")
    ref.init(mesh)
    h = ref.create([c.gids for c in cells], [c.data for c in cells], [1e-15] * len(cells))
    try:
        mom = ref.full_step(h, B, dt, 2, CHARGE, MASS_PROTON, moments=True)
        for ci, c in enumerate(cells):
            g, d, _, _, m, _ = orc_sp.accelerate_step(mesh, c.gids, c.data, c.B, dt[ci], 2, MASS_PROTON, CHARGE)
            gr, dr = ref.extract(h, ci)
            np.testing.assert_array_equal(gr, g)
            np.testing.assert_array_equal(dr, d)
            assert mom[ci, 0] == pytest.approx(m[0], rel=1e-12)
            np.testing.assert_allclose(mom[ci, 1:4] / mom[ci, 0], m[5:8], rtol=1e-9, atol=1e-6)
            np.testing.assert_allclose(MASS_PROTON * mom[ci, 4:10], m[9:15], rtol=1e-9,
                                       atol=1e-9 * np.abs(m[9:12]).max())
    finally:
        ref.destroy(h)


def test_reference_vlasov_step_matches_restatement(mesh, orc_sp):
    """The reference arm's Vlasov step of a periodic grid (translation z, x, y,
    then the full acceleration step with spatial neighbours in the
    adjustment) gives the restated composition's cells."""
    from vlasiator_b200.mesh import CHARGE, MASS_PROTON
    from vlasiator_b200.projects import sinewave_grid
    dims = (4, 3, 2)
    cells = sinewave_grid(dims, mesh)
    B = np.stack([c.B for c in cells])
    dt, mo, dx = 0.2, 1, (3e5, 3e5, 3e5)
    ref = ReferenceBuild("sp")
    ref.init(mesh)
    h = ref.create([c.gids for c in cells], [c.data for c in cells], [1e-15] * len(cells))
    try:
        ref.vlasov_step(h, dims, dx, B, dt, mo, CHARGE, MASS_PROTON, grid_neighbors(dims))
        want, *_ = orc_sp.vlasov_step(mesh, dims, [(c.gids, c.data) for c in cells], B, dt, mo, dx, MASS_PROTON,
                                      CHARGE)
        for ci in range(len(cells)):
            gr, dr = ref.extract(h, ci)
            np.testing.assert_array_equal(gr, want[ci][0])
            np.testing.assert_array_equal(dr, want[ci][1])
    finally:
        ref.destroy(h)
