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

