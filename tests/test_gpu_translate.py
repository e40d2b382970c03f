"""Parity of the CUDA spatial translation (uniform periodic grid) with the
oracle's restatement of trans_map_1d_amr (vlasovsolver/cpu_trans_map_amr.cpp:
214-443), itself bit-exact against the reference's own build.

In its exact mode the CUDA path evaluates the reference's arithmetic
operation by operation, so block lists and values are compared bit for bit:
cells with different block sets (mass flowing into a missing block is
dropped), pencils of 1 to 6 cells, positive and negative velocities, after a
block adjustment (an indirect state), and the z, x, y sequence of
calculateSpatialTranslation.  The default fused mode is held to 1e-5 of each
cell's peak per sweep.
"""
import numpy as np
import pytest

from vlasiator_b200.mesh import WID3
from vlasiator_b200.projects import maxwellian_cell

pytestmark = pytest.mark.gpu

DZ = 3e5


@pytest.fixture(scope="module")
def vl():
    from vlasiator_b200 import vlgpu
    vlgpu.load()
    return vlgpu


def grid_cells(mesh, grid, seed=0):
    rng = np.random.default_rng(seed)
    cells = []
    n = grid[0] * grid[1] * grid[2]
    for c in range(n):
        x = c % grid[0]
        dens = 1e6 * (1 + 0.5 * np.sin(2 * np.pi * x / grid[0]))
        V = (4e5 + rng.uniform(-5e4, 5e4), rng.uniform(-1e5, 1e5), rng.uniform(-2e5, 2e5))
        cells.append(maxwellian_cell(mesh, dens, rng.uniform(1.5e5, 3e5), V))
    return cells


def packed(cells):
    offs = np.zeros(len(cells) + 1, np.uint64)
    offs[1:] = np.cumsum([len(g) for g, _ in cells])
    return offs, np.concatenate([g for g, _ in cells]), np.concatenate([d for _, d in cells])


def unpack(offs, gids, data):
    out = []
    for c in range(len(offs) - 1):
        g, d = gids[offs[c]:offs[c + 1]], data[offs[c]:offs[c + 1]]
        o = np.argsort(g, kind="stable")
        out.append((g[o], d[o]))
    return out


def oracle_translate(orc, mesh, grid, state, dim, dt):
    offs, gids, data = packed(state)
    out = orc.translate(mesh, grid, offs, gids, data, dim, dt, DZ)
    return [(g, out[offs[c]:offs[c + 1]]) for c, (g, _) in enumerate(state)]


def assert_same(got, ref, what):
    for ci, ((g1, d1), (g2, d2)) in enumerate(zip(got, ref)):
        o = np.argsort(g2, kind="stable")
        np.testing.assert_array_equal(g1, g2[o], err_msg=f"{what}: cell {ci} block IDs")
        assert np.array_equal(d1, d2[o]), f"{what}: cell {ci} max |diff| {np.abs(d1 - d2[o]).max()}"


@pytest.mark.parametrize("grid,dim,dt", [((6, 3, 2), 0, 0.05), ((6, 3, 2), 1, -0.04), ((6, 3, 2), 2, 0.03),
                                         ((5, 4, 1), 0, -0.05), ((3, 1, 4), 2, -0.05), ((1, 5, 2), 1, 0.05)])
def test_translation_sweep_bit_exact(vl, mesh, orc_sp, grid, dim, dt):
    cells = grid_cells(mesh, grid, seed=sum(grid) + dim)
    state = [(c.gids, c.data) for c in cells]
    total = sum(c.n_blocks for c in cells)
    with vl.Batch(mesh, len(cells), 2 * total + 4096, exact=True) as b:
        b.upload([g for g, _ in state], [d for _, d in state])
        b.set_grid(grid, DZ)
        b.translate(dim, dt)
        got = b.cells()
        b.sync()
        assert not b.status().any()
    assert_same(got, oracle_translate(orc_sp, mesh, grid, state, dim, dt), f"grid {grid} dim {dim}")


def test_translation_after_adjust_and_three_dimensions(vl, mesh, orc_sp):
    """Adjustment first (translation then reads an indirect state with added
    zero blocks), then z, x, y as calculateSpatialTranslation orders them."""
    grid = (4, 3, 3)
    cells = grid_cells(mesh, grid, seed=7)
    total = sum(c.n_blocks for c in cells)
    dt = 0.04
    with vl.Batch(mesh, len(cells), 4 * total + 65536, exact=True) as b:
        b.upload([c.gids for c in cells], [c.data for c in cells])
        b.set_grid(grid, DZ)
        b.adjust()
        state = [(g.copy(), d.copy()) for g, d in b.cells()]
        for dim in (2, 0, 1):
            b.translate(dim, dt)
            state = oracle_translate(orc_sp, mesh, grid, state, dim, dt)
            assert_same(b.cells(), state, f"dim {dim}")
        b.sync()
        assert not b.status().any()


def test_translation_conserves_mass_with_common_blocks(vl, mesh):
    grid = (8, 2, 1)
    cells = grid_cells(mesh, grid, seed=3)
    union = np.unique(np.concatenate([c.gids for c in cells]))
    data = []
    for c in cells:
        d = np.zeros((len(union), WID3), np.float32)
        d[np.searchsorted(union, c.gids)] = c.data
        data.append(d)
    with vl.Batch(mesh, len(cells), 2 * len(union) * len(cells)) as b:
        b.upload([union] * len(cells), data)
        b.set_grid(grid, DZ)
        m0 = sum(float(d.astype(np.float64).sum()) for d in data)
        b.translate(0, 0.05)
        b.translate(1, -0.05)
        m1 = sum(float(d.astype(np.float64).sum()) for _, d in b.cells())
    assert abs(m1 / m0 - 1.0) < 1e-6


@pytest.mark.parametrize("grid,dim,dt", [((6, 3, 2), 0, 0.05), ((6, 3, 2), 1, -0.04), ((6, 3, 2), 2, 0.03),
                                         ((1, 2, 3), 0, 0.05), ((1, 2, 3), 1, -0.05), ((1, 2, 3), 2, 0.04),
                                         ((20, 2, 1), 0, -0.03)])
def test_fused_translation_within_tolerance(vl, mesh, orc_sp, grid, dim, dt):
    """Pencils of 1 to 20 cells: the walk's window wraps around a short
    pencil several times, and a 20-cell pencil takes three batches."""
    cells = grid_cells(mesh, grid, seed=40 + dim + sum(grid))
    state = [(c.gids, c.data) for c in cells]
    total = sum(c.n_blocks for c in cells)
    with vl.Batch(mesh, len(cells), 2 * total + 4096) as b:
        assert not b.exact
        b.upload([g for g, _ in state], [d for _, d in state])
        b.set_grid(grid, DZ)
        b.translate(dim, dt)
        got = b.cells()
    ref = oracle_translate(orc_sp, mesh, grid, state, dim, dt)
    for ci, ((g1, d1), (g2, d2)) in enumerate(zip(got, ref)):
        o = np.argsort(g2, kind="stable")
        np.testing.assert_array_equal(g1, g2[o])
        peak = float(np.abs(d2).max())
        assert np.abs(d1 - d2[o]).max() <= 1e-5 * peak, f"cell {ci}"
        m1, m2 = float(d1.astype(np.float64).sum()), float(d2.astype(np.float64).sum())
        assert abs(m1 / m2 - 1) <= 1e-6
