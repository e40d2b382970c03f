"""Pins the restated spatial translation (uniform periodic grid) to the
reference's own trans_map_1d_amr (vlasovsolver/cpu_trans_map_amr.cpp:214-443),
compiled into oracle/_ref, and checks conservation and drift."""
import numpy as np
import pytest

from oracle.oracle import ReferenceBuild, reference_available
from vlasiator_b200.mesh import WID3
from vlasiator_b200.projects import maxwellian_cell


def small_grid(mesh, grid, seed=0):
    rng = np.random.default_rng(seed)
    cells = []
    n = grid[0] * grid[1] * grid[2]
    for c in range(n):
        x = c % grid[0]
        dens = 1e6 * (1 + 0.5 * np.sin(2 * np.pi * x / grid[0]))
        V = (4e5 + rng.uniform(-5e4, 5e4), rng.uniform(-1e5, 1e5), rng.uniform(-1e5, 1e5))
        cells.append(maxwellian_cell(mesh, dens, 2e5, V))
    offs = np.zeros(n + 1, np.uint64)
    offs[1:] = np.cumsum([c.n_blocks for c in cells])
    gids = np.concatenate([c.gids for c in cells])
    data = np.concatenate([c.data for c in cells])
    return cells, offs, gids, data


@pytest.mark.skipif(not reference_available("sp"), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("dim", [0, 1, 2])
def test_translation_matches_reference(mesh, orc_sp, dim):
    grid = (6, 3, 2)
    cells, offs, gids, data = small_grid(mesh, grid, seed=dim)
    dz = 3e5
    dt = 0.5 * dz / 8e5 * (1 if dim != 1 else -1) * (1 if dim != 2 else 1)
    dt = abs(dt)
    out = orc_sp.translate(mesh, grid, offs, gids, data, dim, dt, dz)
    ref = ReferenceBuild("sp")
    ref.init(mesh)
    h = ref.create([c.gids for c in cells], [c.data for c in cells], [1e-15] * len(cells))
    try:
        ref.translate(h, grid, dim, dt, dz)
        for ci, c in enumerate(cells):
            g, d = ref.extract(h, ci)
            np.testing.assert_array_equal(g, c.gids)
            mine = out[offs[ci]:offs[ci + 1]]
            assert np.array_equal(d, mine), f"cell {ci}: max |diff| {np.abs(d - mine).max()}"
    finally:
        ref.destroy(h)


def test_translation_conserves_mass_when_all_blocks_exist(mesh, orc_sp):
    grid = (8, 1, 1)
    cells, offs, gids, data = small_grid(mesh, grid, seed=3)
    # give every cell the union of the block sets so no mass can be dropped
    union = np.unique(gids)
    data2 = []
    for c in cells:
        d = np.zeros((len(union), WID3), np.float32)
        d[np.searchsorted(union, c.gids)] = c.data
        data2.append(d)
    offs2 = np.arange(len(cells) + 1, dtype=np.uint64) * len(union)
    g2 = np.tile(union, len(cells))
    d2 = np.concatenate(data2)
    out = orc_sp.translate(mesh, grid, offs2, g2, d2, 0, 0.3, 3e5)
    assert abs(out.astype(np.float64).sum() / d2.astype(np.float64).sum() - 1) < 1e-6
    # the density profile moves towards +x (V_x ~ +400 km/s)
    n0 = d2.reshape(len(cells), -1).astype(np.float64).sum(1)
    n1 = out.reshape(len(cells), -1).astype(np.float64).sum(1)
    shift = np.angle(np.fft.fft(n1)[1] / np.fft.fft(n0)[1])
    assert shift < 0  # phase of the first harmonic moves to larger x
