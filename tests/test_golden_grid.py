"""The oracle's grid operations against the committed fixture
tests/golden/grid_sp.npz, which the reference's own FP32 build produced
(tests/golden/make_golden_grid.py): translation along each dimension
(cpu_trans_map_amr.cpp:214-443), block adjustment with the 26 spatial
neighbours (grid.cpp:775-817, block_adjust_cpu.cpp:55-117,
spatial_cell_cpu.cpp:179-273), the r-space time-step limit (arch_dt.cpp:33-97),
one whole Vlasov step and the map-order draw (vlasovmover.cpp:422-426).
These pins hold without the reference tree or its build."""
import os

import numpy as np
import pytest

from tests.grid_cases import r_dt_restated
from vlasiator_b200.mesh import CHARGE, MASS_PROTON, WID3

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "grid_sp.npz")


class _Cell:
    def __init__(self, gids, data):
        self.gids, self.data = gids, data


@pytest.fixture(scope="module")
def fx():
    with np.load(PATH) as z:
        return {k: z[k] for k in z.files}


def _cells(fx, prefix):
    o = fx[f"{prefix}/offsets"].astype(np.int64)
    g = fx[f"{prefix}/gids"]
    d = fx[f"{prefix}/data"].reshape(-1, WID3)
    return [(g[o[c]:o[c + 1]], d[o[c]:o[c + 1]]) for c in range(len(o) - 1)]


@pytest.mark.parametrize("dim", [0, 1, 2])
def test_translation_matches_fixture(fx, mesh, orc_sp, dim):
    dims, dx, dt = tuple(int(v) for v in fx["dims"]), fx["dx"], float(fx["dt"])
    out = orc_sp.translate(mesh, dims, fx["input/offsets"], fx["input/gids"], fx["input/data"], dim, dt, dx[dim])
    want = fx[f"trans{dim}/data"].reshape(-1, WID3)
    assert np.array_equal(out, want), f"max |diff| {np.abs(out - want).max()}"


def test_grid_adjust_matches_fixture(fx, mesh, orc_sp):
    dims = tuple(int(v) for v in fx["dims"])
    cells = _cells(fx, "adjust_in")
    out, loss = orc_sp.adjust_grid(mesh, dims, cells, 1e-15)
    o = fx["adjust/offsets"].astype(np.int64)
    for c, (g, d) in enumerate(cells):
        want_g = fx["adjust/gids"][o[c]:o[c + 1]]
        np.testing.assert_array_equal(out[c][0], want_g, err_msg=f"cell {c} block IDs")
        # the reference moves no values: each output block is its input row, or zeros
        row = {int(x): q for q, x in enumerate(g)}
        want_d = np.stack([d[row[int(x)]] if int(x) in row else np.zeros(WID3, np.float32) for x in want_g])
        np.testing.assert_array_equal(out[c][1], want_d, err_msg=f"cell {c} values")
    np.testing.assert_allclose(loss, fx["adjust/loss"], rtol=1e-12, atol=0)
    # the case both removes blocks that hold mass and adds blocks
    assert (fx["adjust/loss"] > 0).any()
    assert any(len(np.setdiff1d(fx["adjust/gids"][o[c]:o[c + 1]], g)) for c, (g, _) in enumerate(cells))


@pytest.mark.parametrize("q", [0, 1])
def test_r_dt_matches_fixture(fx, mesh, q):
    cells = [_Cell(g, d) for g, d in _cells(fx, "input")]
    np.testing.assert_array_equal(r_dt_restated(mesh, cells, fx[f"dt/dx{q}"]), fx[f"dt/r{q}"])


def test_vlasov_step_matches_fixture(fx, mesh, orc_sp):
    dims, dx, dt = tuple(int(v) for v in fx["dims"]), tuple(fx["dx"]), float(fx["dt"])
    cells = _cells(fx, "input")
    got, loss, _, mom_v, _ = orc_sp.vlasov_step(mesh, dims, cells, fx["B"], dt, int(fx["map_order"]), dx,
                                                MASS_PROTON, CHARGE)
    for c, (g, d) in enumerate(_cells(fx, "vstep")):
        np.testing.assert_array_equal(got[c][0], g, err_msg=f"cell {c} block IDs")
        np.testing.assert_array_equal(got[c][1], d, err_msg=f"cell {c} values")
    np.testing.assert_allclose(loss, fx["vstep/loss"], rtol=1e-12, atol=0)
    ref = fx["vstep/moments"]  # n, nV, sum f (v - V)(v - V) per cell
    np.testing.assert_allclose(mom_v[:, 0], ref[:, 0], rtol=1e-12)
    np.testing.assert_allclose(mom_v[:, 5:8], ref[:, 1:4] / ref[:, :1], rtol=1e-9, atol=1e-6)
    np.testing.assert_allclose(mom_v[:, 9:15], MASS_PROTON * ref[:, 4:10], rtol=1e-9,
                               atol=1e-9 * np.abs(mom_v[:, 9:12]).max())


def test_map_order_matches_fixture(fx):
    from vlasiator_b200.populations import map_order_for_step
    got = [map_order_for_step(int(t)) for t in fx["map_order/steps"]]
    assert got == fx["map_order/order"].tolist()
    assert set(got) == {0, 1, 2}
