"""Two populations on one grid (protons and alphas, one batch each), the
interpolated moments, and subcycled acceleration against the oracle."""
import numpy as np
import pytest

from vlasiator_b200.mesh import CHARGE, MASS_PROTON
from vlasiator_b200.projects import random_drifting_cells, sinewave_grid

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def vl():
    from vlasiator_b200 import vlgpu
    vlgpu.load()
    return vlgpu


def test_two_populations_and_interpolated_moments(vl, mesh):
    from vlasiator_b200.populations import combine_moments
    dims = (4, 2, 2)
    species = [(MASS_PROTON, CHARGE, 1.0), (4.0 * MASS_PROTON, 2.0 * CHARGE, 0.05)]
    records_r, records_v, interp = [], [], []
    for m, q, frac in species:
        cells = sinewave_grid(dims, mesh, n0=1e6 * frac)
        params = vl.make_params(charge=q, mass=m)
        total = sum(c.n_blocks for c in cells)
        with vl.Batch(mesh, len(cells), 6 * total + 65536, params=params) as b:
            b.upload([c.gids for c in cells], [c.data for c in cells])
            b.set_grid(dims, 3e5)
            b.vlasov_step(np.stack([c.B for c in cells]), 0.1, 1)
            records_r.append(b.moments_r())
            records_v.append(b.moments(second=True))
            interp.append(b.interpolated_moments())
            assert not b.status().any()
    for r, v, i in zip(records_r, records_v, interp):
        np.testing.assert_allclose(i, 0.5 * (r + v), rtol=1e-15, atol=0)
    cell = combine_moments(records_v, [s[0] for s in species], [s[1] for s in species])
    # the alphas carry 5% of the density and 20% of the mass density
    assert np.allclose(cell[:, 0], records_v[0][:, 4] + records_v[1][:, 4], rtol=1e-12)
    assert (cell[:, 4] > records_v[0][:, 8]).all()


def test_subcycled_acceleration_matches_oracle(vl, mesh, orc_sp):
    from vlasiator_b200.populations import accelerate_subcycled, subcycle_dt
    cells = random_drifting_cells(6, seed=8)
    B = np.stack([c.B for c in cells])
    Tg = 2 * np.pi * MASS_PROTON / (CHARGE * np.linalg.norm(B, axis=1))
    max_v_dt = 0.01 * Tg                  # at most 3.6 degrees per subcycle
    dt = float(0.025 * Tg.min())          # 1 to 3 subcycles per cell
    orders = [0, 1, 2]
    total = sum(c.n_blocks for c in cells)
    with vl.Batch(mesh, len(cells), 6 * total + 65536, exact=True) as b:
        b.upload([c.gids for c in cells], [c.data for c in cells])
        n = accelerate_subcycled(b, B, dt, max_v_dt, orders)
        got = b.cells()
        assert not b.status().any()
    assert n == 3
    for ci, c in enumerate(cells):
        g, d = c.gids, c.data
        for s in range(n):
            sdt = float(subcycle_dt(s, dt, max_v_dt)[ci])
            g, d, *_ = orc_sp.accelerate_step(mesh, g, d, c.B, sdt, orders[s % 3], MASS_PROTON, CHARGE)
        g1, d1 = got[ci]
        common = np.intersect1d(g1, g)
        assert len(common) >= 0.99 * max(len(g), len(g1))
        i1, i2 = np.searchsorted(g1, common), np.searchsorted(g, common)
        assert np.abs(d1[i1] - d[i2]).max() <= 1e-5 * float(np.abs(d).max())
