"""Two populations on one grid (protons and alphas, one batch each), the
interpolated moments, and subcycled acceleration against the oracle
following the reference's subcycle loop (vlasovmover.cpp:503-565)."""
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


def test_two_populations_and_interpolated_moments(vl, mesh, orc_sp):
    """calculateInterpolatedVelocityMoments (vlasovmover.cpp:587-631): every
    moment is 0.5 (_R + _V), the _R set after the translation and the _V set
    after the acceleration; checked against the oracle's own Vlasov step of
    the same grid (exact arithmetic on both sides)."""
    from vlasiator_b200.populations import combine_moments
    dims = (4, 2, 2)
    dx = 3e5
    dt, mo = 0.1, 1
    species = [(MASS_PROTON, CHARGE, 1.0), (4.0 * MASS_PROTON, 2.0 * CHARGE, 0.05)]
    records_v = []
    for m, q, frac in species:
        cells = sinewave_grid(dims, mesh, n0=1e6 * frac)
        params = vl.make_params(charge=q, mass=m)
        total = sum(c.n_blocks for c in cells)
        B = np.stack([c.B for c in cells])
        with vl.Batch(mesh, len(cells), 6 * total + 65536, params=params, exact=True) as b:
            b.upload([c.gids for c in cells], [c.data for c in cells])
            b.set_grid(dims, dx)
            b.vlasov_step(B, dt, mo)
            rec_v = b.moments(second=True)
            interp = b.interpolated_moments()
            assert not b.status().any()
        _, _, mom_r, mom_v, _ = orc_sp.vlasov_step(mesh, dims, [(c.gids, c.data) for c in cells], B, dt, mo,
                                                   (dx, dx, dx), m, q)
        want = 0.5 * (mom_r + mom_v)
        # each moment relative to the size of the quantity it belongs to: a
        # vector component to the vector, a pressure term to the trace
        groups = [[0], [1, 2, 3], [4], [5, 6, 7], [8], [9, 10, 11, 12, 13, 14], [15]]
        for cols in groups:
            scale = np.abs(want[:, cols[0]:cols[-1] + 1]).max()
            for col in cols:
                np.testing.assert_allclose(interp[:, col], want[:, col], rtol=0, atol=1e-9 * scale + 1e-300,
                                           err_msg=f"moment {col}")
        records_v.append(rec_v)
    cell = combine_moments(records_v, [s[0] for s in species], [s[1] for s in species])
    # the alphas carry 5% of the density and 20% of the mass density
    assert np.allclose(cell[:, 0], records_v[0][:, 4] + records_v[1][:, 4], rtol=1e-12)
    assert (cell[:, 4] > records_v[0][:, 8]).all()


def test_subcycled_acceleration_matches_oracle(vl, mesh, orc_sp):
    """The reference's subcycle loop: one dimension order for all subcycles of
    the step, each cell accelerated for its own number of subcycles (the last
    one shortened) and left out afterwards, blocks adjusted after every
    subcycle.  The oracle follows that loop cell by cell."""
    from vlasiator_b200.populations import accelerate_subcycled, cell_subcycles, map_order_for_step, subcycle_dt
    cells = random_drifting_cells(6, seed=8)
    B = np.stack([c.B for c in cells])
    Tg = 2 * np.pi * MASS_PROTON / (CHARGE * np.linalg.norm(B, axis=1))
    max_v_dt = 0.01 * Tg                  # at most 3.6 degrees per subcycle
    dt = float(0.025 * Tg.min())          # 1 to 3 subcycles per cell
    tstep = 60000
    mo = map_order_for_step(tstep)
    counts = cell_subcycles(dt, max_v_dt)
    assert counts.min() < counts.max() == 3
    total = sum(c.n_blocks for c in cells)
    with vl.Batch(mesh, len(cells), 6 * total + 65536, exact=True) as b:
        b.upload([c.gids for c in cells], [c.data for c in cells])
        n = accelerate_subcycled(b, B, dt, max_v_dt, mo)
        got = b.cells()
        assert not b.status().any()
    assert n == 3
    exact = 0
    for ci, c in enumerate(cells):
        g, d = c.gids, c.data
        for s in range(counts[ci]):
            sdt = float(subcycle_dt(s, dt, max_v_dt)[ci])
            assert sdt > 0
            g, d, *_ = orc_sp.accelerate_step(mesh, g, d, c.B, sdt, mo, MASS_PROTON, CHARGE)
        g1, d1 = got[ci]
        if np.array_equal(g1, g) and np.array_equal(d1, d):
            exact += 1
            continue
        # the device's FP64 geometry may differ from the host's in the last
        # bits, which can move a Realf intersection by one ulp
        common = np.intersect1d(g1, g)
        assert len(common) >= 0.99 * max(len(g), len(g1))
        i1, i2 = np.searchsorted(g1, common), np.searchsorted(g, common)
        assert np.abs(d1[i1] - d[i2]).max() <= 1e-5 * float(np.abs(d).max())
    assert exact >= len(cells) - 1


def test_cells_with_zero_dt_pass_through(vl, mesh):
    """A cell whose substep length is zero is not remapped: its blocks and
    values come out of the step as they went in (after an adjustment that
    finds nothing to change)."""
    cells = random_drifting_cells(8, seed=19)
    B = np.stack([c.B for c in cells])
    Tg = 2 * np.pi * MASS_PROTON / (CHARGE * np.linalg.norm(B, axis=1))
    dt = 0.01 * Tg
    still = np.arange(len(cells)) % 3 == 0
    dt[still] = 0.0
    total = sum(c.n_blocks for c in cells)
    for exact in (False, True):
        with vl.Batch(mesh, len(cells), 6 * total + 65536, exact=exact) as b:
            b.upload([c.gids for c in cells], [c.data for c in cells])
            b.adjust()
            before = b.cells()
            b.accelerate(B, dt, 2)
            after = b.cells()
            loss = b.rho_loss()
            assert not b.status().any()
        for ci in range(len(cells)):
            if still[ci]:
                np.testing.assert_array_equal(after[ci][0], before[ci][0])
                assert np.array_equal(after[ci][1], before[ci][1]), f"cell {ci} changed"
            else:
                assert not np.array_equal(after[ci][1][:10], before[ci][1][:10]) or \
                    len(after[ci][0]) != len(before[ci][0])
