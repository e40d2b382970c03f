"""The r-space time-step statement used by the grid tests, pinned to the
reference's own reduce_vlasov_dt (vlasovsolver/arch_dt.cpp:33-97, compiled by
oracle/build_ref.sh): per cell the minimum over its blocks of dx/|v| at the
centres of each block's first and last cells, exactly."""
import numpy as np
import pytest

from oracle.oracle import ReferenceBuild, reference_available
from tests.grid_cases import r_dt_restated, varied_grid
from vlasiator_b200.projects import random_drifting_cells

pytestmark = pytest.mark.skipif(not reference_available("sp"), reason="reference build (oracle/_ref) not present")


@pytest.mark.parametrize("dx", [(3e5, 3e5, 3e5), (3e5, 2e5, 4e5)])
def test_r_dt_matches_reference(mesh, dx):
    cells = varied_grid(mesh, (3, 2, 2), seed=11) + random_drifting_cells(6, seed=3, mesh=mesh)
    ref = ReferenceBuild("sp")
    ref.init(mesh)
    h = ref.create([c.gids for c in cells], [c.data for c in cells], [1e-15] * len(cells))
    try:
        r_ref, total = ref.max_r_dt(h, dx)
    finally:
        ref.destroy(h)
    r = r_dt_restated(mesh, cells, dx)
    np.testing.assert_array_equal(r, r_ref)
    assert total == r.min()
