"""Host-side facts the benchmark-config parity tests rely on (no GPU)."""
import numpy as np

import bench
from vlasiator_b200.projects import random_drifting_cells


def test_drifting_cells_generator_is_prefix_stable(mesh):
    """Cell k of the batched-acceleration workload depends only on the seed
    and k, so the first cells of bench.py's 4096 are the same cells as a
    smaller workload of the same seed (the GPU parity tests use 64)."""
    small = random_drifting_cells(16, seed=bench.DEFAULT_SEED, mesh=mesh)
    big = random_drifting_cells(48, seed=bench.DEFAULT_SEED, mesh=mesh)
    for a, b in zip(small, big):
        np.testing.assert_array_equal(a.gids, b.gids)
        np.testing.assert_array_equal(a.data, b.data)
        np.testing.assert_array_equal(a.B, b.B)
    m, offs, gids, data, B, dt = bench.workload(16, bench.DEFAULT_SEED)
    for c, cell in enumerate(small):
        np.testing.assert_array_equal(gids[offs[c]:offs[c + 1]], cell.gids)
        np.testing.assert_array_equal(B[c], cell.B)
