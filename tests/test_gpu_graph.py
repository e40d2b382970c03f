"""CUDA-graph capture of device steps (vlgpu_batch_capture / _replay): replays
give results bit-identical to issuing the same steps one call at a time, for
acceleration steps and for full Vlasov steps of a grid, and a replay is
refused when the batch is not in the buffer state of its capture."""
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


def _same(a, b):
    assert len(a) == len(b)
    for (g1, d1), (g2, d2) in zip(a, b):
        np.testing.assert_array_equal(g1, g2)
        assert np.array_equal(d1, d2)


def test_acceleration_graph_replays_match(vl, mesh):
    cells = random_drifting_cells(16, seed=12)
    B = np.stack([c.B for c in cells])
    dt = np.array([0.01 * 2 * np.pi * MASS_PROTON / (CHARGE * np.linalg.norm(c.B)) for c in cells])
    total = sum(c.n_blocks for c in cells)
    outs = []
    for graph in (False, True):
        with vl.Batch(mesh, len(cells), 4 * total + 65536) as b:
            b.upload([c.gids for c in cells], [c.data for c in cells])
            b.accelerate(B, dt, 0)
            if graph:
                b.capture(0, "accel", [1, 2])
                for _ in range(3):
                    b.replay(0)
            else:
                for _ in range(3):
                    b.accelerate_device(1)
                    b.accelerate_device(2)
            outs.append((b.cells(), b.moments(second=True)))
            b.sync()
    _same(outs[0][0], outs[1][0])
    np.testing.assert_array_equal(outs[0][1], outs[1][1])


def test_vlasov_graph_replays_match_and_state_is_checked(vl, mesh):
    dims = (4, 2, 2)
    cells = sinewave_grid(dims, mesh)
    B = np.stack([c.B for c in cells])
    total = sum(c.n_blocks for c in cells)
    dt = 0.1
    outs = []
    for graph in (False, True):
        with vl.Batch(mesh, len(cells), 6 * total + 65536) as b:
            b.upload([c.gids for c in cells], [c.data for c in cells])
            b.set_grid(dims, 3e5)
            b.vlasov_step(B, dt, 0)
            if graph:
                b.capture(3, "vlasov", [1, 2], dt)
                b.replay(3)
                b.replay(3)
            else:
                for o in (1, 2, 1, 2):
                    b.vlasov_step_device(dt, o)
            outs.append(b.cells())
            if graph:
                b.vlasov_step_device(dt, 0)  # an odd step: the buffers are the other set now
                with pytest.raises(vl.VlgpuError):
                    b.replay(3)
            b.sync()
    _same(outs[0], outs[1])
