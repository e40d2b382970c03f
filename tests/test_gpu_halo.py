"""A grid split in y-slabs over batches (vlasiator_b200/halo.py): full Vlasov
steps of the slabs, with the ghost rows exchanged through the device pack and
unpack entry points, against the same steps of the whole grid in one batch.
The owned cells must come out bit-identical (block IDs, values, first
moments); the pressure tensors agree to 1e-12 (see _check).

One slab (its ghost rows from its own boundary rows across the periodic
wrap) runs in this process; two slabs run as two processes on the one GPU of
the test, exchanging through a gloo group on the host.  The ranks' kernels
never wait on one another: every exchange is a host-side step between
launches."""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

DIMS = (4, 8, 2)
DX = 3e5
STEPS = 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _grid(mesh):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from grid_cases import r_dt_restated, varied_grid
    cells = varied_grid(mesh, DIMS, seed=5)
    dt = 0.8 * float(r_dt_restated(mesh, cells, (DX, DX, DX)).min())
    return cells, dt


def _run_slab(rank, world, group=None):
    """STEPS sharded Vlasov steps of rank's slab; returns its owned cells'
    global indices, (gids, data) and moment records."""
    from vlasiator_b200 import halo, vlgpu
    from vlasiator_b200.mesh import VelocityMesh
    mesh = VelocityMesh()
    cells, dt = _grid(mesh)
    slab = halo.Slab(DIMS, rank, world)
    local = [cells[g] for g in slab.local_cells_global()]
    total = sum(c.n_blocks for c in local)
    B = np.stack([c.B for c in local])
    with vlgpu.Batch(mesh, len(local), 8 * total + 65536) as b:
        b.upload([c.gids for c in local], [c.data for c in local])
        b.set_grid(slab.local_dims, DX)
        for s in range(STEPS):
            halo.vlasov_step(b, slab, B, dt, s % 3, group)
        got = b.cells()
        mom = b.moments(second=True)
        status = b.status()
    owned = slab.owned.astype(np.int64)
    assert not status[owned].any()
    return (slab.global_of_local(owned), [got[c] for c in owned], mom[owned])


def _rank_main(rank, world, port, out):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        glob, cells, mom = _run_slab(rank, world)
        out[rank] = (glob.tolist(), [(g.tolist(), d.tolist()) for g, d in cells], mom.tolist())
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def whole_grid():
    from vlasiator_b200 import vlgpu
    from vlasiator_b200.mesh import VelocityMesh
    mesh = VelocityMesh()
    cells, dt = _grid(mesh)
    total = sum(c.n_blocks for c in cells)
    B = np.stack([c.B for c in cells])
    with vlgpu.Batch(mesh, len(cells), 8 * total + 65536) as b:
        b.upload([c.gids for c in cells], [c.data for c in cells])
        b.set_grid(DIMS, DX)
        for s in range(STEPS):
            b.vlasov_step(B, dt, s % 3) if s == 0 else b.vlasov_step_device(dt, s % 3)
        got = b.cells()
        mom = b.moments(second=True)
        assert not b.status().any()
    return got, mom


def _check(whole_grid, glob, cells, mom):
    """Block IDs, values, the first moments and the plain mass sum bit-identical;
    the pressure tensor to 1e-12 of its diagonal.  (The whole grid's last step
    keeps the translation's pivot and the slabs' the acceleration's; the
    moments below are taken about that pivot, which moves the pressure by a
    few ulp.)"""
    ref_cells, ref_mom = whole_grid
    for gi, (g, d), m in zip(glob, cells, mom):
        np.testing.assert_array_equal(np.asarray(g, np.uint32), ref_cells[gi][0], err_msg=f"cell {gi} block IDs")
        np.testing.assert_array_equal(np.asarray(d, np.float32), ref_cells[gi][1], err_msg=f"cell {gi} values")
        m = np.asarray(m)
        np.testing.assert_array_equal(m[:9], ref_mom[gi][:9], err_msg=f"cell {gi} first moments")
        assert m[15] == ref_mom[gi][15], f"cell {gi} mass sum"
        np.testing.assert_allclose(m[9:15], ref_mom[gi][9:15], rtol=0,
                                   atol=1e-12 * np.abs(ref_mom[gi][9:12]).max(), err_msg=f"cell {gi} pressure")


def test_one_slab_with_wrapped_ghosts_matches_the_whole_grid(whole_grid):
    glob, cells, mom = _run_slab(0, 1)
    assert len(glob) == np.prod(DIMS)
    _check(whole_grid, glob, cells, mom)


def test_two_slabs_match_the_whole_grid(whole_grid):
    world = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:  # no fork of a process that holds CUDA
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert sorted(res) == [0, 1]
    owned = sorted(sum((res[r][0] for r in res), []))
    assert owned == list(range(int(np.prod(DIMS))))
    for r in res:
        _check(whole_grid, *res[r])
