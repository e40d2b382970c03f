"""The y-slab ghost exchange of a sharded grid (vlasiator_b200/halo.py) on the
host, with two (and three) gloo ranks, one process each: the slab
bookkeeping, the exchange itself (ghost rows filled with the neighbouring
slabs' owned rows across the periodic wrap), the translation z, x,
exchange, y of every slab with the oracle against the same translation of
the whole grid (bit-identical owned cells), and whole Vlasov steps of the
slabs with three ghost rows and two exchanges, or four and one.  The slabs' cells live in numpy
here; on a GPU the same exchange runs over batches
(tests/test_gpu_halo.py)."""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from vlasiator_b200.halo import Slab

DIMS = (4, 9, 2)
DX = 3e5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class HostSide:
    """The exchange's view of a slab whose cells are numpy (gids, data) pairs."""

    def __init__(self, cells):
        self.cells = list(cells)
        self.device = torch.device("cpu")

    def export(self, cells):
        counts = np.array([len(self.cells[c][0]) for c in cells], np.int32)
        g = np.concatenate([self.cells[c][0] for c in cells] + [np.zeros(0, np.uint32)]).astype(np.int32)
        d = np.concatenate([self.cells[c][1].reshape(-1, 64) for c in cells] + [np.zeros((0, 64), np.float32)])
        return counts, torch.from_numpy(g), torch.from_numpy(d.astype(np.float32))

    def import_(self, cells, counts, gids, data):
        g = gids.cpu().numpy().astype(np.uint32)
        d = data.cpu().numpy()
        o = 0
        for c, n in zip(cells, counts):
            self.cells[int(c)] = (g[o:o + int(n)], d[o:o + int(n)])
            o += int(n)


def _translate(orc, mesh, dims, cells, dim, dt):
    offs = np.zeros(len(cells) + 1, np.uint64)
    offs[1:] = np.cumsum([len(g) for g, _ in cells])
    out = orc.translate(mesh, dims, offs, np.concatenate([g for g, _ in cells]),
                        np.concatenate([d for _, d in cells]), dim, dt, DX)
    return [(g, out[offs[c]:offs[c + 1]]) for c, (g, _) in enumerate(cells)]


def _rank_main(rank, world, port, dims, out):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch.distributed as dist
    from grid_cases import r_dt_restated, varied_grid
    from oracle.oracle import Restatement
    from vlasiator_b200.halo import exchange_ghosts
    from vlasiator_b200.mesh import VelocityMesh
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        mesh = VelocityMesh()
        cells = varied_grid(mesh, dims, seed=3)  # the whole grid, the same on every rank
        whole = [(c.gids, c.data) for c in cells]
        slab = Slab(dims, rank, world)
        glob = slab.local_cells_global()
        side = HostSide([whole[g] for g in glob])
        ghosts = np.concatenate([slab.recv_down, slab.recv_up])
        for c in ghosts:  # nothing in the ghost rows before the exchange
            side.cells[c] = (np.zeros(0, np.uint32), np.zeros((0, 64), np.float32))
        exchange_ghosts(side, slab)
        filled = all(np.array_equal(side.cells[c][0], whole[glob[c]][0]) and
                     np.array_equal(side.cells[c][1], whole[glob[c]][1]) for c in ghosts)
        # translation z, x (slab-local), exchange, y against the whole grid's
        orc = Restatement("sp")
        dt = 0.8 * float(r_dt_restated(mesh, cells, (DX, DX, DX)).min())
        ref = whole
        for dim in (2, 0, 1):
            ref = _translate(orc, mesh, dims, ref, dim, dt)
        for dim in (2, 0):
            side.cells = _translate(orc, mesh, slab.local_dims, side.cells, dim, dt)
        exchange_ghosts(side, slab)
        side.cells = _translate(orc, mesh, slab.local_dims, side.cells, 1, dt)
        owned_equal = all(np.array_equal(side.cells[c][1], ref[glob[c]][1]) for c in slab.owned)
        exchange_ghosts(side, slab)  # the ghost rows now hold the neighbours' translated rows
        ghosts_after = all(np.array_equal(side.cells[c][1], ref[glob[c]][1]) for c in ghosts)
        out[rank] = (filled, owned_equal, ghosts_after, len(slab.owned))
    finally:
        dist.destroy_process_group()


def _rank_step(rank, world, port, dims, ghost, out):
    """A whole Vlasov step of rank's slab with the oracle: translation z, x,
    exchange, y, (exchange,) acceleration with the adjustment over the 26
    neighbours; against the same step of the whole grid."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch.distributed as dist
    from grid_cases import r_dt_restated, varied_grid
    from oracle.oracle import Restatement
    from vlasiator_b200.halo import GHOST_ONE_EXCHANGE, exchange_ghosts
    from vlasiator_b200.mesh import CHARGE, MASS_PROTON, VelocityMesh
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        mesh = VelocityMesh()
        cells = varied_grid(mesh, dims, seed=3)
        whole = [(c.gids, c.data) for c in cells]
        B = np.stack([c.B for c in cells])
        orc = Restatement("sp")
        dt = 0.8 * float(r_dt_restated(mesh, cells, (DX, DX, DX)).min())
        ref, ref_loss, _, ref_mom, _ = orc.vlasov_step(mesh, dims, whole, B, dt, 1, (DX, DX, DX), MASS_PROTON, CHARGE)
        translated = whole
        for dim in (2, 0, 1):
            translated = _translate(orc, mesh, dims, translated, dim, dt)
        slab = Slab(dims, rank, world, ghost)
        glob = slab.local_cells_global()
        side = HostSide([whole[g] for g in glob])
        for dim in (2, 0):
            side.cells = _translate(orc, mesh, slab.local_dims, side.cells, dim, dt)
        exchange_ghosts(side, slab)
        side.cells = _translate(orc, mesh, slab.local_dims, side.cells, 1, dt)
        # the ghost rows next to the owned ones, which the owned cells' adjustment reads
        inner = np.concatenate([slab.rows([ghost - 1]), slab.rows([ghost + slab.n_own])])
        inner_current = all(np.array_equal(side.cells[c][1], translated[glob[c]][1]) for c in inner)
        exchanges = 1
        if ghost < GHOST_ONE_EXCHANGE:
            exchange_ghosts(side, slab)
            exchanges += 1
        got, loss, mom, _ = orc.accelerate_grid(mesh, slab.local_dims, side.cells, B[glob], dt, 1, MASS_PROTON,
                                                CHARGE)
        own = [int(c) for c in slab.owned]
        cells_equal = all(np.array_equal(got[c][0], ref[glob[c]][0]) and np.array_equal(got[c][1], ref[glob[c]][1])
                          for c in own)
        mom_equal = all(np.array_equal(mom[c], ref_mom[glob[c]]) and loss[c] == ref_loss[glob[c]] for c in own)
        out[rank] = (inner_current, cells_equal, mom_equal, exchanges, len(own))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,ghost", [(2, 3), (2, 4), (3, 4)])
def test_sharded_vlasov_step_matches_the_whole_grid(world, ghost):
    """Three ghost rows need the second exchange; with four the rows next to
    the owned ones come out of the y translation current, and one exchange
    per step gives the same owned cells, moments and RHOLOSSADJUST."""
    from vlasiator_b200.halo import GHOST_ONE_EXCHANGE
    dims = (4, 12, 2)
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:  # no fork of a process that holds CUDA
        out = m.dict()
        mp.spawn(_rank_step, args=(world, port, dims, ghost, out), nprocs=world, join=True)
        res = dict(out)
    assert sorted(res) == list(range(world))
    for r, (inner_current, cells_equal, mom_equal, exchanges, _) in res.items():
        assert exchanges == (1 if ghost >= GHOST_ONE_EXCHANGE else 2)
        if ghost >= GHOST_ONE_EXCHANGE:
            assert inner_current, f"rank {r}: the ghost rows next to the owned ones are not current"
        assert cells_equal, f"rank {r}: owned cells differ from the whole grid's step"
        assert mom_equal, f"rank {r}: owned moments or RHOLOSSADJUST differ"
    assert sum(v[4] for v in res.values()) == np.prod(dims)


def test_slab_bookkeeping():
    dims = (3, 10, 2)
    slabs = [Slab(dims, r, 3) for r in range(3)]
    assert [s.n_own for s in slabs] == [4, 3, 3]
    assert [s.y0 for s in slabs] == [0, 4, 7]
    owned = np.concatenate([s.global_of_local(s.owned) for s in slabs])
    assert np.array_equal(np.sort(owned), np.arange(np.prod(dims)))  # every cell owned once
    for r, s in enumerate(slabs):
        up, down = slabs[(r + 1) % 3], slabs[(r - 1) % 3]
        # what I send up is what the slab above keeps as its lower ghost rows, in the same order
        assert np.array_equal(s.global_of_local(s.send_up), up.global_of_local(up.recv_down))
        assert np.array_equal(s.global_of_local(s.send_down), down.global_of_local(down.recv_up))
    with pytest.raises(ValueError):
        Slab((3, 4, 2), 0, 2)  # two rows per slab cannot supply three ghost rows
    with pytest.raises(ValueError):
        Slab((3, 10, 2), 0, 2, ghost=2)  # fewer ghost rows than the translation's stencil reads


@pytest.mark.parametrize("world", [2, 3])
def test_ghost_exchange_and_sharded_translation(world):
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:  # no fork of a process that holds CUDA
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, DIMS, out), nprocs=world, join=True)
        res = dict(out)
    assert sorted(res) == list(range(world))
    for r, (filled, owned_equal, ghosts_after, n_owned) in res.items():
        assert filled, f"rank {r}: ghost rows differ from the neighbours' rows"
        assert owned_equal, f"rank {r}: owned cells differ from the whole grid's translation"
        assert ghosts_after, f"rank {r}: ghost rows after the second exchange"
    assert sum(v[3] for v in res.values()) == np.prod(DIMS)
