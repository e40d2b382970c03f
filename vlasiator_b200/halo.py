"""A spatial grid split over ranks in y-slabs, with the ghost-row exchange its
Vlasov step needs.

The reference distributes its grid with dccrg and exchanges the remote
neighbours' block data around the translation
(update_remote_mapping_contribution_amr, vlasovsolver/cpu_trans_map_amr.cpp:
493-810) and the content lists around the block adjustment (grid.cpp:775-817).
Here a global periodic grid (nx, ny, nz), cells x fastest, is split along y
into one slab per rank: rank r owns the rows y0 <= y < y1 and keeps GHOST = 3
rows of each neighbouring slab, so its batch holds a (nx, n_own + 6, nz) grid
that is periodic in y within itself.  One Vlasov step of a slab:

  1. translation along z and x: rank-local, the pencils lie inside the slab;
  2. ghost exchange: the ghost rows receive the neighbours' owned boundary
     rows (the fused translation reads up to three cells upwind);
  3. translation along y: every owned cell's stencil is local and current;
     the ghost rows take wrapped values that step 4 overwrites;
  4. ghost exchange again, so the ghost rows hold the neighbours' translated
     rows;
  5. the acceleration of every local cell (cells are independent, so a
     ghost cell is accelerated exactly as its owner accelerates it) and the
     block adjustment over the 26 neighbours, whose owned cells see only
     local, current neighbours, with the fused "_V" moments.

The owned cells then equal those of the same step on the whole grid.  With
four ghost rows (Slab(..., ghost=GHOST_ONE_EXCHANGE)) step 4 is left out: the
y translation of the ghost row next to the owned rows reads only rows that
the exchange filled, so it comes out current, and it is the only ghost row
the adjustment of owned cells reads.  That moves four rows per side and step
instead of six, in one exchange instead of two.  The
exchange packs the boundary rows on the device (vlgpu_batch_pack_cells),
moves counts, block IDs and values with point-to-point sends of the process
group (NCCL over NVLink when the group is NCCL; through host memory for
gloo), and unpacks them into the ghost rows (vlgpu_batch_unpack_cells).  No
collective touches the data path; the time-step limit of a sharded grid is
one all-reduce of one double (min over ranks), which the caller makes.
"""
from __future__ import annotations

import numpy as np

GHOST = 3  # rows of each neighbouring slab a rank keeps (the fused walk reads three cells upwind)
GHOST_ONE_EXCHANGE = 4  # with one more row, one ghost exchange per step suffices
_TAG_UP, _TAG_DOWN = 11, 12  # messages travelling towards higher / lower y


class Slab:
    """Rank `rank`'s slab of a (nx, ny, nz) periodic grid split along y over
    `world` ranks, and the local cell indices of its owned and ghost rows."""

    def __init__(self, dims, rank: int, world: int, ghost: int = GHOST):
        nx, ny, nz = (int(v) for v in dims)
        if ghost < GHOST:
            raise ValueError(f"{ghost} ghost rows are fewer than the {GHOST} the translation's stencil reads")
        base, extra = divmod(ny, world)
        self.n_own = base + (1 if rank < extra else 0)
        if self.n_own < ghost:
            raise ValueError(f"slab of {self.n_own} rows is narrower than the {ghost} ghost rows it must supply")
        self.y0 = rank * base + min(rank, extra)
        self.y1 = self.y0 + self.n_own
        self.dims, self.rank, self.world, self.ghost = (nx, ny, nz), rank, world, ghost
        self.local_dims = (nx, self.n_own + 2 * ghost, nz)
        g = ghost
        self.owned = self.rows(range(g, g + self.n_own))
        self.send_up = self.rows(range(self.n_own, self.n_own + g))   # my highest rows -> rank + 1's lower ghosts
        self.send_down = self.rows(range(g, 2 * g))                   # my lowest rows -> rank - 1's upper ghosts
        self.recv_down = self.rows(range(0, g))                       # from rank - 1
        self.recv_up = self.rows(range(g + self.n_own, 2 * g + self.n_own))  # from rank + 1

    def rows(self, local_rows) -> np.ndarray:
        """Local cell indices of the given local y rows, z slowest, then y, then x."""
        nx, ly, nz = self.local_dims
        ys = np.asarray(list(local_rows), np.int64)
        z, y, x = np.meshgrid(np.arange(nz), ys, np.arange(nx), indexing="ij")
        return (x + nx * (y + ly * z)).reshape(-1).astype(np.uint32)

    def global_of_local(self, cells) -> np.ndarray:
        """Global cell index of local cells (periodic in y)."""
        nx, ny, nz = self.dims
        ly = self.local_dims[1]
        c = np.asarray(cells, np.int64)
        x, y, z = c % nx, (c // nx) % ly, c // (nx * ly)
        gy = (self.y0 - self.ghost + y) % ny
        return (x + nx * (gy + ny * z)).astype(np.int64)

    def local_cells_global(self) -> np.ndarray:
        """Global cell index of every local cell, in local order."""
        return self.global_of_local(np.arange(int(np.prod(self.local_dims))))


class BatchSide:
    """The exchange's view of a vlgpu batch: boundary rows out to device
    tensors, received rows into its ghost cells."""

    def __init__(self, batch):
        import torch
        self.batch = batch
        self.device = torch.device("cuda", batch.device)

    def export(self, cells):
        import torch
        counts_all = self.batch.block_counts()
        cap = int(counts_all[np.asarray(cells, np.int64)].sum())
        g = torch.empty(max(cap, 1), dtype=torch.int32, device=self.device)
        d = torch.empty((max(cap, 1), 64), dtype=torch.float32, device=self.device)
        # torch may hand out memory that its own stream still reads; the batch
        # writes it on its stream, which waits for no other
        torch.cuda.current_stream(self.device).synchronize()
        counts, used = self.batch.pack_cells(cells, g.data_ptr(), d.data_ptr(), cap)
        return counts.astype(np.int32), g[:used], d[:used]

    def import_(self, cells, counts, gids, data):
        import torch
        gids = gids.to(self.device).contiguous()
        data = data.to(self.device).contiguous()
        # the received rows were made on torch's stream (an NCCL receive, or a
        # copy from host memory and a cat); the batch reads them on its own
        torch.cuda.current_stream(self.device).synchronize()
        self.batch.unpack_cells(cells, np.asarray(counts, np.uint32), gids.data_ptr(), data.data_ptr())


def _p2p(ops_spec, group, device):
    """Runs (op, tensor, peer, tag) point-to-point operations as one batch,
    with `device` current (NCCL launches its transfers on the current GPU)."""
    import contextlib

    import torch
    import torch.distributed as dist
    ops = [dist.P2POp(dist.isend if kind == "send" else dist.irecv, t, peer, group, tag)
           for kind, t, peer, tag in ops_spec]
    with torch.cuda.device(device) if device.type == "cuda" else contextlib.nullcontext():
        for req in dist.batch_isend_irecv(ops):
            req.wait()


def exchange_ghosts(side, slab: Slab, group=None) -> None:
    """Fills the slab's ghost rows with the neighbouring slabs' owned boundary
    rows.  Every rank of the group calls it at the same point of its step."""
    import torch
    cu, gu, du = side.export(slab.send_up)
    cd, gd, dd = side.export(slab.send_down)
    if slab.world == 1:
        # one slab: its own boundary rows, across the periodic wrap
        rd = (cu, gu, du)
        ru = (cd, gd, dd)
    else:
        import torch.distributed as dist
        backend = dist.get_backend(group)
        comm = side.device if backend == "nccl" else torch.device("cpu")
        up, down = (slab.rank + 1) % slab.world, (slab.rank - 1) % slab.world
        # the per-cell block counts (each side knows how many cells it gets)
        t_cu = torch.from_numpy(cu).to(comm)
        t_cd = torch.from_numpy(cd).to(comm)
        r_cd = torch.empty(len(slab.recv_down), dtype=torch.int32, device=comm)
        r_cu = torch.empty(len(slab.recv_up), dtype=torch.int32, device=comm)
        _p2p([("send", t_cu, up, _TAG_UP), ("send", t_cd, down, _TAG_DOWN),
              ("recv", r_cd, down, _TAG_UP), ("recv", r_cu, up, _TAG_DOWN)], group, comm)
        n_d, n_u = int(r_cd.sum()), int(r_cu.sum())
        # the block IDs and values
        rg_d = torch.empty(max(n_d, 1), dtype=torch.int32, device=comm)
        rv_d = torch.empty((max(n_d, 1), 64), dtype=torch.float32, device=comm)
        rg_u = torch.empty(max(n_u, 1), dtype=torch.int32, device=comm)
        rv_u = torch.empty((max(n_u, 1), 64), dtype=torch.float32, device=comm)
        ops = []
        if len(gu):
            ops += [("send", gu.to(comm).contiguous(), up, _TAG_UP), ("send", du.to(comm).contiguous(), up, _TAG_UP)]
        if len(gd):
            ops += [("send", gd.to(comm).contiguous(), down, _TAG_DOWN),
                    ("send", dd.to(comm).contiguous(), down, _TAG_DOWN)]
        if n_d:
            ops += [("recv", rg_d, down, _TAG_UP), ("recv", rv_d, down, _TAG_UP)]
        if n_u:
            ops += [("recv", rg_u, up, _TAG_DOWN), ("recv", rv_u, up, _TAG_DOWN)]
        if ops:
            _p2p(ops, group, comm)
        rd = (r_cd.cpu().numpy(), rg_d[:n_d], rv_d[:n_d])
        ru = (r_cu.cpu().numpy(), rg_u[:n_u], rv_u[:n_u])
    cells = np.concatenate([slab.recv_down, slab.recv_up])
    counts = np.concatenate([rd[0], ru[0]]).astype(np.uint32)
    side.import_(cells, counts, torch.cat([rd[1].to(side.device), ru[1].to(side.device)]),
                 torch.cat([rd[2].to(side.device), ru[2].to(side.device)]))


def vlasov_step(batch, slab: Slab, B, dt: float, map_order: int, group=None) -> None:
    """One Vlasov step of the rank's slab (the module docstring's order; one
    exchange with GHOST_ONE_EXCHANGE ghost rows, two with fewer).  batch: the
    slab's cells (slab.local_dims, declared with set_grid); B: the field of
    every local cell (ghost cells included)."""
    side = BatchSide(batch)
    batch.translate(2, dt)
    batch.translate(0, dt)
    exchange_ghosts(side, slab, group)
    batch.translate(1, dt)
    if slab.ghost < GHOST_ONE_EXCHANGE:
        exchange_ghosts(side, slab, group)
    batch.accelerate(B, dt, map_order)
