"""Generates tests/golden/grid_sp.npz from the reference's own code (FP32
build, oracle/build_ref.sh into oracle/_ref/), on a small periodic grid of
narrow drifting Maxwellians:

  trans{0,1,2}/*  one translation sweep along x, y, z
                  (trans_map_1d_amr, vlasovsolver/cpu_trans_map_amr.cpp:214-443);
  adjust/*        block adjustment of perturbed cells with their 26 spatial
                  neighbours (adjustVelocityBlocks with the NEAREST
                  neighbourhood, grid.cpp:775-817; adjust_velocity_blocks_in_cells,
                  spatial_cells/block_adjust_cpu.cpp:55-117;
                  SpatialCell::adjust_velocity_blocks, spatial_cell_cpu.cpp:179-273);
  dt/*            the r-space time-step limit per cell for two cell sizes
                  (reduce_vlasov_dt, vlasovsolver/arch_dt.cpp:33-97);
  vstep/*         one whole Vlasov step: translation z, x, y, then the
                  acceleration of every cell and the adjustment with
                  neighbours (vlasovmover.cpp:65-381, 410-569);
  map_order       the dimension order drawn for time steps 0..199 and a few
                  large ones (vlasovmover.cpp:422-426).

The adjustment moves no values: the generator checks that every output
block holds the input row of its block ID (or zeros for an added block), so
the fixture stores only the output block IDs.  Translation keeps each cell's
block set, so it stores only the output values.

    python tests/golden/make_golden_grid.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import ReferenceBuild  # noqa: E402
from vlasiator_b200.grid import grid_neighbors  # noqa: E402
from vlasiator_b200.mesh import CHARGE, MASS_PROTON, WID3, VelocityMesh  # noqa: E402
from vlasiator_b200.projects import maxwellian_cell  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
DIMS = (4, 2, 2)
DX = (3e5, 3e5, 3e5)
DT = 0.2
MAP_ORDER = 1
MAP_ORDER_STEPS = np.array(list(range(200)) + [42589, 42590, 99991, 1234567, 2 ** 31 - 2, 2 ** 31 - 1], np.int64)


def grid_cells(mesh, seed=20261203):
    """Narrow drifting Maxwellians, density a sine in x, with B of random
    direction and 5-10 nT; (gids, data) per cell and B."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = DIMS
    cells, B = [], []
    for c in range(nx * ny * nz):
        x = c % nx
        n = 1e6 * (1 + 0.5 * np.sin(2 * np.pi * x / nx))
        V = (4e5 + rng.uniform(-5e4, 5e4), rng.uniform(-5e4, 5e4), rng.uniform(-5e4, 5e4))
        cell = maxwellian_cell(mesh, n, float(rng.uniform(4e4, 8e4)), V)
        b = rng.normal(size=3)
        B.append(b / np.linalg.norm(b) * rng.uniform(5e-9, 1e-8))
        cells.append((cell.gids, cell.data))
    return cells, np.stack(B)


def perturbed(mesh, cells, seed):
    """The cells with about 15% of their blocks removed and empty or faint
    blocks added near the rest, in shuffled order, so that the adjustment
    both adds and removes blocks."""
    rng = np.random.default_rng(seed)
    out = []
    for g, d in cells:
        keep = rng.random(len(g)) > 0.15
        g, d = g[keep], d[keep]
        i, j, k = mesh.indices(g)
        extra = set()
        for _ in range(max(4, len(g) // 8)):
            q = rng.integers(0, len(g))
            off = rng.integers(-3, 4, size=3)
            x, y, z = i[q] + off[0], j[q] + off[1], k[q] + off[2]
            if 0 <= x < mesh.length[0] and 0 <= y < mesh.length[1] and 0 <= z < mesh.length[2]:
                extra.add(int(mesh.gid(x, y, z)))
        extra = np.array(sorted(extra - set(g.tolist())), np.uint32)
        de = np.zeros((len(extra), WID3), np.float32)
        faint = rng.random(len(extra)) < 0.5
        de[faint] = rng.uniform(0, 2e-15, size=(faint.sum(), WID3)).astype(np.float32)
        o = rng.permutation(len(g) + len(extra))
        out.append((np.concatenate([g, extra])[o], np.concatenate([d, de])[o]))
    return out


def _pack(prefix, cells, out):
    out[f"{prefix}/offsets"] = np.concatenate([[0], np.cumsum([len(g) for g, _ in cells])]).astype(np.uint64)
    out[f"{prefix}/gids"] = np.concatenate([g for g, _ in cells]).astype(np.uint32)
    out[f"{prefix}/data"] = np.concatenate([d for _, d in cells]).astype(np.float32)


def make() -> str:
    mesh = VelocityMesh()
    ref = ReferenceBuild("sp")
    ref.init(mesh)
    cells, B = grid_cells(mesh)
    n = len(cells)
    nbrs = grid_neighbors(DIMS)
    out = {"dims": np.array(DIMS), "dx": np.array(DX), "dt": np.array(DT), "map_order": np.array(MAP_ORDER),
           "B": B}
    _pack("input", cells, out)

    for dim in range(3):
        h = ref.create([g for g, _ in cells], [d for _, d in cells], [1e-15] * n)
        try:
            ref.translate(h, DIMS, dim, DT, DX[dim])
            rows = []
            for c, (g, _) in enumerate(cells):
                gr, dr = ref.extract(h, c)
                assert np.array_equal(gr, np.sort(g)), "translation changed a block set"
                rows.append(dr[np.searchsorted(gr, g)])  # in the input's block order
            out[f"trans{dim}/data"] = np.concatenate(rows).astype(np.float32)
        finally:
            ref.destroy(h)

    pert = perturbed(mesh, cells, seed=77)
    _pack("adjust_in", pert, out)
    h = ref.create([g for g, _ in pert], [d for _, d in pert], [1e-15] * n)
    try:
        out["adjust/loss"] = ref.adjust(h, n, 1e-15, add_width=1, neighbors=nbrs)
        res = []
        for c, (g, d) in enumerate(pert):
            gr, dr = ref.extract(h, c)
            for q, gid in enumerate(gr):
                hit = np.nonzero(g == gid)[0]
                want = d[hit[0]] if len(hit) else np.zeros(WID3, np.float32)
                assert np.array_equal(dr[q], want), "adjustment changed a block's values"
            res.append((gr, dr))
        out["adjust/offsets"] = np.concatenate([[0], np.cumsum([len(g) for g, _ in res])]).astype(np.uint64)
        out["adjust/gids"] = np.concatenate([g for g, _ in res]).astype(np.uint32)
    finally:
        ref.destroy(h)

    h = ref.create([g for g, _ in cells], [d for _, d in cells], [1e-15] * n)
    try:
        for q, dx in enumerate([DX, (3e5, 2e5, 4e5)]):
            r, total = ref.max_r_dt(h, dx)
            out[f"dt/dx{q}"] = np.array(dx)
            out[f"dt/r{q}"] = r
            assert total == r.min()
    finally:
        ref.destroy(h)

    h = ref.create([g for g, _ in cells], [d for _, d in cells], [1e-15] * n)
    try:
        mom, loss = ref.vlasov_step(h, DIMS, DX, B, DT, MAP_ORDER, CHARGE, MASS_PROTON, nbrs, moments=True)
        _pack("vstep", [ref.extract(h, c) for c in range(n)], out)
        out["vstep/moments"] = mom
        out["vstep/loss"] = loss
        assert ref.bailouts() == 0
    finally:
        ref.destroy(h)

    out["map_order/steps"] = MAP_ORDER_STEPS
    out["map_order/order"] = np.array([ref.map_order(int(t)) for t in MAP_ORDER_STEPS], np.int32)

    path = os.path.join(HERE, "grid_sp.npz")
    np.savez_compressed(path, **out)
    return path


if __name__ == "__main__":
    print(make())
