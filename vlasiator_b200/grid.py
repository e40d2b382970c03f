"""Uniform periodic spatial grids of cells, as the batch's translation and
block adjustment see them.

Cells are numbered x fastest, cell = x + nx*(y + ny*z), as dccrg numbers the
cells of a uniform grid (minus its 1-based offset).  A pencil along dimension d
is the line of cells through one transverse position; its cells wrap around
periodically (the configs' periodic boundaries).
"""
from __future__ import annotations

import numpy as np


def cell_index(dims, x, y, z):
    nx, ny, _ = dims
    return x + nx * (y + ny * z)


def grid_neighbors(dims) -> np.ndarray:
    """The 26 nearest neighbours of every cell (Neighborhoods::NEAREST,
    grid.cpp:979-997), periodic; entries equal to the cell itself are -1, as
    adjust_velocity_blocks_in_cells excludes the cell from its neighbour list
    (spatial_cells/block_adjust_cpu.cpp:84-90).  Shape (n_cells, 26), int32."""
    nx, ny, nz = (int(v) for v in dims)
    n = nx * ny * nz
    c = np.arange(n)
    x, y, z = c % nx, (c // nx) % ny, c // (nx * ny)
    out = np.empty((n, 26), np.int32)
    q = 0
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                if dx == 0 and dy == 0 and dz == 0:
                    continue
                nb = (x + dx) % nx + nx * (((y + dy) % ny) + ny * ((z + dz) % nz))
                out[:, q] = np.where(nb == c, -1, nb)
                q += 1
    return out
