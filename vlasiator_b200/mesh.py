"""Velocity mesh description and block-index helpers.

Mirrors the reference's ``vmesh::MeshParameters`` (velocity_mesh_parameters.h:53)
and the global-ID layout of ``vmesh::VelocityMesh``
(spatial_cells/velocity_mesh_cpu.h:253-290): a block's global ID is
``i + j*Nx + k*Nx*Ny`` and each block holds WID^3 = 64 phase-space cells stored
``x`` fastest (``cellIndex(i,j,k) = k*16 + j*4 + i``, common.h:514).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

WID = 4
WID2 = WID * WID
WID3 = WID2 * WID

# physicalconstants (common.h:559-567)
K_B = 1.3806503e-23
CHARGE = 1.60217653e-19
MASS_PROTON = 1.67262158e-27
MU_0 = 1.25663706e-6


@dataclass(frozen=True)
class VelocityMesh:
    """Bounding box [vmin, vmax] (m/s) split into ``length`` blocks per axis."""

    vmin: tuple = (-4.02e6, -4.02e6, -4.02e6)
    vmax: tuple = (4.02e6, 4.02e6, 4.02e6)
    length: tuple = (67, 67, 67)

    @property
    def dv(self) -> np.ndarray:
        """Cell size per axis, computed as (max-min)/length/WID like initVelocityMeshes."""
        return np.array([(self.vmax[d] - self.vmin[d]) / self.length[d] / WID for d in range(3)])

    @property
    def block_size(self) -> np.ndarray:
        return np.array([(self.vmax[d] - self.vmin[d]) / self.length[d] for d in range(3)])

    @property
    def max_blocks(self) -> int:
        return int(self.length[0]) * int(self.length[1]) * int(self.length[2])

    def gid(self, i, j, k):
        return np.asarray(i) + self.length[0] * (np.asarray(j) + self.length[1] * np.asarray(k))

    def indices(self, gid):
        gid = np.asarray(gid, dtype=np.int64)
        i = gid % self.length[0]
        j = (gid // self.length[0]) % self.length[1]
        k = gid // (self.length[0] * self.length[1])
        return i, j, k

    def cell_centres(self, gids):
        """Velocity coordinates of the 64 cell centres of each block, [nb, 64] per axis."""
        bi, bj, bk = self.indices(gids)
        c = np.arange(WID3)
        ci, cj, ck = c % WID, (c // WID) % WID, c // WID2
        dv = self.dv
        bs = self.block_size
        vx = self.vmin[0] + bi[:, None] * bs[0] + (ci[None, :] + 0.5) * dv[0]
        vy = self.vmin[1] + bj[:, None] * bs[1] + (cj[None, :] + 0.5) * dv[1]
        vz = self.vmin[2] + bk[:, None] * bs[2] + (ck[None, :] + 0.5) * dv[2]
        return vx, vy, vz


class CMesh(ctypes.Structure):
    """C layout shared by the C ABI (include/vlgpu.h ``vlgpu_mesh``) and the oracle."""

    _fields_ = [("vmin", ctypes.c_double * 3), ("vmax", ctypes.c_double * 3), ("len", ctypes.c_uint32 * 3)]

    @classmethod
    def of(cls, mesh: VelocityMesh) -> "CMesh":
        m = cls()
        for d in range(3):
            m.vmin[d] = mesh.vmin[d]
            m.vmax[d] = mesh.vmax[d]
            m.len[d] = mesh.length[d]
        return m
