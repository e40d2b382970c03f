"""ctypes bindings for the parity oracle (test infrastructure only).

Two back ends:

* ``Restatement`` -- ``oracle/liborc_{sp,dp}.so`` built from vlasov_oracle.c,
  the plain-C restatement of the reference's algorithm.
* ``ReferenceBuild`` -- ``oracle/_ref/libvlasov_ref_{sp,dp}.so`` built by
  oracle/build_ref.sh from the reference's own sources; present only where the
  reference tree was available at build time.

Only tests, the smoke check and bench.py's CPU-baseline leg import this.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from vlasiator_b200.grid import grid_neighbors
from vlasiator_b200.mesh import WID3, CMesh, VelocityMesh

HERE = os.path.dirname(os.path.abspath(__file__))
_u32p = ctypes.POINTER(ctypes.c_uint32)
_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p


def _ptr(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def reference_root() -> str:
    """The Vlasiator source tree the reference build reads: $VLASIATOR_REF, else /root/reference."""
    return os.environ.get("VLASIATOR_REF", "/root/reference")


def build(with_reference: bool = False) -> None:
    """Compiles the restatement (and, if asked and available, the reference build)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    ref = reference_root()
    if with_reference and os.path.isdir(os.path.join(ref, "vlasovsolver")):
        subprocess.run([os.path.join(HERE, "build_ref.sh"), ref], check=True, stdout=subprocess.DEVNULL)


class Restatement:
    def __init__(self, precision: str = "sp"):
        path = os.path.join(HERE, f"liborc_{precision}.so")
        if not os.path.exists(path):
            build()
        self.lib = ctypes.CDLL(path)
        self.realf = np.float32 if precision == "sp" else np.float64
        ct = ctypes.c_float if precision == "sp" else ctypes.c_double
        self._ct = ct
        L = self.lib
        L.orc_map_1d.restype = ctypes.c_int
        L.orc_map_1d.argtypes = [ctypes.POINTER(CMesh), ctypes.c_uint32, _u32p, ctypes.POINTER(ct), ctypes.c_double,
                                 ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_uint32, ctypes.c_double,
                                 ctypes.c_uint32, ctypes.c_uint32, _u32p, _u32p, ctypes.POINTER(ct), _u32p]
        L.orc_acceleration_transform.restype = None
        L.orc_acceleration_transform.argtypes = [_dp, _dp, ctypes.c_double, _dp, _dp, ctypes.c_double,
                                                 ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                                 ctypes.c_double, _dp, _dp]
        L.orc_cell_intersections.restype = None
        L.orc_cell_intersections.argtypes = [_dp, _dp, ctypes.POINTER(CMesh), ctypes.c_uint32, _dp]
        L.orc_moments.restype = None
        L.orc_moments.argtypes = [ctypes.POINTER(CMesh), ctypes.c_uint32, _u32p, ctypes.POINTER(ct), ctypes.c_double,
                                  ctypes.c_double, ctypes.c_int, _dp]
        L.orc_translate.restype = ctypes.c_int
        L.orc_translate.argtypes = [ctypes.POINTER(CMesh), _u32p, ctypes.POINTER(ctypes.c_uint64), _u32p,
                                    ctypes.POINTER(ct), ctypes.c_uint32, ct, ct, ctypes.c_double, ctypes.POINTER(ct)]
        L.orc_adjust.restype = ctypes.c_int
        L.orc_adjust.argtypes = [ctypes.POINTER(CMesh), ctypes.c_uint32, _u32p, ctypes.POINTER(ct), ctypes.c_double,
                                 ctypes.c_int, ctypes.c_uint32, _u32p, _u32p, ctypes.POINTER(ct), _dp]
        L.orc_adjust_with.restype = ctypes.c_int
        L.orc_adjust_with.argtypes = [ctypes.POINTER(CMesh), ctypes.c_uint32, _u32p, ctypes.POINTER(ct),
                                      ctypes.c_double, ctypes.c_int, ctypes.c_uint32, _u32p, ctypes.c_uint32, _u32p,
                                      _u32p, ctypes.POINTER(ct), _dp]
        L.orc_content_gids.restype = ctypes.c_uint32
        L.orc_content_gids.argtypes = [ctypes.c_uint32, _u32p, ctypes.POINTER(ct), ctypes.c_double, _u32p]

    def map_1d(self, mesh: VelocityMesh, gids, data, isect4, dim: int, min_value: float, wall_margin: int = 1,
               cap: int | None = None):
        gids = np.ascontiguousarray(gids, dtype=np.uint32)
        data = np.ascontiguousarray(data, dtype=self.realf).reshape(-1, WID3)
        cap = cap or max(4 * len(gids) + 4096, 8192)
        go = np.zeros(cap, np.uint32)
        do = np.zeros((cap, WID3), self.realf)
        n = ctypes.c_uint32(0)
        fl = ctypes.c_uint32(0)
        cm = CMesh.of(mesh)
        rc = self.lib.orc_map_1d(ctypes.byref(cm), len(gids), _ptr(gids, ctypes.c_uint32), _ptr(data, self._ct),
                                 float(isect4[0]), float(isect4[1]), float(isect4[2]), float(isect4[3]), dim,
                                 float(min_value), wall_margin, cap, ctypes.byref(n), _ptr(go, ctypes.c_uint32),
                                 _ptr(do, self._ct), ctypes.byref(fl))
        if rc != 0:
            raise RuntimeError(f"orc_map_1d failed with status {rc}")
        return go[: n.value].copy(), do[: n.value].copy(), fl.value

    def moments(self, mesh: VelocityMesh, gids, data, mass, charge, second=True):
        gids = np.ascontiguousarray(gids, dtype=np.uint32)
        data = np.ascontiguousarray(data, dtype=self.realf).reshape(-1, WID3)
        out = np.zeros(16)
        cm = CMesh.of(mesh)
        self.lib.orc_moments(ctypes.byref(cm), len(gids), _ptr(gids, ctypes.c_uint32), _ptr(data, self._ct),
                             float(mass), float(charge), int(second), _ptr(out, ctypes.c_double))
        return out

    def adjust(self, mesh: VelocityMesh, gids, data, min_value, add_width=1):
        gids = np.ascontiguousarray(gids, dtype=np.uint32)
        data = np.ascontiguousarray(data, dtype=self.realf).reshape(-1, WID3)
        cap = max(30 * len(gids) + 64, 1024)
        go = np.zeros(cap, np.uint32)
        do = np.zeros((cap, WID3), self.realf)
        n = ctypes.c_uint32(0)
        loss = ctypes.c_double(0)
        cm = CMesh.of(mesh)
        rc = self.lib.orc_adjust(ctypes.byref(cm), len(gids), _ptr(gids, ctypes.c_uint32), _ptr(data, self._ct),
                                 float(min_value), int(add_width), cap, ctypes.byref(n), _ptr(go, ctypes.c_uint32),
                                 _ptr(do, self._ct), ctypes.byref(loss))
        if rc != 0:
            raise RuntimeError(f"orc_adjust failed with status {rc}")
        return go[: n.value].copy(), do[: n.value].copy(), loss.value

    def content_gids(self, gids, data, min_value):
        gids = np.ascontiguousarray(gids, dtype=np.uint32)
        data = np.ascontiguousarray(data, dtype=self.realf).reshape(-1, WID3)
        out = np.zeros(max(len(gids), 1), np.uint32)
        k = self.lib.orc_content_gids(len(gids), _ptr(gids, ctypes.c_uint32), _ptr(data, self._ct),
                                      float(min_value), _ptr(out, ctypes.c_uint32))
        return out[:k].copy()

    def adjust_grid(self, mesh: VelocityMesh, grid, cells, min_value, add_width=1):
        """adjustVelocityBlocks (grid.cpp:775-817) over a uniform periodic grid:
        content lists of every cell first, then each cell adjusted with the
        content of its 26 nearest neighbours.  cells: [(gids, data)] x fastest.
        Returns [(gids sorted, data)], loss per cell."""
        content = [self.content_gids(g, d, min_value) for g, d in cells]
        nbrs = grid_neighbors(grid)
        out, losses = [], []
        cm = CMesh.of(mesh)
        for c, (g, d) in enumerate(cells):
            extra = np.unique(np.concatenate([content[n] for n in nbrs[c] if n >= 0] + [np.zeros(0, np.uint32)]))
            extra = np.ascontiguousarray(extra, np.uint32)
            g = np.ascontiguousarray(g, np.uint32)
            d = np.ascontiguousarray(d, self.realf).reshape(-1, WID3)
            cap = max(30 * len(g) + len(extra) + 64, 1024)
            go = np.zeros(cap, np.uint32)
            do = np.zeros((cap, WID3), self.realf)
            n = ctypes.c_uint32(0)
            loss = ctypes.c_double(0)
            rc = self.lib.orc_adjust_with(ctypes.byref(cm), len(g), _ptr(g, ctypes.c_uint32), _ptr(d, self._ct),
                                          float(min_value), int(add_width), len(extra),
                                          _ptr(extra, ctypes.c_uint32), cap, ctypes.byref(n),
                                          _ptr(go, ctypes.c_uint32), _ptr(do, self._ct), ctypes.byref(loss))
            if rc != 0:
                raise RuntimeError(f"orc_adjust_with failed with status {rc}")
            out.append((go[: n.value].copy(), do[: n.value].copy()))
            losses.append(loss.value)
        return out, np.array(losses)

    def translate(self, mesh: VelocityMesh, grid, offsets, gids, data, dim, dt, dz, min_value=1e-15):
        """One spatial dimension of the translation of a uniform periodic grid (cells x fastest)."""
        g3 = np.ascontiguousarray(grid, np.uint32)
        offs = np.ascontiguousarray(offsets, np.uint64)
        gids = np.ascontiguousarray(gids, np.uint32)
        data = np.ascontiguousarray(data, self.realf).reshape(-1, WID3)
        out = np.zeros_like(data)
        cm = CMesh.of(mesh)
        rc = self.lib.orc_translate(ctypes.byref(cm), _ptr(g3, ctypes.c_uint32), _ptr(offs, ctypes.c_uint64),
                                    _ptr(gids, ctypes.c_uint32), _ptr(data, self._ct), dim, self._ct(dt),
                                    self._ct(dz), float(min_value), _ptr(out, self._ct))
        if rc != 0:
            raise RuntimeError(f"orc_translate failed with status {rc}")
        return out

    def accelerate_step(self, mesh: VelocityMesh, gids, data, B, dt, map_order, mass, charge, min_value=1e-15,
                        add_width=1, hall_min_rhoq=1.60217653e-19, mu0=1.25663706e-6):
        """One acceleration step of one cell as the reference's calculateAcceleration
        does it for one subcycle: moments -> transform -> intersections -> three
        map_1d -> block adjustment -> moments with pressure."""
        m0 = self.moments(mesh, gids, data, mass, charge, second=False)
        L, t = self.acceleration_transform(B, np.zeros(3), m0[8], m0[5:8], np.zeros(3), charge, mass, dt,
                                           hall_min_rhoq, 0, mu0)
        isect = self.cell_intersections(L, t, mesh, map_order)
        g, d = gids, data
        wall = 0
        for dim in [[0, 1, 2], [1, 2, 0], [2, 0, 1]][map_order]:
            g, d, fl = self.map_1d(mesh, g, d, isect[4 * dim:4 * dim + 4], dim, min_value)
            wall |= fl
        g, d, loss = self.adjust(mesh, g, d, min_value, add_width)
        m1 = self.moments(mesh, g, d, mass, charge, second=True)
        return g, d, isect, loss, m1, wall

    def vlasov_step(self, mesh: VelocityMesh, grid, cells, B, dt, map_order, dx, mass, charge, min_value=1e-15,
                    add_width=1, hall_min_rhoq=1.60217653e-19, mu0=1.25663706e-6):
        """One Vlasov step of a uniform periodic grid in the reference's main-loop
        order: calculateSpatialTranslation (vlasovmover.cpp:65-381: z, x, y, then
        calculateMoments_R), then calculateAcceleration for one subcycle
        (vlasovmover.cpp:410-475: moments_V, transform, intersections, three
        map_1d per cell) and its final adjustVelocityBlocks with the spatial
        neighbours plus calculateMoments_V (vlasovmover.cpp:564-569).
        cells: [(gids, data)] x fastest.  Returns (cells sorted by GID, loss per
        cell, moments_R, moments_V, intersections)."""
        state = [(np.asarray(g, np.uint32), np.asarray(d, self.realf).reshape(-1, WID3)) for g, d in cells]
        for dim in (2, 0, 1):
            offs = np.zeros(len(state) + 1, np.uint64)
            offs[1:] = np.cumsum([len(g) for g, _ in state])
            out = self.translate(mesh, grid, offs, np.concatenate([g for g, _ in state]),
                                 np.concatenate([d for _, d in state]), dim, dt, dx[dim], min_value)
            state = [(g, out[offs[c]:offs[c + 1]]) for c, (g, _) in enumerate(state)]
        mom_r = np.stack([self.moments(mesh, g, d, mass, charge, second=True) for g, d in state])
        adjusted, loss, mom_v, isects = self.accelerate_grid(mesh, grid, state, B, dt, map_order, mass, charge,
                                                             min_value, add_width, hall_min_rhoq, mu0)
        return adjusted, loss, mom_r, mom_v, isects

    def accelerate_grid(self, mesh: VelocityMesh, grid, cells, B, dt, map_order, mass, charge, min_value=1e-15,
                        add_width=1, hall_min_rhoq=1.60217653e-19, mu0=1.25663706e-6):
        """calculateAcceleration of a uniform periodic grid for one subcycle
        (vlasovmover.cpp:410-475: moments_V, transform, intersections, three
        map_1d per cell), its final adjustVelocityBlocks with the spatial
        neighbours and calculateMoments_V (vlasovmover.cpp:564-569).
        cells: [(gids, data)] x fastest.  Returns (cells sorted by GID, loss
        per cell, moments_V, intersections)."""
        state = [(np.asarray(g, np.uint32), np.asarray(d, self.realf).reshape(-1, WID3)) for g, d in cells]
        swept, isects = [], []
        for c, (g, d) in enumerate(state):
            m0 = self.moments(mesh, g, d, mass, charge, second=False)
            L, t = self.acceleration_transform(B[c], np.zeros(3), m0[8], m0[5:8], np.zeros(3), charge, mass, dt,
                                               hall_min_rhoq, 0, mu0)
            isect = self.cell_intersections(L, t, mesh, map_order)
            for dim in [[0, 1, 2], [1, 2, 0], [2, 0, 1]][map_order]:
                g, d, _ = self.map_1d(mesh, g, d, isect[4 * dim:4 * dim + 4], dim, min_value)
            swept.append((g, d))
            isects.append(isect)
        adjusted, loss = self.adjust_grid(mesh, grid, swept, min_value, add_width)
        mom_v = np.stack([self.moments(mesh, g, d, mass, charge, second=True) for g, d in adjusted])
        return adjusted, loss, mom_v, np.stack(isects)

    def acceleration_transform(self, B, curl, rhoq, V, egradpe, q, m, dt, hall_min_rhoq, ohm_gradpe, mu0):
        L = np.zeros(9)
        t = np.zeros(3)
        B = np.ascontiguousarray(B, dtype=np.float64)
        curl = np.ascontiguousarray(curl, dtype=np.float64)
        V = np.ascontiguousarray(V, dtype=np.float64)
        eg = np.ascontiguousarray(egradpe, dtype=np.float64)
        self.lib.orc_acceleration_transform(_ptr(B, ctypes.c_double), _ptr(curl, ctypes.c_double), float(rhoq),
                                            _ptr(V, ctypes.c_double), _ptr(eg, ctypes.c_double), float(q), float(m),
                                            float(dt), float(hall_min_rhoq), int(ohm_gradpe), float(mu0),
                                            _ptr(L, ctypes.c_double), _ptr(t, ctypes.c_double))
        return L.reshape(3, 3), t

    def cell_intersections(self, L, t, mesh: VelocityMesh, map_order: int):
        L = np.ascontiguousarray(L, dtype=np.float64).reshape(9)
        t = np.ascontiguousarray(t, dtype=np.float64)
        out = np.zeros(12)
        cm = CMesh.of(mesh)
        self.lib.orc_cell_intersections(_ptr(L, ctypes.c_double), _ptr(t, ctypes.c_double), ctypes.byref(cm),
                                        map_order, _ptr(out, ctypes.c_double))
        return out


def reference_available(precision: str = "sp") -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", f"libvlasov_ref_{precision}.so"))


class ReferenceBuild:
    """The reference's own map_1d and moment templates, driven through oracle/ref_harness.cpp."""

    _mesh_set = {}

    def __init__(self, precision: str = "sp"):
        """precision: "sp" / "dp" (PPM), or "sp_pqm" / "sp_plm" for the
        reference's other acceleration reconstructions (FP32)."""
        path = os.path.join(HERE, "_ref", f"libvlasov_ref_{precision}.so")
        self.lib = ctypes.CDLL(path)
        sp = precision.startswith("sp")
        self.realf = np.float32 if sp else np.float64
        ct = ctypes.c_float if sp else ctypes.c_double
        self._ct = ct
        L = self.lib
        L.ref_init.argtypes = [_dp, _dp, _u32p, ctypes.c_uint32]
        L.ref_cells_create.restype = _vp
        L.ref_cells_create.argtypes = [ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint64), _u32p, ctypes.POINTER(ct), _dp]
        L.ref_cells_destroy.argtypes = [_vp]
        L.ref_cells_count.restype = ctypes.c_uint32
        L.ref_cells_count.argtypes = [_vp]
        L.ref_cells_block_count.restype = ctypes.c_uint64
        L.ref_cells_block_count.argtypes = [_vp, ctypes.c_uint32]
        L.ref_cells_extract.restype = ctypes.c_uint64
        L.ref_cells_extract.argtypes = [_vp, ctypes.c_uint32, _u32p, ctypes.POINTER(ct), ctypes.c_uint64]
        L.ref_cells_map_1d.argtypes = [_vp, _dp, ctypes.c_uint32, ctypes.c_int]
        L.ref_cells_accelerate.argtypes = [_vp, _dp, ctypes.c_uint32, ctypes.c_int]
        L.ref_cells_moments.argtypes = [_vp, ctypes.c_uint32, _dp, _dp, _dp]
        L.ref_bailouts.restype = ctypes.c_int
        L.ref_cells_accelerate_step.argtypes = [_vp, _dp, _dp, ctypes.c_uint32, ctypes.c_double, ctypes.c_double,
                                                ctypes.c_int]
        L.ref_max_threads.restype = ctypes.c_int
        L.ref_cells_translate.argtypes = [_vp, _u32p, ctypes.c_uint32, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_int]
        L.ref_cells_adjust.argtypes = [_vp, ctypes.POINTER(ctypes.c_int32), ctypes.c_uint32, ctypes.c_double,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp]
        L.ref_cells_max_r_dt.restype = ctypes.c_double
        L.ref_cells_max_r_dt.argtypes = [_vp, _dp, _dp]
        L.ref_cells_full_step.argtypes = [_vp, _dp, _dp, ctypes.c_uint32, ctypes.c_double, ctypes.c_double,
                                          ctypes.POINTER(ctypes.c_int32), ctypes.c_uint32, ctypes.c_int, _dp]
        L.ref_cells_vlasov_step.argtypes = [_vp, _u32p, _dp, _dp, ctypes.c_double, ctypes.c_uint32, ctypes.c_double,
                                            ctypes.c_double, ctypes.POINTER(ctypes.c_int32), ctypes.c_uint32,
                                            ctypes.c_int, _dp, _dp]
        L.ref_map_order.restype = ctypes.c_uint32
        L.ref_map_order.argtypes = [ctypes.c_uint32]
        L.ref_cells_content.restype = ctypes.c_uint64
        L.ref_cells_content.argtypes = [_vp, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint8), ctypes.c_uint64]
        L.ref_fill_blocks.argtypes = [ctypes.c_uint64, _u32p, _dp, ctypes.c_double, _dp, ctypes.c_double,
                                      ctypes.c_double, ctypes.POINTER(ct)]

    def init(self, mesh: VelocityMesh, wall_margin: int = 1):
        vmin = np.array(mesh.vmin, np.float64)
        vmax = np.array(mesh.vmax, np.float64)
        ln = np.array(mesh.length, np.uint32)
        self.lib.ref_init(_ptr(vmin, ctypes.c_double), _ptr(vmax, ctypes.c_double), _ptr(ln, ctypes.c_uint32),
                          wall_margin)

    def create(self, gid_list, data_list, min_values):
        offs = np.zeros(len(gid_list) + 1, np.uint64)
        offs[1:] = np.cumsum([len(g) for g in gid_list])
        gids = np.ascontiguousarray(np.concatenate(gid_list).astype(np.uint32))
        data = np.ascontiguousarray(np.concatenate([d.reshape(-1, WID3) for d in data_list]).astype(self.realf))
        mv = np.ascontiguousarray(np.asarray(min_values, np.float64))
        return self.lib.ref_cells_create(len(gid_list), _ptr(offs, ctypes.c_uint64), _ptr(gids, ctypes.c_uint32),
                                         _ptr(data, self._ct), _ptr(mv, ctypes.c_double))

    def destroy(self, h):
        self.lib.ref_cells_destroy(h)

    def fill_blocks(self, gids, V, T, rho, mass, T_aniso=None):
        """The projects' initial fill of the given blocks (the Maxwellian, or
        with T_aniso = (Tx, Ty, Tz) the axis-aligned tri-Maxwellian, of
        projects/project.h:45-73 at the cell centres); (n_blocks, 64)."""
        g = np.ascontiguousarray(gids, np.uint32)
        v = np.ascontiguousarray(V, np.float64)
        ta = None if T_aniso is None else np.ascontiguousarray(T_aniso, np.float64)
        out = np.zeros((len(g), WID3), self.realf)
        self.lib.ref_fill_blocks(len(g), _ptr(g, ctypes.c_uint32), _ptr(v, ctypes.c_double), float(T),
                                 None if ta is None else _ptr(ta, ctypes.c_double), float(rho), float(mass),
                                 _ptr(out, self._ct))
        return out

    def extract(self, h, c, sort=True):
        n = self.lib.ref_cells_block_count(h, c)
        g = np.zeros(max(n, 1), np.uint32)
        d = np.zeros((max(n, 1), WID3), self.realf)
        self.lib.ref_cells_extract(h, c, _ptr(g, ctypes.c_uint32), _ptr(d, self._ct), n)
        g, d = g[:n], d[:n]
        if sort:
            o = np.argsort(g, kind="stable")
            g, d = g[o], d[o]
        return g, d

    def map_1d(self, h, isect, dim, nthreads=0):
        isect = np.ascontiguousarray(isect, np.float64)
        self.lib.ref_cells_map_1d(h, _ptr(isect, ctypes.c_double), dim, nthreads)

    def accelerate(self, h, isect12, map_order, nthreads=0):
        isect12 = np.ascontiguousarray(isect12, np.float64)
        self.lib.ref_cells_accelerate(h, _ptr(isect12, ctypes.c_double), map_order, nthreads)

    def accelerate_step(self, h, B, dt, map_order, charge, mass, nthreads=0):
        B = np.ascontiguousarray(B, np.float64)
        dt = np.ascontiguousarray(dt, np.float64)
        self.lib.ref_cells_accelerate_step(h, _ptr(B, ctypes.c_double), _ptr(dt, ctypes.c_double), map_order,
                                           charge, mass, nthreads)

    def translate(self, h, grid, dim, dt, dz, nthreads=0):
        g = np.ascontiguousarray(grid, np.uint32)
        self.lib.ref_cells_translate(h, _ptr(g, ctypes.c_uint32), dim, float(dt), float(dz), nthreads)

    def max_threads(self) -> int:
        return self.lib.ref_max_threads()

    def moments(self, h, c, bulk_v):
        bv = np.ascontiguousarray(bulk_v, np.float64)
        f = np.zeros(4)
        s = np.zeros(6)
        self.lib.ref_cells_moments(h, c, _ptr(bv, ctypes.c_double), _ptr(f, ctypes.c_double),
                                   _ptr(s, ctypes.c_double))
        return f, s

    def adjust(self, h, n_cells, min_value, add_width=1, neighbors=None, conserve_mass=False, nthreads=0):
        """adjustVelocityBlocks (grid.cpp:775-817) with the reference's own
        content lists and adjust_velocity_blocks on every cell of the set;
        neighbors: (n_cells, k) cell indices (-1: none) or None.  Returns the
        RHOLOSSADJUST each cell gained."""
        loss = np.zeros(n_cells)
        if neighbors is None:
            nb, k = None, 0
        else:
            nbr = np.ascontiguousarray(neighbors, np.int32)
            nb, k = _ptr(nbr, ctypes.c_int32), nbr.shape[1]
        self.lib.ref_cells_adjust(h, nb, k, float(min_value), int(add_width), int(conserve_mass), nthreads,
                                  _ptr(loss, ctypes.c_double))
        return loss

    def max_r_dt(self, h, dx):
        """reduce_vlasov_dt (arch_dt.cpp:33-97) over the set: each cell's MAXRDT
        and the minimum over the cells."""
        n = self.lib.ref_cells_count(h)
        out = np.zeros(n)
        d = np.ascontiguousarray(dx, np.float64)
        total = self.lib.ref_cells_max_r_dt(h, _ptr(d, ctypes.c_double), _ptr(out, ctypes.c_double))
        return out, total

    def full_step(self, h, B, dt, map_order, charge, mass, neighbors=None, nthreads=0, moments=False):
        """calculateAcceleration for one population and one subcycle on every
        cell: pivot moments, geometry, map_1d x3, adjustVelocityBlocks (with the
        given NEAREST neighbours, or none) and the moments with pressure.
        Returns (n_cells, 10) moments (n, nV, sum f (v-V)(v-V)) if asked."""
        B = np.ascontiguousarray(B, np.float64)
        dt = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, np.float64), (len(B),)))
        nb, k = self._neighbors(neighbors)
        out = np.zeros((len(B), 10)) if moments else None
        self.lib.ref_cells_full_step(h, _ptr(B, ctypes.c_double), _ptr(dt, ctypes.c_double), map_order, charge,
                                     mass, nb, k, nthreads, None if out is None else _ptr(out, ctypes.c_double))
        return out

    def vlasov_step(self, h, grid, dx, B, dt, map_order, charge, mass, neighbors, nthreads=0, moments=False):
        """One full Vlasov step of the periodic grid: translation z, x, y, the _R
        moments, then full_step with the spatial neighbours.  With moments=True
        returns ((n_cells, 10) moments as full_step, the RHOLOSSADJUST each cell
        gained in the step)."""
        g = np.ascontiguousarray(grid, np.uint32)
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dx, np.float64), (3,)))
        B = np.ascontiguousarray(B, np.float64)
        nb, k = self._neighbors(neighbors)
        out = np.zeros((len(B), 10)) if moments else None
        loss = np.zeros(len(B)) if moments else None
        self.lib.ref_cells_vlasov_step(h, _ptr(g, ctypes.c_uint32), _ptr(d, ctypes.c_double),
                                       _ptr(B, ctypes.c_double), float(dt), map_order, charge, mass, nb, k,
                                       nthreads, None if out is None else _ptr(out, ctypes.c_double),
                                       None if loss is None else _ptr(loss, ctypes.c_double))
        return (out, loss) if moments else None

    def _neighbors(self, neighbors):
        if neighbors is None:
            return None, 0
        self._nbr = np.ascontiguousarray(neighbors, np.int32)
        return _ptr(self._nbr, ctypes.c_int32), self._nbr.shape[1]

    def map_order(self, tstep: int) -> int:
        """The dimension order the reference draws for time step tstep (vlasovmover.cpp:422-426)."""
        return int(self.lib.ref_map_order(int(tstep)))

    def content(self, h, c):
        """compute_block_has_content of cell c's blocks, in local-ID order."""
        n = self.lib.ref_cells_block_count(h, c)
        f = np.zeros(max(n, 1), np.uint8)
        self.lib.ref_cells_content(h, c, _ptr(f, ctypes.c_uint8), n)
        return f[:n].astype(bool)

    def bailouts(self) -> int:
        return self.lib.ref_bailouts()
