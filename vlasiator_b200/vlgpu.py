"""Host-side binding of libvlgpu.so (the CUDA hot path) through its C ABI.

``Batch`` mirrors what the reference's solver drivers act on: a set of
spatial cells, each with one population's velocity mesh (block global IDs)
and block container (64 Realf per block).  Its methods map one to one onto
the reference's entry points for that data:

* ``map_1d(intersections, dim)``    -> map_1d per cell (vlasovsolver/cpu_acc_map.cpp:121)
* ``accelerate_with_intersections`` -> cpu_accelerate_cell (vlasovsolver/cpu_acc_semilag.cpp:92)

The library must be built for sm_100a (``python -m vlasiator_b200.build``);
there is no CPU fallback, and every call raises on a non-zero status.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .mesh import WID3, VelocityMesh

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvlgpu.so")

STATUS = {0: "VLGPU_OK", 1: "VLGPU_EINVAL", 2: "VLGPU_ENOMEM", 3: "VLGPU_EWALL", 4: "VLGPU_ETIMEDOUT",
          5: "VLGPU_ERANGE", 6: "VLGPU_ECUDA", 7: "VLGPU_ENODEV", 8: "VLGPU_EAGAIN", 9: "VLGPU_ENOENT"}
CELL_WALL, CELL_RANGE, CELL_NOMEM, CELL_BADDK = 1, 2, 4, 8


class VlgpuError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what}: {STATUS.get(code, code)}")
        self.code = code


class CMeshT(ctypes.Structure):
    _fields_ = [("vmin", ctypes.c_double * 3), ("vmax", ctypes.c_double * 3), ("len", ctypes.c_uint32 * 3)]


class CParamsT(ctypes.Structure):
    _fields_ = [("charge", ctypes.c_double), ("mass", ctypes.c_double), ("min_value", ctypes.c_double),
                ("add_width_v", ctypes.c_uint32), ("wall_margin", ctypes.c_uint32),
                ("hall_minimum_rhoq", ctypes.c_double), ("ohm_gradpe", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]


class CMaxwellianT(ctypes.Structure):
    _fields_ = [("n", ctypes.c_double), ("T", ctypes.c_double * 3), ("frame", ctypes.c_double * 9),
                ("V", ctypes.c_double * 3)]


class CFieldsT(ctypes.Structure):
    _fields_ = [("B", ctypes.c_double * 3), ("curl", ctypes.c_double * 3), ("egradpe", ctypes.c_double * 3)]


_lib = None

# every symbol include/vlgpu.h declares, with its ctypes signature
class CLaunchT(ctypes.Structure):
    """vlgpu_launch: CTAs per SM of the remap, moments, adjustment and translation kernels (0 = maximum)."""
    _fields_ = [("remap_ctas_per_sm", ctypes.c_uint32), ("moments_ctas_per_sm", ctypes.c_uint32),
                ("adjust_ctas_per_sm", ctypes.c_uint32), ("translate_ctas_per_sm", ctypes.c_uint32)]

    def as_tuple(self):
        return (self.remap_ctas_per_sm, self.moments_ctas_per_sm, self.adjust_ctas_per_sm,
                self.translate_ctas_per_sm)


_vp = ctypes.c_void_p
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)
SIGNATURES = {
    "vlgpu_batch_create": (ctypes.c_int, [ctypes.POINTER(CMeshT), ctypes.POINTER(CParamsT), ctypes.c_uint32,
                                          ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(_vp)]),
    "vlgpu_batch_destroy": (ctypes.c_int, [_vp]),
    "vlgpu_batch_upload": (ctypes.c_int, [_vp, _u64p, _u32p, _fp]),
    "vlgpu_batch_block_counts": (ctypes.c_int, [_vp, _u32p]),
    "vlgpu_batch_download": (ctypes.c_int, [_vp, _u64p, _u32p, _fp, ctypes.c_uint64]),
    "vlgpu_batch_status": (ctypes.c_int, [_vp, _u32p]),
    "vlgpu_batch_pack_cells": (ctypes.c_int, [_vp, ctypes.c_uint32, _u32p, _u32p, _vp, _vp, ctypes.c_uint64,
                                              _u64p]),
    "vlgpu_batch_unpack_cells": (ctypes.c_int, [_vp, ctypes.c_uint32, _u32p, _u32p, _vp, _vp]),
    "vlgpu_map_1d": (ctypes.c_int, [_vp, _dp, ctypes.c_uint32]),
    "vlgpu_map_1d_per_cell": (ctypes.c_int, [_vp, _dp, ctypes.c_uint32]),
    "vlgpu_accelerate_with_intersections": (ctypes.c_int, [_vp, _dp, ctypes.c_uint32]),
    "vlgpu_accelerate": (ctypes.c_int, [_vp, ctypes.POINTER(CFieldsT), _dp, ctypes.c_uint32]),
    "vlgpu_accelerate_device": (ctypes.c_int, [_vp, ctypes.c_uint32]),
    "vlgpu_compute_intersections": (ctypes.c_int, [_vp, ctypes.POINTER(CFieldsT), _dp, ctypes.c_uint32]),
    "vlgpu_accelerate_per_cell": (ctypes.c_int, [_vp, ctypes.c_uint32]),
    "vlgpu_adjust_blocks": (ctypes.c_int, [_vp]),
    "vlgpu_batch_rho_loss": (ctypes.c_int, [_vp, _dp]),
    "vlgpu_batch_moments": (ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    "vlgpu_batch_intersections": (ctypes.c_int, [_vp, _dp]),
    "vlgpu_batch_stream": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "vlgpu_batch_profile": (ctypes.c_int, [_vp, ctypes.c_int]),
    "vlgpu_batch_stats": (ctypes.c_int, [_vp, _u64p]),
    "vlgpu_batch_stats2": (ctypes.c_int, [_vp, _u64p]),
    "vlgpu_batch_download_raw": (ctypes.c_int, [_vp, _u32p, _u32p, _u32p, _fp, ctypes.c_uint64, _u64p]),
    "vlgpu_batch_sync": (ctypes.c_int, [_vp]),
    "vlgpu_batch_upload_async": (ctypes.c_int, [_vp, _u64p, _u32p, _fp]),
    "vlgpu_batch_download_begin": (ctypes.c_int, [_vp]),
    "vlgpu_batch_download_end": (ctypes.c_int, [_vp, _u32p, _u32p, _u32p, _fp, ctypes.c_uint64, _u64p]),
    "vlgpu_batch_set_exact": (ctypes.c_int, [_vp, ctypes.c_int]),
    "vlgpu_batch_set_reconstruction": (ctypes.c_int, [_vp, ctypes.c_int]),
    "vlgpu_batch_capture": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_uint32, _u32p, ctypes.c_double]),
    "vlgpu_batch_replay": (ctypes.c_int, [_vp, ctypes.c_int]),
    "vlgpu_batch_set_grid": (ctypes.c_int, [_vp, _u32p, _dp]),
    "vlgpu_translate": (ctypes.c_int, [_vp, ctypes.c_uint32, ctypes.c_double]),
    "vlgpu_batch_max_dt": (ctypes.c_int, [_vp, ctypes.c_double, _dp, _dp]),
    "vlgpu_vlasov_step": (ctypes.c_int, [_vp, ctypes.POINTER(CFieldsT), ctypes.c_double, ctypes.c_uint32]),
    "vlgpu_vlasov_step_device": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_uint32]),
    "vlgpu_batch_moments_r": (ctypes.c_int, [_vp, _dp]),
    "vlgpu_batch_interpolated_moments": (ctypes.c_int, [_vp, _dp]),
    "vlgpu_batch_fill_maxwellian": (ctypes.c_int, [_vp, ctypes.POINTER(CMaxwellianT)]),
    "vlgpu_server_create": (ctypes.c_int, [ctypes.POINTER(CMeshT), ctypes.POINTER(CParamsT), ctypes.c_uint32,
                                           ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(_vp)]),
    "vlgpu_server_destroy": (ctypes.c_int, [_vp]),
    "vlgpu_server_submit": (ctypes.c_int, [_vp, ctypes.c_uint32, _u32p, _fp, ctypes.POINTER(CFieldsT),
                                           ctypes.c_double, ctypes.c_uint32, _u64p]),
    "vlgpu_server_tick": (ctypes.c_int, [_vp, _u32p, _u32p, _u32p]),
    "vlgpu_server_result": (ctypes.c_int, [_vp, ctypes.c_uint64, _u32p, _u32p, _fp, ctypes.c_uint64, _u32p, _dp]),
    "vlgpu_server_stats": (ctypes.c_int, [_vp, _u64p]),
    "vlgpu_server_batch": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "vlgpu_map_1d_noalloc": (ctypes.c_int, [ctypes.POINTER(CMeshT), ctypes.POINTER(CParamsT), ctypes.c_uint32, _u64p,
                                            _vp, _vp, _dp, ctypes.c_uint32, _vp, _vp, ctypes.c_uint64, _u32p, _u32p,
                                            _u32p, _vp]),
    "vlgpu_batch_set_launch": (ctypes.c_int, [_vp, ctypes.POINTER(CLaunchT)]),
    "vlgpu_batch_get_launch": (ctypes.c_int, [_vp, ctypes.POINTER(CLaunchT)]),
    "vlgpu_launch_table_lookup": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double,
                                                 ctypes.POINTER(CLaunchT)]),
    "vlgpu_version": (ctypes.c_char_p, []),
}


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads libvlgpu.so; raises if it has not been built (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: build it with `python -m vlasiator_b200.build`")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(code: int, what: str):
    if code != 0:
        raise VlgpuError(code, what)


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def make_params(charge=1.60217653e-19, mass=1.67262158e-27, min_value=1e-15, add_width_v=1, wall_margin=1,
                hall_minimum_rhoq=1.60217653e-19, ohm_gradpe=0) -> CParamsT:
    p = CParamsT()
    p.charge, p.mass, p.min_value = charge, mass, min_value
    p.add_width_v, p.wall_margin = add_width_v, wall_margin
    p.hall_minimum_rhoq, p.ohm_gradpe = hall_minimum_rhoq, ohm_gradpe
    return p


class Batch:
    """A device-resident batch of spatial cells (one population)."""

    def __init__(self, mesh: VelocityMesh, n_cells: int, capacity: int, params: CParamsT | None = None,
                 device: int = 0, exact: bool = False, recon: str = "ppm"):
        self.lib = load()
        self.mesh = mesh
        self.n_cells = int(n_cells)
        self.capacity = int(capacity)
        m = CMeshT()
        for d in range(3):
            m.vmin[d], m.vmax[d], m.len[d] = mesh.vmin[d], mesh.vmax[d], mesh.length[d]
        self.params = params or make_params()
        h = _vp()
        _check(self.lib.vlgpu_batch_create(ctypes.byref(m), ctypes.byref(self.params), self.n_cells, self.capacity,
                                           device, ctypes.byref(h)), "vlgpu_batch_create")
        self.h = h
        self.device = int(device)
        self._inflight = None  # host arrays an asynchronous upload still reads
        self.set_reconstruction(recon)
        self.set_exact(exact)

    def capture(self, slot: int, kind: str, map_orders, dt: float = 0.0):
        """Captures len(map_orders) (even) device steps, kind "accel" or "vlasov", into graph slot `slot`."""
        o = np.ascontiguousarray(map_orders, np.uint32)
        _check(self.lib.vlgpu_batch_capture(self.h, slot, {"accel": 0, "vlasov": 1}[kind], len(o),
                                            _p(o, ctypes.c_uint32), float(dt)), "vlgpu_batch_capture")

    def replay(self, slot: int):
        _check(self.lib.vlgpu_batch_replay(self.h, slot), "vlgpu_batch_replay")

    def set_reconstruction(self, recon: str):
        """"plm", "ppm" (default) or "pqm": the reference's ACC_SEMILAG_* choice."""
        order = {"plm": 1, "ppm": 2, "pqm": 4}[recon]
        _check(self.lib.vlgpu_batch_set_reconstruction(self.h, order), "vlgpu_batch_set_reconstruction")
        self.recon = recon

    def set_exact(self, exact: bool):
        """exact=True: bit-identical to the reference's map_1d; False: fused remap (1e-5 of peak)."""
        _check(self.lib.vlgpu_batch_set_exact(self.h, int(bool(exact))), "vlgpu_batch_set_exact")
        self.exact = bool(exact)

    def close(self):
        if getattr(self, "h", None):
            self.lib.vlgpu_batch_destroy(self.h)  # waits for the batch's stream
            self.h = None
        self._inflight = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- data movement ----
    def upload(self, gid_list, data_list):
        offs = np.zeros(self.n_cells + 1, np.uint64)
        offs[1:] = np.cumsum([len(g) for g in gid_list])
        gids = np.ascontiguousarray(np.concatenate(gid_list).astype(np.uint32))
        data = np.ascontiguousarray(np.concatenate([np.asarray(d, np.float32).reshape(-1, WID3) for d in data_list]))
        _check(self.lib.vlgpu_batch_upload(self.h, _p(offs, ctypes.c_uint64), _p(gids, ctypes.c_uint32),
                                           _p(data, ctypes.c_float)), "vlgpu_batch_upload")

    def upload_packed(self, offsets, gids, data):
        offs = np.ascontiguousarray(offsets, np.uint64)
        gids = np.ascontiguousarray(gids, np.uint32)
        data = np.ascontiguousarray(data, np.float32)
        _check(self.lib.vlgpu_batch_upload(self.h, _p(offs, ctypes.c_uint64), _p(gids, ctypes.c_uint32),
                                           _p(data, ctypes.c_float)), "vlgpu_batch_upload")

    def block_counts(self) -> np.ndarray:
        c = np.zeros(self.n_cells, np.uint32)
        _check(self.lib.vlgpu_batch_block_counts(self.h, _p(c, ctypes.c_uint32)), "vlgpu_batch_block_counts")
        return c

    def pack_cells(self, cells, gids_ptr: int, data_ptr: int, capacity: int):
        """The blocks of `cells` into device buffers (addresses on the batch's
        device: capacity uint32 IDs and capacity x 64 floats), cell after cell;
        returns (block count per cell, blocks written)."""
        c = np.ascontiguousarray(cells, np.uint32)
        counts = np.zeros(max(len(c), 1), np.uint32)
        used = ctypes.c_uint64(0)
        _check(self.lib.vlgpu_batch_pack_cells(self.h, len(c), _p(c, ctypes.c_uint32), _p(counts, ctypes.c_uint32),
                                               ctypes.c_void_p(gids_ptr), ctypes.c_void_p(data_ptr), int(capacity),
                                               ctypes.byref(used)), "vlgpu_batch_pack_cells")
        return counts[:len(c)], int(used.value)

    def unpack_cells(self, cells, counts, gids_ptr: int, data_ptr: int):
        """Replaces the blocks of `cells` with counts[i] blocks each, read cell
        after cell from device buffers (as pack_cells writes them)."""
        c = np.ascontiguousarray(cells, np.uint32)
        n = np.ascontiguousarray(counts, np.uint32)
        if len(c) != len(n):
            raise ValueError("cells and counts differ in length")
        _check(self.lib.vlgpu_batch_unpack_cells(self.h, len(c), _p(c, ctypes.c_uint32), _p(n, ctypes.c_uint32),
                                                 ctypes.c_void_p(gids_ptr), ctypes.c_void_p(data_ptr)),
               "vlgpu_batch_unpack_cells")

    def status(self) -> np.ndarray:
        s = np.zeros(self.n_cells, np.uint32)
        _check(self.lib.vlgpu_batch_status(self.h, _p(s, ctypes.c_uint32)), "vlgpu_batch_status")
        return s

    def download(self):
        """Returns (offsets, gids, data) with blocks sorted by GID inside each cell."""
        total = int(self.block_counts().astype(np.uint64).sum())
        offs = np.zeros(self.n_cells + 1, np.uint64)
        gids = np.zeros(max(total, 1), np.uint32)
        data = np.zeros((max(total, 1), WID3), np.float32)
        _check(self.lib.vlgpu_batch_download(self.h, _p(offs, ctypes.c_uint64), _p(gids, ctypes.c_uint32),
                                             _p(data, ctypes.c_float), max(total, 1)), "vlgpu_batch_download")
        return offs, gids[:total], data[:total]

    def download_raw(self, gids_out=None, data_out=None):
        """Unsorted copy of the current pool: (cell_off, cell_count, gids, data) views."""
        off = np.zeros(self.n_cells, np.uint32)
        cnt = np.zeros(self.n_cells, np.uint32)
        used = ctypes.c_uint64(0)
        if gids_out is None:
            gids_out = np.zeros(self.capacity, np.uint32)
            data_out = np.zeros((self.capacity, WID3), np.float32)
        _check(self.lib.vlgpu_batch_download_raw(self.h, _p(off, ctypes.c_uint32), _p(cnt, ctypes.c_uint32),
                                                 _p(gids_out, ctypes.c_uint32), _p(data_out, ctypes.c_float),
                                                 len(gids_out), ctypes.byref(used)), "vlgpu_batch_download_raw")
        u = int(used.value)
        return off, cnt, gids_out[:u], data_out[:u]

    def upload_async(self, offsets, gids, data):
        """Enqueues the upload; the arrays (pinned for overlap) are kept
        referenced here until the next sync."""
        offs = np.ascontiguousarray(offsets, np.uint64)
        gids = np.ascontiguousarray(gids, np.uint32)
        data = np.ascontiguousarray(data, np.float32)
        self._inflight = (offs, gids, data)
        _check(self.lib.vlgpu_batch_upload_async(self.h, _p(offs, ctypes.c_uint64), _p(gids, ctypes.c_uint32),
                                                 _p(data, ctypes.c_float)), "vlgpu_batch_upload_async")

    def download_begin(self):
        _check(self.lib.vlgpu_batch_download_begin(self.h), "vlgpu_batch_download_begin")

    def download_end(self, gids_out, data_out):
        """(cell_off, cell_count, gids, data) as download_raw; gids and data
        hold the result after sync()."""
        off = np.zeros(self.n_cells, np.uint32)
        cnt = np.zeros(self.n_cells, np.uint32)
        used = ctypes.c_uint64(0)
        _check(self.lib.vlgpu_batch_download_end(self.h, _p(off, ctypes.c_uint32), _p(cnt, ctypes.c_uint32),
                                                 _p(gids_out, ctypes.c_uint32), _p(data_out, ctypes.c_float),
                                                 len(gids_out), ctypes.byref(used)), "vlgpu_batch_download_end")
        u = int(used.value)
        return off, cnt, gids_out[:u], data_out[:u]

    def cells(self):
        offs, g, d = self.download()
        return [(g[offs[c]:offs[c + 1]], d[offs[c]:offs[c + 1]]) for c in range(self.n_cells)]

    # ---- the hot path ----
    def map_1d(self, intersections, dim: int, per_cell: bool = False):
        I = np.ascontiguousarray(intersections, np.float64).reshape(self.n_cells, 4)
        fn = self.lib.vlgpu_map_1d_per_cell if per_cell else self.lib.vlgpu_map_1d
        _check(fn(self.h, _p(I, ctypes.c_double), dim), "vlgpu_map_1d")

    def accelerate_with_intersections(self, intersections12, map_order: int):
        I = np.ascontiguousarray(intersections12, np.float64).reshape(self.n_cells, 12)
        _check(self.lib.vlgpu_accelerate_with_intersections(self.h, _p(I, ctypes.c_double), map_order),
               "vlgpu_accelerate_with_intersections")

    def _fields(self, B, dt, curl, egradpe):
        """vlgpu_cell_fields records (B, curl, egradpe: 9 doubles per cell) as
        one contiguous array, and dt per cell; keep F alive for the call."""
        n = self.n_cells
        F = np.zeros((n, 9), np.float64)
        F[:, 0:3] = np.asarray(B, np.float64).reshape(n, 3)
        if curl is not None:
            F[:, 3:6] = np.asarray(curl, np.float64).reshape(n, 3)
        if egradpe is not None:
            F[:, 6:9] = np.asarray(egradpe, np.float64).reshape(n, 3)
        assert ctypes.sizeof(CFieldsT) == 9 * 8
        dt = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, np.float64), (n,)))
        return F, dt

    @staticmethod
    def _fp(F):
        return F.ctypes.data_as(ctypes.POINTER(CFieldsT))

    def compute_intersections(self, B, dt, map_order: int, curl=None, egradpe=None) -> np.ndarray:
        F, dt = self._fields(B, dt, curl, egradpe)
        _check(self.lib.vlgpu_compute_intersections(self.h, self._fp(F), _p(dt, ctypes.c_double), map_order),
               "vlgpu_compute_intersections")
        return self.intersections()

    def accelerate(self, B, dt, map_order: int, curl=None, egradpe=None):
        """One acceleration step (moments -> FP64 geometry -> sweeps -> adjust -> moments) of every cell."""
        F, dt = self._fields(B, dt, curl, egradpe)
        _check(self.lib.vlgpu_accelerate(self.h, self._fp(F), _p(dt, ctypes.c_double), map_order),
               "vlgpu_accelerate")

    def accelerate_device(self, map_order: int, per_cell: bool = False):
        fn = self.lib.vlgpu_accelerate_per_cell if per_cell else self.lib.vlgpu_accelerate_device
        _check(fn(self.h, map_order), "vlgpu_accelerate_device")

    # ---- spatial translation ----
    def set_grid(self, dims, dx):
        """Cells form a uniform periodic grid dims (x fastest) with cell sizes dx (m)."""
        d = np.ascontiguousarray(dims, np.uint32)
        h = np.ascontiguousarray(np.broadcast_to(np.asarray(dx, np.float64), (3,)))
        _check(self.lib.vlgpu_batch_set_grid(self.h, _p(d, ctypes.c_uint32), _p(h, ctypes.c_double)),
               "vlgpu_batch_set_grid")

    def translate(self, dim: int, dt: float):
        """One translation sweep (trans_map_1d_amr) along dim over dt seconds."""
        _check(self.lib.vlgpu_translate(self.h, dim, float(dt)), "vlgpu_translate")

    def vlasov_step(self, B, dt: float, map_order: int, curl=None, egradpe=None):
        """Translation z, x, y + "_R" moments, then one acceleration step (grid batches)."""
        F, _ = self._fields(B, dt, curl, egradpe)
        _check(self.lib.vlgpu_vlasov_step(self.h, self._fp(F), float(dt), map_order), "vlgpu_vlasov_step")

    def vlasov_step_device(self, dt: float, map_order: int):
        _check(self.lib.vlgpu_vlasov_step_device(self.h, float(dt), map_order), "vlgpu_vlasov_step_device")

    def moments_r(self) -> np.ndarray:
        out = np.zeros((self.n_cells, 16))
        _check(self.lib.vlgpu_batch_moments_r(self.h, _p(out, ctypes.c_double)), "vlgpu_batch_moments_r")
        return out

    def fill_maxwellian(self, n, T, V, frame=None):
        """Initial VDF of every cell on the device: n (cells), T (cells or cells x 3),
        V (cells x 3), frame (cells x 3 x 3 rows = temperature axes; identity if None)."""
        k = self.n_cells
        n = np.broadcast_to(np.asarray(n, np.float64), (k,))
        T = np.asarray(T, np.float64)
        if T.ndim == 0:
            T = np.full((k, 3), float(T))
        elif T.ndim == 1:
            T = np.repeat(T[:, None], 3, axis=1)
        V = np.broadcast_to(np.asarray(V, np.float64), (k, 3))
        R = np.broadcast_to(np.eye(3) if frame is None else np.asarray(frame, np.float64), (k, 3, 3))
        arr = (CMaxwellianT * k)()
        for c in range(k):
            arr[c].n = float(n[c])
            for d in range(3):
                arr[c].T[d], arr[c].V[d] = float(T[c, d]), float(V[c, d])
            for q in range(9):
                arr[c].frame[q] = float(R[c].reshape(9)[q])
        _check(self.lib.vlgpu_batch_fill_maxwellian(self.h, arr), "vlgpu_batch_fill_maxwellian")

    def interpolated_moments(self) -> np.ndarray:
        """0.5 (R + V) of every moment (calculateInterpolatedVelocityMoments)."""
        out = np.zeros((self.n_cells, 16))
        _check(self.lib.vlgpu_batch_interpolated_moments(self.h, _p(out, ctypes.c_double)),
               "vlgpu_batch_interpolated_moments")
        return out

    def max_dt(self, max_rotation_deg: float = 22.0):
        """(r_dt, v_dt) per cell: reduce_vlasov_dt and updateAccelerationMaxdt limits."""
        r = np.zeros(self.n_cells)
        v = np.zeros(self.n_cells)
        _check(self.lib.vlgpu_batch_max_dt(self.h, float(max_rotation_deg), _p(r, ctypes.c_double),
                                           _p(v, ctypes.c_double)), "vlgpu_batch_max_dt")
        return r, v

    def adjust(self):
        _check(self.lib.vlgpu_adjust_blocks(self.h), "vlgpu_adjust_blocks")

    def rho_loss(self) -> np.ndarray:
        out = np.zeros(self.n_cells)
        _check(self.lib.vlgpu_batch_rho_loss(self.h, _p(out, ctypes.c_double)), "vlgpu_batch_rho_loss")
        return out

    def moments(self, second: bool = True) -> np.ndarray:
        out = np.zeros((self.n_cells, 16))
        _check(self.lib.vlgpu_batch_moments(self.h, int(second), _p(out, ctypes.c_double)), "vlgpu_batch_moments")
        return out

    def intersections(self) -> np.ndarray:
        out = np.zeros((self.n_cells, 12))
        _check(self.lib.vlgpu_batch_intersections(self.h, _p(out, ctypes.c_double)), "vlgpu_batch_intersections")
        return out

    def set_launch(self, shapes=None):
        """CTAs per SM of the remap, moments, adjustment and translation kernels
        (a 4-tuple, 0 = the occupancy maximum); None: the tuning table again."""
        if shapes is None:
            _check(self.lib.vlgpu_batch_set_launch(self.h, None), "vlgpu_batch_set_launch")
            return
        cfg = CLaunchT(*[int(x) for x in shapes])
        _check(self.lib.vlgpu_batch_set_launch(self.h, ctypes.byref(cfg)), "vlgpu_batch_set_launch")

    def launch(self):
        """The launch shapes in use, resolved to CTAs per SM (translate 0 = its maximum)."""
        cfg = CLaunchT()
        _check(self.lib.vlgpu_batch_get_launch(self.h, ctypes.byref(cfg)), "vlgpu_batch_get_launch")
        return cfg.as_tuple()

    def stream_handle(self) -> int:
        s = _vp()
        _check(self.lib.vlgpu_batch_stream(self.h, ctypes.byref(s)), "vlgpu_batch_stream")
        return int(s.value or 0)

    def profile(self, enable: bool = True):
        _check(self.lib.vlgpu_batch_profile(self.h, int(enable)), "vlgpu_batch_profile")

    def stats(self) -> dict:
        o = np.zeros(8, np.uint64)
        _check(self.lib.vlgpu_batch_stats(self.h, _p(o, ctypes.c_uint64)), "vlgpu_batch_stats")
        keys = ["launches", "cell_sweeps", "src_blocks", "dst_blocks", "remap_launches", "remap_ns",
                "remap_profiled", "sets"]
        d = {k: int(v) for k, v in zip(keys, o)}
        o2 = np.zeros(1, np.uint64)
        _check(self.lib.vlgpu_batch_stats2(self.h, _p(o2, ctypes.c_uint64)), "vlgpu_batch_stats2")
        d["step_blocks"] = int(o2[0])
        return d

    def sync(self):
        _check(self.lib.vlgpu_batch_sync(self.h), "vlgpu_batch_sync")
        self._inflight = None
