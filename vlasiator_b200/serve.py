"""Host side of the serving engine (libvlgpu.so's vlgpu_server_*).

``Server`` admits independent VDF-advance requests into one device-resident
batch and advances all admitted requests together, one acceleration step per
tick; ``run_stream`` feeds it a timed arrival stream and reports latency
percentiles and throughput; ``run_plain`` runs the same requests one at a
time through the plain per-cell launch path, the drop-in baseline.
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

from . import vlgpu
from .mesh import WID3, VelocityMesh

_vp = ctypes.c_void_p
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_fp = ctypes.POINTER(ctypes.c_float)


class Server:
    """A request loop on one GPU (see vlgpu_server_create in include/vlgpu.h)."""

    def __init__(self, mesh: VelocityMesh, max_cells: int, hbm_budget_bytes: int, params=None, device: int = 0):
        self.lib = vlgpu.load()
        self.mesh = mesh
        m = vlgpu.CMeshT()
        for d in range(3):
            m.vmin[d], m.vmax[d], m.len[d] = mesh.vmin[d], mesh.vmax[d], mesh.length[d]
        self.params = params or vlgpu.make_params()
        h = _vp()
        vlgpu._check(self.lib.vlgpu_server_create(ctypes.byref(m), ctypes.byref(self.params), int(max_cells),
                                                  int(hbm_budget_bytes), device, ctypes.byref(h)),
                     "vlgpu_server_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.vlgpu_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, gids, data, B, dt: float, steps: int) -> int:
        g = np.ascontiguousarray(gids, np.uint32)
        d = np.ascontiguousarray(data, np.float32).reshape(-1, WID3)
        f = vlgpu.CFieldsT()
        for r in range(3):
            f.B[r] = float(B[r])
        rid = ctypes.c_uint64(0)
        vlgpu._check(self.lib.vlgpu_server_submit(self.h, len(g), g.ctypes.data_as(_u32p), d.ctypes.data_as(_fp),
                                                  ctypes.byref(f), float(dt), int(steps), ctypes.byref(rid)),
                     "vlgpu_server_submit")
        return int(rid.value)

    def tick(self):
        """(active, pending, finished this tick)"""
        a, p, d = ctypes.c_uint32(0), ctypes.c_uint32(0), ctypes.c_uint32(0)
        vlgpu._check(self.lib.vlgpu_server_tick(self.h, ctypes.byref(a), ctypes.byref(p), ctypes.byref(d)),
                     "vlgpu_server_tick")
        return a.value, p.value, d.value

    def result(self, rid: int):
        """(gids, data, status, rho_loss) of a finished request, or None while it runs."""
        n = ctypes.c_uint32(0)
        st = ctypes.c_uint32(0)
        loss = ctypes.c_double(0)
        rc = self.lib.vlgpu_server_result(self.h, rid, ctypes.byref(n), None, None, 0, ctypes.byref(st),
                                          ctypes.byref(loss))
        if rc == 8:  # VLGPU_EAGAIN
            return None
        if rc == 0:  # no blocks left; the request is gone now
            return np.zeros(0, np.uint32), np.zeros((0, WID3), np.float32), int(st.value), float(loss.value)
        if rc != 2:  # anything but "buffer too small"
            vlgpu._check(rc, "vlgpu_server_result")
        g = np.zeros(max(n.value, 1), np.uint32)
        d = np.zeros((max(n.value, 1), WID3), np.float32)
        vlgpu._check(self.lib.vlgpu_server_result(self.h, rid, ctypes.byref(n), g.ctypes.data_as(_u32p),
                                                  d.ctypes.data_as(_fp), len(g), ctypes.byref(st),
                                                  ctypes.byref(loss)), "vlgpu_server_result")
        return g[: n.value], d[: n.value], int(st.value), float(loss.value)

    def stats(self) -> dict:
        o = np.zeros(4, np.uint64)
        vlgpu._check(self.lib.vlgpu_server_stats(self.h, o.ctypes.data_as(_u64p)), "vlgpu_server_stats")
        return {"ticks": int(o[0]), "completed": int(o[1]), "cell_steps": int(o[2]), "cell_updates": int(o[3])}


def run_stream(server: Server, requests, rate_per_s: float, seed: int = 0, collect: bool = False):
    """Submits `requests` (dicts: cell, B, dt, steps) at Poisson arrival times
    of the given mean rate and ticks the server until all are done.
    Returns per-request latencies (s), wall time (s), and results if collect."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate_per_s, size=len(requests)))
    t0 = time.perf_counter()
    nxt = 0
    ids = {}
    latency = np.zeros(len(requests))
    results = {}
    remaining = len(requests)
    while remaining > 0:
        now = time.perf_counter() - t0
        while nxt < len(requests) and arrivals[nxt] <= now:
            q = requests[nxt]
            ids[server.submit(q["cell"].gids, q["cell"].data, q["B"], q["dt"], q["steps"])] = nxt
            nxt += 1
        active, pending, done = server.tick()
        if done:
            for rid in list(ids):
                r = server.result(rid)
                if r is None:
                    continue
                k = ids.pop(rid)
                latency[k] = (time.perf_counter() - t0) - arrivals[k]
                remaining -= 1
                if collect:
                    results[k] = r
        if active == 0 and pending == 0 and nxt < len(requests):
            time.sleep(max(0.0, min(arrivals[nxt] - (time.perf_counter() - t0), 0.01)))
    return latency, time.perf_counter() - t0, results


def run_plain(mesh: VelocityMesh, requests, params=None):
    """Each request alone through the plain per-cell launch path: upload, its
    steps with dimension order s mod 3, download.  Returns per-request wall
    times (s) and results."""
    out, times = [], []
    for q in requests:
        c = q["cell"]
        t0 = time.perf_counter()
        with vlgpu.Batch(mesh, 1, max(4 * c.n_blocks, 65536), params=params) as b:
            b.upload([c.gids], [c.data])
            b.compute_intersections(q["B"][None, :], q["dt"], 0)  # stages the fields
            for s in range(q["steps"]):
                b.accelerate_device(s % 3, per_cell=True)
            (g, d), = b.cells()
            st = int(b.status()[0])
        times.append(time.perf_counter() - t0)
        out.append((g, d, st))
    return np.array(times), out

