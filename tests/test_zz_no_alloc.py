"""vlgpu_map_1d_noalloc: the SLICE-3D sweep without any device allocation.

This entry point is for callers that cannot call cudaMalloc: host codes that
reserve all of the GPU's memory for their own pool at start-up, and codes that
sweep on a latency-critical path where an allocation would synchronise the
device.  Its work arrays live in a fixed device array inside libvlgpu.so, so
a call must give the same result as vlgpu_map_1d, which allocates its work
arrays with the batch, and a second call must not see anything the first one
left in that shared array.

The file is named to be collected last: the GPU test runs after every other
test of a run, and also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from vlasiator_b200.mesh import CHARGE, MASS_PROTON, MU_0, WID3, VelocityMesh
from vlasiator_b200.projects import random_drifting_cells

ORDERS = [[0, 1, 2], [1, 2, 0], [2, 0, 1]]
TOL = 1e-5  # of the cell's peak value, the sweep tolerance of the GPU tests


def _c_mesh(vl, mesh):
    m = vl.CMeshT()
    for d in range(3):
        m.vmin[d], m.vmax[d], m.len[d] = mesh.vmin[d], mesh.vmax[d], mesh.length[d]
    return m


def _geometry(orc, c, frac, mesh, map_order):
    Tg = 2 * np.pi * MASS_PROTON / (CHARGE * float(np.linalg.norm(c.B)))
    L, t = orc.acceleration_transform(c.B, np.zeros(3), 0.0, c.V, np.zeros(3), CHARGE, MASS_PROTON, frac * Tg,
                                      CHARGE, 0, MU_0)
    return orc.cell_intersections(L, t, mesh, map_order)


def _noalloc(vl, lib, mesh, params, offsets, gids_dev, data_dev, I, dim, out_capacity, stream):
    """One call through the C ABI; returns (status code, cells as sorted (gids, data), per-cell bits)."""
    import torch
    n = len(offsets) - 1
    offs = np.ascontiguousarray(offsets, np.uint64)
    Ic = np.ascontiguousarray(I, np.float64).reshape(n, 4)
    g_out = torch.zeros(max(out_capacity, 1), dtype=torch.int32, device="cuda")
    d_out = torch.zeros((max(out_capacity, 1), WID3), dtype=torch.float32, device="cuda")
    off = np.zeros(n, np.uint32)
    cnt = np.zeros(n, np.uint32)
    st = np.zeros(n, np.uint32)
    code = lib.vlgpu_map_1d_noalloc(
        ctypes.byref(_c_mesh(vl, mesh)), ctypes.byref(params), n, offs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
        gids_dev.data_ptr(), data_dev.data_ptr(), Ic.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), dim,
        g_out.data_ptr(), d_out.data_ptr(), out_capacity, off.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
        cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), st.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
        stream)
    g = g_out.cpu().numpy().view(np.uint32)
    d = d_out.cpu().numpy()
    cells = []
    for c in range(n):
        gg, dd = g[off[c]:off[c] + cnt[c]], d[off[c]:off[c] + cnt[c]]
        order = np.argsort(gg, kind="stable")
        cells.append((gg[order], dd[order]))
    return code, cells, st


def _pack(cells):
    """Cells as (offsets, device gids, device data) in cell order, for the next call's input."""
    import torch
    offs = np.zeros(len(cells) + 1, np.uint64)
    offs[1:] = np.cumsum([len(g) for g, _ in cells])
    g = np.concatenate([g for g, _ in cells]).astype(np.uint32)
    d = np.concatenate([np.asarray(x, np.float32).reshape(-1, WID3) for _, x in cells])
    return offs, torch.from_numpy(g.view(np.int32)).cuda(), torch.from_numpy(d).cuda()


def _assert_cells_close(got, ref, what):
    assert len(got) == len(ref)
    for ci, ((g1, d1), (g2, d2)) in enumerate(zip(got, ref)):
        np.testing.assert_array_equal(g1, g2, err_msg=f"{what}: cell {ci} block IDs")
        peak = float(np.abs(d2).max()) if d2.size else 0.0
        err = float(np.abs(d1 - d2).max()) if d2.size else 0.0
        assert err <= TOL * peak, f"{what}: cell {ci} max |diff| {err:.3e} vs peak {peak:.3e}"


@pytest.mark.gpu
def test_noalloc_matches_map_1d_on_two_calls_in_a_row(orc_sp):
    import torch

    from vlasiator_b200 import vlgpu
    lib = vlgpu.load()
    mesh = VelocityMesh()
    params = vlgpu.make_params()
    mo = 1
    cells = random_drifting_cells(16, seed=31, mesh=mesh)
    I = np.stack([_geometry(orc_sp, c, 0.03, mesh, mo) for c in cells])
    total = sum(c.n_blocks for c in cells)
    assert total <= 32768  # room for the sweeps to add blocks below the 65536-block limit
    stream = torch.cuda.current_stream().cuda_stream

    # the existing entry point: two sweeps of a batch
    ref = []
    with vlgpu.Batch(mesh, len(cells), 3 * total + 65536, params=params) as b:
        b.upload([c.gids for c in cells], [c.data for c in cells])
        for dim in ORDERS[mo][:2]:
            b.map_1d(I[:, 4 * dim:4 * dim + 4], dim)
            ref.append(b.cells())
        b.sync()
        assert not b.status().any()

    # the no-allocation entry point: the same two sweeps, call 2 reading call 1's output
    offs, g_dev, d_dev = _pack([(c.gids, c.data) for c in cells])
    for call, dim in enumerate(ORDERS[mo][:2]):
        code, got, st = _noalloc(vlgpu, lib, mesh, params, offs, g_dev, d_dev, I[:, 4 * dim:4 * dim + 4], dim,
                                 65536, stream)
        assert code == 0, vlgpu.STATUS.get(code, code)
        assert not st.any()
        _assert_cells_close(got, ref[call], f"call {call + 1} (dim {dim})")
        offs, g_dev, d_dev = _pack(got)

    # an output that does not fit is reported, and the next call is unaffected
    offs, g_dev, d_dev = _pack([(c.gids, c.data) for c in cells])
    dim = ORDERS[mo][0]
    code, _, _ = _noalloc(vlgpu, lib, mesh, params, offs, g_dev, d_dev, I[:, 4 * dim:4 * dim + 4], dim, 16, stream)
    assert vlgpu.STATUS.get(code) == "VLGPU_ENOMEM"
    code, got, st = _noalloc(vlgpu, lib, mesh, params, offs, g_dev, d_dev, I[:, 4 * dim:4 * dim + 4], dim, 65536,
                             stream)
    assert code == 0 and not st.any()
    _assert_cells_close(got, ref[0], "call after an overflow")


def test_noalloc_rejects_sizes_beyond_its_limit(capfd):
    """Checked on the host before any device work (no GPU needed; the device
    pointers are NULL, so nothing could reach a kernel either way)."""
    from vlasiator_b200 import vlgpu
    lib = vlgpu.load()
    mesh = VelocityMesh()
    params = vlgpu.make_params()
    I = np.zeros((2048, 4))
    I[:, 3] = 3e4
    out = np.zeros(2048, np.uint32)
    u32 = ctypes.POINTER(ctypes.c_uint32)

    def call(offsets):
        offs = np.ascontiguousarray(offsets, np.uint64)
        n = len(offs) - 1
        return lib.vlgpu_map_1d_noalloc(
            ctypes.byref(_c_mesh(vlgpu, mesh)), ctypes.byref(params), n,
            offs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), None, None,
            I.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 0, None, None, 0, out.ctypes.data_as(u32),
            out.ctypes.data_as(u32), None, None)

    cases = [np.zeros(1026, np.uint64),  # 1025 cells: 1024 at most
             [0, 65537],                  # 65537 input blocks: 65536 at most
             [70000, 70001]]              # block indices beyond the limit
    for offsets in cases:
        assert call(offsets) == 1  # VLGPU_EINVAL
        assert "the limit is" in capfd.readouterr().err
