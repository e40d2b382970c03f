"""vlgpu_map_1d_noalloc: the SLICE-3D sweep without any device allocation.

This entry point is for callers that cannot call cudaMalloc: host codes that
reserve all of the GPU's memory for their own pool at start-up, and codes that
sweep on a latency-critical path where an allocation would synchronise the
device.  Its work arrays live in a fixed device array inside libvlgpu.so.  It
launches the same kernels as vlgpu_map_1d (which allocates its work arrays
with the batch), so a call must give bit for bit the same blocks and values,
and a second call must not see anything the first one left in that shared
array.

The file is named to be collected last: the GPU test runs after every other
test of a run, and also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from vlasiator_b200.mesh import CHARGE, MASS_PROTON, MU_0, WID3, VelocityMesh
from vlasiator_b200.projects import random_drifting_cells

ORDERS = [[0, 1, 2], [1, 2, 0], [2, 0, 1]]


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


def _pack(cells, lead=0):
    """Cells as (offsets, device gids, device data) in cell order, for the next
    call's input; `lead` unused blocks (of another caller) come first."""
    import torch
    offs = np.full(len(cells) + 1, lead, np.uint64)
    offs[1:] += np.cumsum([len(g) for g, _ in cells]).astype(np.uint64)
    g = np.concatenate([np.full(lead, 7, np.uint32)] + [np.asarray(g, np.uint32) for g, _ in cells])
    d = np.concatenate([np.full((lead, WID3), -1.0, np.float32)] +
                       [np.asarray(x, np.float32).reshape(-1, WID3) for _, x in cells])
    return offs, torch.from_numpy(g.view(np.int32)).cuda(), torch.from_numpy(d).cuda()


def _assert_cells_equal(got, ref, what):
    """Same kernels, same inputs: the same block sets and bit-identical values."""
    assert len(got) == len(ref)
    for ci, ((g1, d1), (g2, d2)) in enumerate(zip(got, ref)):
        np.testing.assert_array_equal(g1, g2, err_msg=f"{what}: cell {ci} block IDs")
        np.testing.assert_array_equal(d1, d2, err_msg=f"{what}: cell {ci} values")


def _batch_sweeps(vlgpu, mesh, params, cells, I, dims):
    """The existing entry point: vlgpu_map_1d sweeps of one batch."""
    total = sum(len(g) for g, _ in cells)
    ref = []
    with vlgpu.Batch(mesh, len(cells), 3 * total + 65536, params=params) as b:
        b.upload([g for g, _ in cells], [d for _, d in cells])
        for dim in dims:
            b.map_1d(I[:, 4 * dim:4 * dim + 4], dim)
            ref.append(b.cells())
        b.sync()
        assert not b.status().any()
    return ref


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
    assert sum(c.n_blocks for c in cells) <= 32768  # room for the sweeps to add blocks below the 65536-block limit
    stream = torch.cuda.current_stream().cuda_stream
    ref = _batch_sweeps(vlgpu, mesh, params, [(c.gids, c.data) for c in cells], I, ORDERS[mo][:2])

    # the no-allocation entry point: the same two sweeps, call 2 reading call 1's output
    offs, g_dev, d_dev = _pack([(c.gids, c.data) for c in cells])
    for call, dim in enumerate(ORDERS[mo][:2]):
        code, got, st = _noalloc(vlgpu, lib, mesh, params, offs, g_dev, d_dev, I[:, 4 * dim:4 * dim + 4], dim,
                                 65536, stream)
        assert code == 0, vlgpu.STATUS.get(code, code)
        assert not st.any()
        _assert_cells_equal(got, ref[call], f"call {call + 1} (dim {dim})")
        offs, g_dev, d_dev = _pack(got)

    # an output that does not fit is reported, and the next call is unaffected
    offs, g_dev, d_dev = _pack([(c.gids, c.data) for c in cells])
    dim = ORDERS[mo][0]
    code, _, _ = _noalloc(vlgpu, lib, mesh, params, offs, g_dev, d_dev, I[:, 4 * dim:4 * dim + 4], dim, 16, stream)
    assert vlgpu.STATUS.get(code) == "VLGPU_ENOMEM"
    code, got, st = _noalloc(vlgpu, lib, mesh, params, offs, g_dev, d_dev, I[:, 4 * dim:4 * dim + 4], dim, 65536,
                             stream)
    assert code == 0 and not st.any()
    _assert_cells_equal(got, ref[0], "call after an overflow")


@pytest.mark.gpu
def test_noalloc_offset_input_and_empty_cell(orc_sp):
    """Inputs that start at offsets[0] > 0 behind another caller's blocks, and
    a cell without blocks: the absolute block indexing of the sweep."""
    import torch

    from vlasiator_b200 import vlgpu
    lib = vlgpu.load()
    mesh = VelocityMesh()
    params = vlgpu.make_params()
    mo = 2
    src = random_drifting_cells(5, seed=57, mesh=mesh)
    cells = [(c.gids, c.data) for c in src]
    cells.insert(2, (np.zeros(0, np.uint32), np.zeros((0, WID3), np.float32)))
    I = np.stack([_geometry(orc_sp, c, 0.02, mesh, mo) for c in src])
    I = np.insert(I, 2, I[0], axis=0)
    stream = torch.cuda.current_stream().cuda_stream
    ref = _batch_sweeps(vlgpu, mesh, params, cells, I, ORDERS[mo][:2])
    offs, g_dev, d_dev = _pack(cells, lead=37)
    for call, dim in enumerate(ORDERS[mo][:2]):
        code, got, st = _noalloc(vlgpu, lib, mesh, params, offs, g_dev, d_dev, I[:, 4 * dim:4 * dim + 4], dim,
                                 65536, stream)
        assert code == 0, vlgpu.STATUS.get(code, code)
        assert not st.any()
        assert len(got[2][0]) == 0
        _assert_cells_equal(got, ref[call], f"offset input, call {call + 1} (dim {dim})")
        offs, g_dev, d_dev = _pack(got, lead=5)


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


def test_noalloc_rejects_output_equal_to_input(capfd):
    """Writing over the input would let one cell's output overwrite blocks
    another cell has not read yet; the call refuses before any device work (the
    pointer values are only compared, never used)."""
    from vlasiator_b200 import vlgpu
    lib = vlgpu.load()
    mesh = VelocityMesh()
    params = vlgpu.make_params()
    I = np.zeros((1, 4))
    I[:, 3] = 3e4
    offs = np.array([0, 4], np.uint64)
    out = np.zeros(1, np.uint32)
    u32 = ctypes.POINTER(ctypes.c_uint32)
    fake_g, fake_d, other = ctypes.c_void_p(1 << 20), ctypes.c_void_p(1 << 21), ctypes.c_void_p(1 << 22)
    for g_out, d_out in ((other, fake_d), (fake_g, other)):
        code = lib.vlgpu_map_1d_noalloc(
            ctypes.byref(_c_mesh(vlgpu, mesh)), ctypes.byref(params), 1,
            offs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), fake_g, fake_d,
            I.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 0, g_out, d_out, 16, out.ctypes.data_as(u32),
            out.ctypes.data_as(u32), None, None)
        assert code == 1  # VLGPU_EINVAL
        assert "must not be the input" in capfd.readouterr().err
