"""The C++ drop-in layer (include/vlgpu.hpp) against the reference.

oracle/_ref/libvlasov_ref_sp_dropin.so holds the reference's own map_1d and
the drop-in functions instantiated with the same stand-in SpatialCell.  Two
copies of the same cells go through the reference's map_1d
(cpu_acc_map.cpp:121-636) and through vlgpu_dropin::map_1d, which runs the
sweep on the GPU and writes the result back into the cell's VelocityMesh and
VelocityBlockContainer; their block sets, values and block parameters (seen
through the reference's moment templates, which read each block's corner and
cell size) must agree: bit for bit in the exact arithmetic, to 1e-5 of the
peak in the fused one.  vlgpu_dropin::gpu_accelerate_cells is checked the same
way against the reference's three sweeps with the oracle's FP64 geometry.
"""
import ctypes
import os

import numpy as np
import pytest

from oracle.oracle import HERE as ORACLE_DIR
from oracle.oracle import ReferenceBuild
from tests.geometry_ref import intersections, transform
from vlasiator_b200.mesh import CHARGE, MASS_PROTON, MU_0
from vlasiator_b200.projects import random_drifting_cells

LIB = os.path.join(ORACLE_DIR, "_ref", "libvlasov_ref_sp_dropin.so")
pytestmark = pytest.mark.skipif(not os.path.exists(LIB), reason="drop-in test build (oracle/_ref) not present")
ORDERS = [[0, 1, 2], [1, 2, 0], [2, 0, 1]]


def _dropin():
    ref = ReferenceBuild("sp_dropin")
    L = ref.lib
    L.dropin_set_exact.argtypes = [ctypes.c_int]
    L.dropin_set_species.argtypes = [ctypes.c_double, ctypes.c_double]
    dp = ctypes.POINTER(ctypes.c_double)
    L.dropin_cells_map_1d.argtypes = [ctypes.c_void_p, dp, ctypes.c_uint32]
    L.dropin_cells_accelerate.argtypes = [ctypes.c_void_p, dp, dp, ctypes.c_uint32, dp]
    return ref


def _ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _intersections(orc, mesh, cells, frac, mo):
    out = []
    for c in cells:
        Tg = 2 * np.pi * MASS_PROTON / (CHARGE * float(np.linalg.norm(c.B)))
        L, t = orc.acceleration_transform(c.B, np.zeros(3), 0.0, c.V, np.zeros(3), CHARGE, MASS_PROTON, frac * Tg,
                                          CHARGE, 0, MU_0)
        out.append(orc.cell_intersections(L, t, mesh, mo))
    return np.stack(out)


def _compare(ref, h1, h2, n, exact):
    for c in range(n):
        g1, d1 = ref.extract(h1, c)
        g2, d2 = ref.extract(h2, c)
        np.testing.assert_array_equal(g2, g1, err_msg=f"cell {c}: block IDs")
        if exact:
            assert np.array_equal(d2, d1), f"cell {c}: values"
        else:
            assert np.abs(d2 - d1).max() <= 1e-5 * float(np.abs(d1).max()), f"cell {c}: values"
        # block parameters (corner, cell size) written back as the reference sets them
        f1, s1 = ref.moments(h1, c, np.zeros(3))
        f2, s2 = ref.moments(h2, c, np.zeros(3))
        np.testing.assert_allclose(f2, f1, rtol=1e-5 if not exact else 1e-12)
        np.testing.assert_allclose(s2, s1, rtol=1e-5 if not exact else 1e-12)


def test_dropin_library_loads_without_a_gpu():
    """The drop-in build links libvlgpu.so and exports its entry points; no
    device call is made."""
    ref = _dropin()
    for name in ("dropin_set_exact", "dropin_cells_map_1d", "dropin_cells_accelerate", "ref_cells_map_1d"):
        assert hasattr(ref.lib, name)


@pytest.mark.gpu
@pytest.mark.parametrize("exact", [1, 0])
def test_dropin_map_1d_matches_reference(mesh, orc_sp, exact):
    ref = _dropin()
    ref.init(mesh)
    ref.lib.dropin_set_exact(exact)
    cells = random_drifting_cells(8, seed=61, mesh=mesh)
    mo = 1
    I = _intersections(orc_sp, mesh, cells, 0.02, mo)
    args = ([c.gids for c in cells], [c.data for c in cells], [1e-15] * len(cells))
    h1, h2 = ref.create(*args), ref.create(*args)
    try:
        for dim in ORDERS[mo]:
            Id = np.ascontiguousarray(I[:, 4 * dim:4 * dim + 4])
            ref.map_1d(h1, Id, dim)                            # the reference's map_1d
            ref.lib.dropin_cells_map_1d(h2, _ptr(Id), dim)     # vlgpu_dropin::map_1d
            _compare(ref, h1, h2, len(cells), exact)
        assert ref.bailouts() == 0
    finally:
        ref.destroy(h1)
        ref.destroy(h2)


@pytest.mark.gpu
@pytest.mark.parametrize("exact", [1, 0])
def test_dropin_accelerate_cells_matches_reference(mesh, orc_sp, exact):
    ref = _dropin()
    ref.init(mesh)
    ref.lib.dropin_set_exact(exact)
    ref.lib.dropin_set_species(CHARGE, MASS_PROTON)
    cells = random_drifting_cells(10, seed=62, mesh=mesh)
    B = np.ascontiguousarray(np.stack([c.B for c in cells]))
    dt = np.ascontiguousarray(0.01 * 2 * np.pi * MASS_PROTON / (CHARGE * np.linalg.norm(B, axis=1)))
    mo = 2
    args = ([c.gids for c in cells], [c.data for c in cells], [1e-15] * len(cells))
    h1, h2 = ref.create(*args), ref.create(*args)
    try:
        # the pivot: first moments of the cells before the step, with the
        # reference's own template (double sums, as calculateMoments_V)
        pivots = [ref.moments(h1, c, np.zeros(3))[0] for c in range(len(cells))]
        ref.accelerate_step(h1, B, dt, mo, CHARGE, MASS_PROTON)    # reference sweeps, oracle geometry
        I = np.zeros((len(cells), 12))
        ref.lib.dropin_cells_accelerate(h2, _ptr(B), _ptr(dt), mo, _ptr(I))
        # the intersections stored in the populations: the closed-form geometry
        want = []
        for c, cell in enumerate(cells):
            V = pivots[c][1:4] / pivots[c][0]
            L, t = transform(cell.B, V, dt[c], CHARGE, MASS_PROTON)
            want.append(intersections(L, t, mesh.vmin, mesh.dv, mo))
        want = np.stack(want)
        scale = np.array([4e6, 3e4, 3e4, 3e4] * 3)
        assert (np.abs(I - want) / scale).max() <= 1e-11
        same = 0
        for c in range(len(cells)):
            g1, d1 = ref.extract(h1, c)
            g2, d2 = ref.extract(h2, c)
            if np.array_equal(g1, g2) and np.array_equal(d1, d2):
                same += 1
                continue
            common = np.intersect1d(g1, g2)
            assert len(common) >= 0.99 * max(len(g1), len(g2))
            i1, i2 = np.searchsorted(g1, common), np.searchsorted(g2, common)
            assert np.abs(d2[i2] - d1[i1]).max() <= 1e-5 * float(np.abs(d1).max())
        if exact:
            assert same >= len(cells) - 1
        assert ref.bailouts() == 0
    finally:
        ref.destroy(h1)
        ref.destroy(h2)
