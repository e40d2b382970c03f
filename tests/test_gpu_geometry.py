"""The device's FP64 gyration geometry pinned by the same closed forms and
independent definitions as the oracle's (tests/geometry_ref.py): the
intersections vlgpu_compute_intersections builds on the GPU for each cell
(cpu_acc_transform.cpp:66-153, cpu_acc_intersections.cpp:44-450), with the
pivot velocity and charge density the device took from the cell's own first
moments.  Tolerance 1e-12 of the scale (4e6 m/s positions, 3e4 m/s steps):
the device's sin/cos and the host's may differ in the last bits.
"""
import numpy as np
import pytest

from tests.geometry_ref import intersections, intersections_b_along_z, transform
from vlasiator_b200.mesh import CHARGE, MASS_PROTON
from vlasiator_b200.projects import random_drifting_cells

pytestmark = pytest.mark.gpu

SCALE = np.array([4e6, 3e4, 3e4, 3e4] * 3)


@pytest.fixture(scope="module")
def vl():
    from vlasiator_b200 import vlgpu
    vlgpu.load()
    return vlgpu


def _gyroperiod(B):
    return 2 * np.pi * MASS_PROTON / (CHARGE * (np.linalg.norm(B) + 1e-30))


def _device_geometry(vl, mesh, cells, B, dt, map_order, curl=None):
    total = sum(c.n_blocks for c in cells)
    with vl.Batch(mesh, len(cells), 2 * total + 4096) as b:
        b.upload([c.gids for c in cells], [c.data for c in cells])
        isect = b.compute_intersections(B, dt, map_order, curl=curl)
        mom = b.moments(second=False)
    return isect, mom


@pytest.mark.parametrize("map_order", [0, 1, 2])
def test_device_intersections_match_definitions(vl, mesh, map_order):
    cells = random_drifting_cells(8, seed=70 + map_order)
    rng = np.random.default_rng(map_order)
    B = np.stack([c.B for c in cells])
    dt = np.array([rng.uniform(0.003, 0.06) * _gyroperiod(b) for b in B])
    isect, mom = _device_geometry(vl, mesh, cells, B, dt, map_order)
    for ci in range(len(cells)):
        L, t = transform(B[ci], mom[ci, 5:8], dt[ci], CHARGE, MASS_PROTON)
        want = intersections(L, t, mesh.vmin, mesh.dv, map_order)
        err = np.abs(isect[ci] - want) / SCALE
        assert err.max() <= 1e-12, f"cell {ci}: {err.max():.2e}"


def test_device_intersections_with_hall_term(vl, mesh):
    cells = random_drifting_cells(6, seed=91)
    rng = np.random.default_rng(5)
    B = np.stack([c.B for c in cells])
    curl = rng.normal(size=(len(cells), 3)) * 1e-14
    dt = np.array([0.0213 * _gyroperiod(b) for b in B])
    isect, mom = _device_geometry(vl, mesh, cells, B, dt, 1, curl=curl)
    for ci in range(len(cells)):
        L, t = transform(B[ci], mom[ci, 5:8], dt[ci], CHARGE, MASS_PROTON, curl=curl[ci], rhoq=mom[ci, 8])
        want = intersections(L, t, mesh.vmin, mesh.dv, 1)
        err = np.abs(isect[ci] - want) / SCALE
        assert err.max() <= 1e-11, f"cell {ci}: {err.max():.2e}"


@pytest.mark.parametrize("map_order", [0, 1, 2])
def test_device_intersections_closed_form_b_along_z(vl, mesh, map_order):
    cells = random_drifting_cells(4, seed=13)
    B = np.tile([0.0, 0.0, 1e-8], (len(cells), 1))
    fr = np.array([0.01, 0.025, -0.015, 0.04])
    dt = fr * _gyroperiod(B[0])
    isect, mom = _device_geometry(vl, mesh, cells, B, dt, map_order)
    for ci in range(len(cells)):
        phi = -2 * np.pi * fr[ci]
        want = intersections_b_along_z(phi, mom[ci, 5:8], mesh.vmin, mesh.dv[0], map_order)
        err = np.abs(isect[ci] - want) / SCALE
        assert err.max() <= 1e-12, f"cell {ci}: {err.max():.2e}"


def test_device_full_gyroperiod_gives_the_identity_grid(vl, mesh):
    cells = random_drifting_cells(3, seed=17)
    B = np.stack([c.B for c in cells])
    dt = np.array([_gyroperiod(b) for b in B])
    dv = mesh.dv
    ident = np.array([mesh.vmin[0], dv[0], 0, 0, mesh.vmin[1], 0, dv[1], 0, mesh.vmin[2], 0, 0, dv[2]])
    for mo in range(3):
        isect, _ = _device_geometry(vl, mesh, cells, B, dt, mo)
        err = np.abs(isect - ident[None, :]) / SCALE
        assert err.max() <= 1e-11, f"map order {mo}: {err.max():.2e}"
