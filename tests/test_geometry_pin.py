"""The oracle's FP64 gyration transform and SLICE-3D intersections pinned by
closed forms and by an independent implementation of their definitions.

The reference computes both with Eigen (vlasovsolver/cpu_acc_transform.cpp:
66-153, cpu_acc_intersections.cpp:44-450), which is absent, so the oracle
restates them in C.  These checks hold the restatement to:
  - the closed form of the transform: a rotation by -2 pi dt / T_g about
    unit B around the bulk velocity (a fixed point of every substep), plus the
    summed Hall drift of the pivot (tests/geometry_ref.py);
  - a full gyroperiod returning the identity;
  - the intersections computed from their geometric definitions with a
    generic line-plane solver on the inverted 4x4 transform;
  - hand-derived closed forms of the intersections for B along z.
"""
import numpy as np
import pytest

from tests.geometry_ref import intersections, intersections_b_along_z, rotation, transform
from vlasiator_b200.mesh import CHARGE, MASS_PROTON, MU_0, VelocityMesh

HALL_MIN = 1.60217653e-19


def _orc_transform(orc, B, V, dt, curl=(0, 0, 0), rhoq=0.0):
    return orc.acceleration_transform(np.asarray(B, float), np.asarray(curl, float), rhoq, np.asarray(V, float),
                                      np.zeros(3), CHARGE, MASS_PROTON, dt, HALL_MIN, 0, MU_0)


def _close(got, want, rel):
    """Intersections agree to `rel` of their scale (4e6 m/s positions, 3e4 m/s steps)."""
    scale = np.array([4e6, 3e4, 3e4, 3e4] * 3)
    err = np.abs(np.asarray(got) - np.asarray(want))
    assert np.all(err <= rel * scale), f"max error / scale {np.max(err / scale):.2e}"


def _gyroperiod(B):
    return 2 * np.pi * MASS_PROTON / (CHARGE * (np.linalg.norm(B) + 1e-30))


@pytest.mark.parametrize("seed", range(6))
def test_transform_is_a_rotation_about_the_bulk_velocity(orc_dp, seed):
    rng = np.random.default_rng(seed)
    B = rng.normal(size=3) * rng.uniform(5e-9, 5e-8)
    V = rng.normal(size=3) * 3e5
    dt = rng.uniform(0.001, 0.05) * _gyroperiod(B)
    L, t = _orc_transform(orc_dp, B, V, dt)
    R, c = transform(B, V, dt, CHARGE, MASS_PROTON)
    np.testing.assert_allclose(L, R, atol=1e-12)
    np.testing.assert_allclose(t, c, rtol=0, atol=1e-12 * np.linalg.norm(V) + 1e-9)
    # the pivot is a fixed point and the axis is invariant
    np.testing.assert_allclose(L @ V + t, V, rtol=0, atol=1e-9)
    np.testing.assert_allclose(L @ (B / np.linalg.norm(B)), B / np.linalg.norm(B), atol=1e-14)
    np.testing.assert_allclose(L @ L.T, np.eye(3), atol=1e-14)
    assert np.linalg.det(L) == pytest.approx(1.0, abs=1e-13)


def test_transform_with_hall_term_follows_the_pivot_recursion(orc_dp):
    rng = np.random.default_rng(11)
    for _ in range(4):
        B = rng.normal(size=3) * 2e-8
        V = rng.normal(size=3) * 2e5
        curl = rng.normal(size=3) * 1e-14  # T/m
        rhoq = rng.uniform(0.5, 5) * 1e6 * CHARGE
        # not a multiple of the 0.1-degree substep, where the substep count
        # would depend on the last bit of |B|
        dt = 0.0213 * _gyroperiod(B)
        L, t = _orc_transform(orc_dp, B, V, dt, curl=curl, rhoq=rhoq)
        R, c = transform(B, V, dt, CHARGE, MASS_PROTON, curl=curl, rhoq=rhoq)
        np.testing.assert_allclose(L, R, atol=1e-12)
        np.testing.assert_allclose(t, c, rtol=1e-10, atol=1e-6)
        # the Hall term moves the pivot: without it the result differs
        _, t0 = _orc_transform(orc_dp, B, V, dt)
        assert np.abs(t - t0).max() > 1e3 * np.abs(t - c).max()


@pytest.mark.parametrize("turns", [1, 3])
def test_full_gyroperiods_return_the_identity(orc_dp, turns):
    B = np.array([1e-8, -2e-8, 4e-9])
    V = np.array([2e5, 1e5, -3e5])
    L, t = _orc_transform(orc_dp, B, V, turns * _gyroperiod(B))
    np.testing.assert_allclose(L, np.eye(3), atol=1e-12)
    np.testing.assert_allclose(t, 0.0, atol=1e-12 * np.linalg.norm(V) * 10)


@pytest.mark.parametrize("map_order", [0, 1, 2])
def test_intersections_match_their_definitions(orc_dp, map_order):
    mesh = VelocityMesh()
    rng = np.random.default_rng(100 + map_order)
    for _ in range(5):
        B = rng.normal(size=3) * 1e-8
        V = rng.normal(size=3) * 4e5
        dt = rng.uniform(0.002, 0.07) * _gyroperiod(B)
        L, t = _orc_transform(orc_dp, B, V, dt)
        got = orc_dp.cell_intersections(L, t, mesh, map_order)
        want = intersections(L, t, mesh.vmin, mesh.dv, map_order)
        _close(got, want, 1e-12)


@pytest.mark.parametrize("map_order", [0, 1, 2])
def test_intersections_closed_form_for_b_along_z(orc_dp, map_order):
    mesh = VelocityMesh()
    dv = mesh.dv[0]
    for frac, V in ((0.01, (0.0, 0.0, 0.0)), (0.03, (2.5e5, -1e5, 7e4)), (-0.02, (-3e5, 4e5, 0.0))):
        B = np.array([0.0, 0.0, 1e-8])
        dt = frac * _gyroperiod(B)
        phi = -2 * np.pi * dt / _gyroperiod(B)
        L, t = _orc_transform(orc_dp, B, V, dt)
        np.testing.assert_allclose(L, rotation([0, 0, 1], phi), atol=1e-13)
        got = orc_dp.cell_intersections(L, t, mesh, map_order)
        want = intersections_b_along_z(phi, V, mesh.vmin, dv, map_order)
        _close(got, want, 1e-12)
