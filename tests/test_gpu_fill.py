"""Initial VDFs generated on the device (vlgpu_batch_fill_maxwellian) against
the host generator of the same project functions (projects.maxwellian_cell:
MaxwellianPhaseSpaceDensity / TriMaxwellianPhaseSpaceDensity at cell centres,
then the first block adjustment)."""
import numpy as np
import pytest

from vlasiator_b200.projects import maxwellian_cell

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def vl():
    from vlasiator_b200 import vlgpu
    vlgpu.load()
    return vlgpu


def _compare(got, ref, what):
    for ci, ((g1, d1), c) in enumerate(zip(got, ref)):
        np.testing.assert_array_equal(g1, c.gids, err_msg=f"{what}: cell {ci}")
        np.testing.assert_allclose(d1, c.data, rtol=2e-7, atol=0, err_msg=f"{what}: cell {ci}")


def test_isotropic_fill_matches_host_generator(vl, mesh):
    rng = np.random.default_rng(6)
    k = 12
    n = 10 ** rng.uniform(5, 7, k)
    T = 10 ** rng.uniform(5, 6.7, k)
    V = rng.normal(size=(k, 3)) * 2e5
    ref = [maxwellian_cell(mesh, n[c], T[c], V[c]) for c in range(k)]
    with vl.Batch(mesh, k, 3 * sum(c.n_blocks for c in ref) + 300000) as b:
        b.fill_maxwellian(n, T, V)
        got = b.cells()
        assert not b.status().any()
        assert (b.rho_loss() == 0).all()
    _compare(got, ref, "isotropic")


def test_trimaxwellian_fill_matches_host_generator(vl, mesh):
    rng = np.random.default_rng(7)
    k = 6
    ref, Ts, frames, V = [], [], [], rng.normal(size=(k, 3)) * 1e5
    for c in range(k):
        b = rng.normal(size=3)
        b /= np.linalg.norm(b)
        e1 = np.cross(b, [1.0, 0.0, 0.0])
        e1 /= np.linalg.norm(e1)
        R = np.stack([e1, np.cross(b, e1), b])
        Tp = 10 ** rng.uniform(5.2, 6.0)
        T3 = (Tp, Tp, rng.uniform(0.5, 3.0) * Tp)
        ref.append(maxwellian_cell(mesh, 1e6, Tp, V[c], T_aniso=(*T3, R)))
        Ts.append(T3)
        frames.append(R)
    with vl.Batch(mesh, k, 3 * sum(c.n_blocks for c in ref) + 300000) as b:
        b.fill_maxwellian(np.full(k, 1e6), np.array(Ts), V, frame=np.array(frames))
        got = b.cells()
    _compare(got, ref, "tri-Maxwellian")


def test_fill_on_a_grid_adds_the_neighbours_content(vl, mesh):
    from vlasiator_b200.projects import sinewave_grid
    dims = (4, 1, 1)
    ref = sinewave_grid(dims, mesh)
    nx = dims[0]
    n = [1e6 * (1 + 0.5 * np.sin(2 * np.pi * x / nx)) for x in range(nx)]
    with vl.Batch(mesh, nx, 4 * sum(c.n_blocks for c in ref) + 300000) as b:
        b.set_grid(dims, 3e5)
        b.fill_maxwellian(n, 1e6, (4e5, 0, 0))
        got = b.cells()
    for ci, ((g1, _), c) in enumerate(zip(got, ref)):
        assert set(c.gids.tolist()) <= set(g1.tolist())
        nb = [(ci - 1) % nx, (ci + 1) % nx]
        content_n = set().union(*[set(ref[j].gids[(ref[j].data >= 1e-15).any(1)].tolist()) for j in nb])
        assert set(g1.tolist()) == set(c.gids.tolist()) | content_n
