"""Parity on the benchmark workloads themselves, against the reference's own
code (oracle/_ref: map_1d, cpu_acc_map.cpp:121-636; adjust_velocity_blocks,
spatial_cell_cpu.cpp:179-273; the moment templates, arch_moments.h:83-155;
the geometry from the oracle's pinned FP64 restatement).

- The batched-acceleration workload: the first 64 cells of bench.py's 4096
  (its generator is prefix-stable, tests/test_configs_host.py), with the
  bench's seed and first dimension order; one full acceleration step.
- The single-cell Larmor case: ten acceleration steps of the gyrating
  Maxwellian, dt = 0.01 gyroperiod, in the dimension order the reference
  draws for steps 1..10.

Tolerances: exact arithmetic is bit-exact wherever the device's FP64
geometry gives the same Realf intersections as the host's; the fused
arithmetic is held to 1e-5 of each cell's peak per step, and mass to 1e-6 per
step (the adjustment's loss accounted).
"""
import numpy as np
import pytest

import bench
from oracle.oracle import ReferenceBuild, reference_available
from vlasiator_b200.mesh import CHARGE, MASS_PROTON
from vlasiator_b200.populations import map_order_for_step
from vlasiator_b200.projects import larmor_cell

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not reference_available("sp"), reason="reference build (oracle/_ref) not present")]

N_SAMPLE = 64


@pytest.fixture(scope="module")
def vl():
    from vlasiator_b200 import vlgpu
    vlgpu.load()
    return vlgpu


@pytest.fixture(scope="module")
def bench_sample():
    mesh, offs, gids, data, B, dt = bench.workload(N_SAMPLE, bench.DEFAULT_SEED)
    g = [gids[offs[c]:offs[c + 1]] for c in range(N_SAMPLE)]
    d = [data[offs[c]:offs[c + 1]] for c in range(N_SAMPLE)]
    mo = bench.map_orders(1, bench.DEFAULT_SEED)[0]
    return mesh, g, d, B, dt, mo


def _reference_steps(mesh, g, d, B, dt_steps, orders):
    """The reference's acceleration steps: pivot moments, geometry, map_1d x3
    (ref_cells_accelerate_step), then adjust_velocity_blocks without spatial
    neighbours; returns sorted cells, total loss and moments per cell."""
    ref = ReferenceBuild("sp")
    ref.init(mesh)
    n = len(g)
    h = ref.create(g, d, [1e-15] * n)
    try:
        loss = np.zeros(n)
        for dt, mo in zip(dt_steps, orders):
            ref.accelerate_step(h, B, dt, mo, CHARGE, MASS_PROTON)
            loss += ref.adjust(h, n, 1e-15)
        cells = [ref.extract(h, c) for c in range(n)]
        mom = []
        for c in range(n):
            first, _ = ref.moments(h, c, np.zeros(3))
            V = first[1:4] / first[0]
            _, second = ref.moments(h, c, V)
            mom.append((first[0], V, MASS_PROTON * second))
    finally:
        ref.destroy(h)
    assert ref.bailouts() == 0
    return cells, loss, mom


def _device_steps(vl, mesh, g, d, B, dt_steps, orders, exact):
    total = sum(len(x) for x in g)
    with vl.Batch(mesh, len(g), 4 * total + 65536, exact=exact) as b:
        b.upload(g, d)
        sums = [np.array([x.astype(np.float64).sum() for x in d])]
        loss = []
        for dt, mo in zip(dt_steps, orders):
            b.accelerate(B, dt, mo)
            m = b.moments(second=True)
            sums.append(m[:, 15])
            loss.append(b.rho_loss().copy())
        out = dict(cells=b.cells(), moments=b.moments(second=True), loss=b.rho_loss(), sums=np.stack(sums),
                   step_loss=np.stack(loss), status=b.status())
    assert not out["status"].any()
    return out


def _compare(got_cells, ref_cells, tol_peak):
    """Number of cells bit-identical to the reference; the others within
    tol_peak of their peak on the common blocks."""
    exact = 0
    for ci, ((g1, d1), (g2, d2)) in enumerate(zip(got_cells, ref_cells)):
        if np.array_equal(g1, g2) and np.array_equal(d1, d2):
            exact += 1
            continue
        common = np.intersect1d(g1, g2)
        assert len(common) >= 0.99 * max(len(g1), len(g2)), f"cell {ci}: block sets differ"
        i1, i2 = np.searchsorted(g1, common), np.searchsorted(g2, common)
        peak = float(np.abs(d2).max())
        err = float(np.abs(d1[i1] - d2[i2]).max())
        assert err <= tol_peak * peak, f"cell {ci}: {err / peak:.2e} of peak"
    return exact


def _check_moments(got, ref_mom, rtol_n, rtol_p):
    for ci, (n, V, P) in enumerate(ref_mom):
        m = got[ci]
        assert m[0] == pytest.approx(n, rel=rtol_n)
        # bulk velocity relative to a thermal-speed scale (1e5 m/s) or |V|
        np.testing.assert_allclose(m[5:8], V, rtol=0, atol=rtol_n * (np.abs(V).max() + 1e5))
        scale = np.abs(P[:3]).max()
        np.testing.assert_allclose(m[9:15], P, rtol=0, atol=rtol_p * scale)


def test_bench_sample_exact_matches_reference(vl, bench_sample):
    mesh, g, d, B, dt, mo = bench_sample
    ref_cells, ref_loss, ref_mom = _reference_steps(mesh, g, d, B, [dt], [mo])
    got = _device_steps(vl, mesh, g, d, B, [dt], [mo], exact=True)
    exact = _compare(got["cells"], ref_cells, 1e-5)
    assert exact >= N_SAMPLE - 2
    np.testing.assert_allclose(got["loss"], ref_loss, rtol=1e-9, atol=1e-30)
    _check_moments(got["moments"], ref_mom, 1e-10, 1e-9)


def test_bench_sample_fused_within_tolerance(vl, bench_sample):
    mesh, g, d, B, dt, mo = bench_sample
    ref_cells, ref_loss, ref_mom = _reference_steps(mesh, g, d, B, [dt], [mo])
    got = _device_steps(vl, mesh, g, d, B, [dt], [mo], exact=False)
    _compare(got["cells"], ref_cells, 1e-5)
    dv3 = float(np.prod(mesh.dv))
    before, after = got["sums"][0], got["sums"][1]
    # the device's own mass balance: what the step kept plus what the
    # adjustment removed is what went in
    np.testing.assert_allclose(after + got["loss"] / dv3, before, rtol=1e-6)
    ref_after = np.array([x.astype(np.float64).sum() for _, x in ref_cells])
    np.testing.assert_allclose(after, ref_after, rtol=1e-6)
    _check_moments(got["moments"], ref_mom, 1e-6, 1e-5)


@pytest.mark.parametrize("exact", [True, False])
def test_larmor_ten_steps_match_reference(vl, mesh, exact):
    c = larmor_cell()
    Tg = 2 * np.pi * MASS_PROTON / (CHARGE * np.linalg.norm(c.B))
    steps = 10
    dts = [np.array([0.01 * Tg])] * steps
    orders = [map_order_for_step(t) for t in range(1, steps + 1)]
    ref_cells, ref_loss, ref_mom = _reference_steps(mesh, [c.gids], [c.data], c.B[None, :], dts, orders)
    got = _device_steps(vl, mesh, [c.gids], [c.data], c.B[None, :], dts, orders, exact=exact)
    if exact:
        assert _compare(got["cells"], ref_cells, 1e-5) == 1
        np.testing.assert_allclose(got["loss"], ref_loss, rtol=1e-9, atol=1e-30)
        _check_moments(got["moments"], ref_mom, 1e-10, 1e-9)
    else:
        # per-step differences of up to 1e-5 of the peak, over ten steps
        _compare(got["cells"], ref_cells, 1e-4)
        _check_moments(got["moments"], ref_mom, 1e-5, 1e-4)
    dv3 = float(np.prod(mesh.dv))
    sums, step_loss = got["sums"], got["step_loss"]
    for s in range(steps):
        lost = (step_loss[s] - (step_loss[s - 1] if s else 0.0)) / dv3
        assert abs(sums[s + 1][0] + lost[0] - sums[s][0]) <= 1e-6 * sums[s][0], f"step {s}"


@pytest.mark.parametrize("exact", [True, False])
def test_wide_cell_matches_reference(vl, mesh, exact):
    """A hot cell (T = 60 MK, about 40 x 40 blocks across) among ordinary
    cells: its transverse planes exceed the columnize launch's shared-memory
    plane, so its sweeps go through the wide-plane kernel, and its dilated box
    exceeds the adjustment's shared-memory rows, so it is adjusted with the
    global scratch masks; one full acceleration step against the reference's."""
    from vlasiator_b200.projects import maxwellian_cell, random_drifting_cells
    cells = random_drifting_cells(5, seed=31, mesh=mesh)
    hot = maxwellian_cell(mesh, 1e6, 6e7, (2e5, -1e5, 1e5))
    hot.B = np.array([1e-8, 2e-8, -3e-8])
    cells.append(hot)
    g = [c.gids for c in cells]
    d = [c.data for c in cells]
    L = mesh.length
    y, z = (hot.gids // L[0]) % L[1], hot.gids // (L[0] * L[1])
    assert (np.ptp(y) + 1) * (np.ptp(z) + 1) > 1024 and (np.ptp(y) + 3) * (np.ptp(z) + 3) > 1600
    B = np.stack([c.B for c in cells])
    dt = 0.01 * 2 * np.pi * MASS_PROTON / (CHARGE * np.linalg.norm(B, axis=1))
    ref_cells, ref_loss, ref_mom = _reference_steps(mesh, g, d, B, [dt], [1])
    got = _device_steps(vl, mesh, g, d, B, [dt], [1], exact=exact)
    if exact:
        assert _compare(got["cells"], ref_cells, 1e-5) >= len(cells) - 1
        np.testing.assert_allclose(got["loss"], ref_loss, rtol=1e-9, atol=1e-30)
        _check_moments(got["moments"], ref_mom, 1e-10, 1e-9)
    else:
        _compare(got["cells"], ref_cells, 1e-5)
        _check_moments(got["moments"], ref_mom, 1e-6, 1e-5)
