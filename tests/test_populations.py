"""Population and subcycle bookkeeping (host logic, no GPU): combining
per-population moment records into cell moments, and the subcycle dt
sequence of calculateAcceleration."""
import numpy as np

from vlasiator_b200.populations import acceleration_subcycles, combine_moments, subcycle_dt


def _record(n, V, P_own):
    r = np.zeros(16)
    r[0] = n
    r[1:4] = n * np.asarray(V)
    r[5:8] = V
    r[9:15] = P_own
    return r


def test_combine_moments_matches_direct_sums():
    rng = np.random.default_rng(4)
    m = [1.67e-27, 6.64e-27]
    q = [1.6e-19, 3.2e-19]
    # two populations of point-like particle sets: compute everything directly
    parts = [rng.normal(size=(500, 3)) * 1e5 + [4e5, 0, 0], rng.normal(size=(300, 3)) * 3e4 - [1e5, 2e5, 0]]
    w = [rng.uniform(0.5, 1.5, 500), rng.uniform(0.5, 1.5, 300)]
    recs = []
    for p, ww, mm in zip(parts, w, m):
        n = ww.sum()
        V = (ww[:, None] * p).sum(0) / n
        d = p - V
        P = [mm * (ww * d[:, a] * d[:, b]).sum() for a, b in [(0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1)]]
        recs.append(_record(n, V, P)[None, :])
    out = combine_moments(recs, m, q)[0]
    rhom = sum(ww.sum() * mm for ww, mm in zip(w, m))
    Vc = sum((ww[:, None] * p).sum(0) * mm for p, ww, mm in zip(parts, w, m)) / rhom
    Pc = [sum(mm * (ww * (p - Vc)[:, a] * (p - Vc)[:, b]).sum() for p, ww, mm in zip(parts, w, m))
          for a, b in [(0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1)]]
    np.testing.assert_allclose(out[0], rhom, rtol=1e-12)
    np.testing.assert_allclose(out[1:4], Vc, rtol=1e-10)
    np.testing.assert_allclose(out[4], sum(ww.sum() * qq for ww, qq in zip(w, q)), rtol=1e-12)
    np.testing.assert_allclose(out[5:11], Pc, rtol=1e-9, atol=1e-12 * max(abs(x) for x in Pc))


def test_subcycle_sequence():
    mvdt = np.array([0.4, 1.0, 0.25])
    dt = 0.9
    n = acceleration_subcycles(dt, mvdt)
    assert n == 4
    steps = np.stack([subcycle_dt(s, dt, mvdt) for s in range(n)])
    np.testing.assert_allclose(steps.sum(0), dt)
    np.testing.assert_allclose(steps[:, 0], [0.4, 0.4, 0.1, 0.0])
    np.testing.assert_allclose(steps[:, 1], [0.9, 0.0, 0.0, 0.0])
    assert (subcycle_dt(0, -dt, mvdt) <= 0).all()


def test_subcycle_counts_follow_the_reference_formula():
    # getAccelerationSubcycles takes ceil(dt / max_v_dt) of the signed dt
    # (vlasovmover.cpp:398-401): a negative dt gives one subcycle
    from vlasiator_b200.populations import cell_subcycles
    m = np.array([0.4, 1.0, 0.25])
    np.testing.assert_array_equal(cell_subcycles(0.9, m), [3, 1, 4])
    np.testing.assert_array_equal(cell_subcycles(0.8, m), [2, 1, 4])
    np.testing.assert_array_equal(cell_subcycles(-0.9, m), [1, 1, 1])


def test_map_order_matches_the_reference_draw():
    """map_order_for_step against the reference's own draw
    (vlasovmover.cpp:422-426) compiled with this machine's C++ library."""
    import pytest

    from oracle.oracle import ReferenceBuild, reference_available
    from vlasiator_b200.populations import map_order_for_step
    if not reference_available("sp"):
        pytest.skip("reference build (oracle/_ref) not present")
    ref = ReferenceBuild("sp")
    # the first draw is 16807 t: every step below about 42,590 gets order 0
    steps = list(range(0, 200)) + list(range(40000, 2000000, 7919)) + [2 ** 31 - 2, 2 ** 31 - 1, 123456789]
    got = [map_order_for_step(t) for t in steps]
    assert got == [ref.map_order(t) for t in steps]
    assert set(got) == {0, 1, 2}
    assert set(got[:200]) == {0}
