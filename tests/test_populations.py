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
