"""Closed forms and an independent implementation of the SLICE-3D geometry,
used by the geometry tests to pin the oracle's FP64 restatement and the
device geometry.

The reference builds the gyration transform with Eigen
(vlasovsolver/cpu_acc_transform.cpp:66-153): N substeps of a rotation by
-2 pi dt / (T_g N) about unit B, each about a pivot p_i = T_i(V) - h that
follows the bulk velocity V through the transform built so far (h is the Hall
term, curl(B) / (mu0 rhoq)).  The pivot recursion has a closed form:
T_{i+1}(V) = T_i(V) + (R1 - I) h, so with R1 the substep rotation,
    T_N(x) = R x + c,   R = R1^N = rotation by -2 pi dt / T_g,
    c = sum_i R1^(N-1-i) (I - R1) (V + i (R1 - I) h - h),
which reduces to c = V - R V (the pivot is a fixed point) without a Hall term.

The intersections (vlasovsolver/cpu_acc_intersections.cpp:132-450) are
line-plane intersections of the Euclidean grid with the grid moved by the
backward transform; `intersections` below restates their definitions with a
generic solver on the 4x4 affine matrices, independently of the oracle's C.
"""
import numpy as np

from vlasiator_b200.mesh import MU_0


def rotation(axis, angle):
    """Rotation matrix by `angle` about the unit vector `axis` (Rodrigues)."""
    a = np.asarray(axis, float)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + np.sin(angle) * K + (1 - np.cos(angle)) * (K @ K)


def transform(B, V, dt, q, m, curl=(0, 0, 0), rhoq=0.0, hall_min_rhoq=1.60217653e-19, mu0=MU_0):
    """Closed form of the forward transform: (R, c) with T(x) = R x + c."""
    B = np.asarray(B, float)
    bmag = np.linalg.norm(B) + 1e-30
    n = B / np.linalg.norm(B) if bmag >= 1e-28 else np.array([0.0, 0.0, 1.0])
    Tg = 2 * np.pi * m / (q * bmag)
    N = max(1, int(abs(dt) / abs(Tg * (0.1 / 360.0))))
    phi = -2 * np.pi * dt / Tg
    R1 = rotation(n, phi / N)
    rq = rhoq + 1e10 * np.finfo(float).tiny
    hall = np.asarray(curl, float) / (mu0 * (hall_min_rhoq if rq <= hall_min_rhoq else rq))
    I3 = np.eye(3)
    V = np.asarray(V, float)
    c = np.zeros(3)
    Rk = I3.copy()  # R1^(N-1-i), built from the last term backwards
    for i in range(N - 1, -1, -1):
        p = V + i * ((R1 - I3) @ hall) - hall
        c += Rk @ ((I3 - R1) @ p)
        Rk = Rk @ R1
    return rotation(n, phi), c


def _affine(L, t):
    A = np.eye(4)
    A[:3, :3] = L
    A[:3, 3] = t
    return A


def _plane_cut(lp, d, pp, n):
    """The point where the line lp + s d meets the plane through pp with normal n."""
    return lp + (np.dot(n, pp - lp) / np.dot(n, d)) * d


def intersections(L, t, vmin, dv, map_order):
    """The 12 intersections (x, y, z; each intersection, di, dj, dk) of a map
    order from the forward transform (L, t), the mesh origin vmin and the cell
    size dv (per axis)."""
    bwd = np.linalg.inv(_affine(L, t))
    Bl = bwd[:3, :3]
    vmin = np.asarray(vmin, float)
    dv = np.asarray(dv, float)
    e = np.eye(3)

    def B(x):
        return bwd[:3, :3] @ x + bwd[:3, 3]

    def cell(frac):
        return vmin + np.asarray(frac, float) * dv

    def four(p000, p100, p010, p001, d):
        return np.array([p000[d], p100[d] - p000[d], p010[d] - p000[d], p001[d] - p000[d]])

    def first(d):
        # Euclidean lines along d through the cell centres, Lagrangian planes normal to d
        n = Bl @ e[d]
        pp = B(np.where(np.arange(3) == d, vmin, 0.0))
        lp = np.where(np.arange(3) == d, 0.0, vmin + 0.5 * dv)
        steps = [dv[q] * e[q] for q in range(3)]
        cuts = [_plane_cut(lp, e[d], pp, n)]
        for q in range(3):
            if q == d:
                cuts.append(_plane_cut(lp, e[d], pp + Bl @ steps[q], n))
            else:
                cuts.append(_plane_cut(lp + steps[q], e[d], pp, n))
        return four(*cuts, d)

    def second(d):
        # Lagrangian lines along the third sweep's axis u, Euclidean planes normal to u
        u = {0: 1, 1: 2, 2: 0}[d]
        n = e[u]
        pp = 0.5 * dv[u] * e[u] + vmin[u] * e[u]
        ld = Bl @ e[u]
        frac = np.full(3, 0.5)
        frac[d] = 0.0
        lp = B(cell(frac))
        cuts = [_plane_cut(lp, ld, pp, n)]
        for q in range(3):
            if q == u:
                cuts.append(_plane_cut(lp, ld, pp + dv[q] * e[q], n))
            else:
                cuts.append(_plane_cut(lp + Bl @ (dv[q] * e[q]), ld, pp, n))
        return four(*cuts, d)

    def third(d):
        # the backward-moved grid points themselves
        frac = np.full(3, 0.5)
        frac[d] = 0.0
        pts = [B(cell(frac))]
        for q in range(3):
            f = frac.copy()
            f[q] += 1.0
            pts.append(B(cell(f)))
        return four(*pts, d)

    order = [[0, 1, 2], [1, 2, 0], [2, 0, 1]][map_order]
    out = np.zeros(12)
    for stage, d in enumerate(order):
        out[4 * d:4 * d + 4] = (first, second, third)[stage](d)
    return out


def intersections_b_along_z(phi, V, vmin, dv, map_order):
    """Closed forms of the intersections for a rotation by phi about +z with
    pivot V (c = cos phi, s = sin phi; the backward transform rotates by
    -phi), uniform cell size dv."""
    c, s = np.cos(phi), np.sin(phi)
    V = np.asarray(V, float)
    xm, ym, zm = vmin
    h = 0.5 * dv
    z = np.array([zm, 0.0, 0.0, dv])
    if map_order in (0, 2):
        # x: Euclidean x lines meet the Lagrangian x planes (order 0) or the
        # Lagrangian y lines meet the Euclidean y planes (order 2)
        X, Y = xm - V[0], ym + h - V[1]
        x = np.array([V[0] + (X + s * Y) / c, dv / c, s / c * dv, 0.0])
        # y: the Lagrangian z lines (order 0) or the moved grid points (order 2)
        X2, Y2 = xm + h - V[0], ym - V[1]
        y = np.array([V[1] - s * X2 + c * Y2, -s * dv, c * dv, 0.0])
    else:
        # y first: Euclidean y lines meet the Lagrangian y planes
        X0, Y0 = xm + h - V[0], ym - V[1]
        y = np.array([V[1] + (Y0 - s * X0) / c, -s / c * dv, dv / c, 0.0])
        # x third: the moved grid points
        X3, Y3 = xm - V[0], ym + h - V[1]
        x = np.array([V[0] + c * X3 + s * Y3, c * dv, s * dv, 0.0])
    return np.concatenate([x, y, z])
