"""Synthetic initial conditions: sparse Maxwellian velocity distributions.

Follows the reference's initial-condition path for one population:
``Project::setVelocitySpace`` (projects/project.cpp:239-260) fills every
block of the mesh with ``MaxwellianPhaseSpaceDensity`` (projects/project.h:45-51)
sampled at cell centres, and the first ``adjustVelocityBlocks``
(grid.cpp:289) keeps the blocks that have content (any cell >= minValue,
spatial_cell_cpu.cpp:290-320) plus their +-1 velocity-space neighbours
(spatial_cell_cpu.cpp:179-273).  Only blocks that can reach minValue are
evaluated, so a cell costs time proportional to its block count.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .mesh import K_B, MASS_PROTON, WID3, VelocityMesh


@dataclass
class CellState:
    """One spatial cell's sparse VDF: global IDs (ascending) and [nb, 64] float32 data."""

    gids: np.ndarray
    data: np.ndarray
    # inputs the acceleration reads from SpatialCell::parameters
    B: np.ndarray = field(default_factory=lambda: np.array([0.0, 0.0, 1e-8]))
    V: np.ndarray = field(default_factory=lambda: np.zeros(3))
    n: float = 1e6
    T: float = 5e5

    @property
    def n_blocks(self) -> int:
        return int(self.gids.shape[0])


def maxwellian_density(vx, vy, vz, n, T, V, mass=MASS_PROTON, T_aniso=None):
    """Phase-space density at the given velocities (double precision).

    ``T_aniso`` = (Tx, Ty, Tz, R) selects the tri-Maxwellian of
    projects/project.h:66-73 evaluated in the frame given by rotation R (3x3,
    rows = frame axes); otherwise the isotropic Maxwellian of project.h:45-51.
    """
    ux, uy, uz = vx - V[0], vy - V[1], vz - V[2]
    if T_aniso is None:
        return n * (mass / (2.0 * np.pi * K_B * T)) ** 1.5 * np.exp(-mass * (ux * ux + uy * uy + uz * uz) / (2.0 * K_B * T))
    Tx, Ty, Tz, R = T_aniso
    a = R[0, 0] * ux + R[0, 1] * uy + R[0, 2] * uz
    b = R[1, 0] * ux + R[1, 1] * uy + R[1, 2] * uz
    c = R[2, 0] * ux + R[2, 1] * uy + R[2, 2] * uz
    return (n * (mass / (2.0 * np.pi * K_B)) ** 1.5
            * np.exp(-mass * (a * a / Tx + b * b / Ty + c * c / Tz) / (2.0 * K_B)) / np.sqrt(Tx * Ty * Tz))


def _dilate(occ: np.ndarray, width: int) -> np.ndarray:
    """3D box dilation of a boolean block grid (the +-addWidthV neighbourhood), clipped at the mesh."""
    out = occ.copy()
    for ax in range(3):
        cur = out.copy()
        for s in range(1, width + 1):
            a = np.zeros_like(cur)
            b = np.zeros_like(cur)
            sl_src = [slice(None)] * 3
            sl_dst = [slice(None)] * 3
            sl_src[ax] = slice(0, -s)
            sl_dst[ax] = slice(s, None)
            a[tuple(sl_dst)] = cur[tuple(sl_src)]
            sl_src[ax] = slice(s, None)
            sl_dst[ax] = slice(0, -s)
            b[tuple(sl_dst)] = cur[tuple(sl_src)]
            out |= a | b
    return out


def maxwellian_cell(mesh: VelocityMesh, n: float, T: float, V, min_value: float = 1e-15, add_width: int = 1,
                    mass: float = MASS_PROTON, T_aniso=None, dtype=np.float32) -> CellState:
    """Sparse Maxwellian cell pruned like the first block adjustment."""
    V = np.asarray(V, dtype=np.float64)
    Tmax = T if T_aniso is None else max(T_aniso[0], T_aniso[1], T_aniso[2])
    peak = n * (mass / (2.0 * np.pi * K_B * Tmax)) ** 1.5
    if T_aniso is not None:
        peak = n * (mass / (2.0 * np.pi * K_B)) ** 1.5 / np.sqrt(T_aniso[0] * T_aniso[1] * T_aniso[2])
    if peak <= min_value:
        radius = 0.0
    else:
        radius = np.sqrt(2.0 * K_B * Tmax / mass * np.log(peak / min_value))
    bs = mesh.block_size
    L = np.array(mesh.length)
    lo = np.floor((V - radius - np.array(mesh.vmin)) / bs).astype(int) - 1
    hi = np.floor((V + radius - np.array(mesh.vmin)) / bs).astype(int) + 1
    lo = np.clip(lo, 0, L - 1)
    hi = np.clip(hi, 0, L - 1)
    ii, jj, kk = np.meshgrid(np.arange(lo[0], hi[0] + 1), np.arange(lo[1], hi[1] + 1), np.arange(lo[2], hi[2] + 1),
                             indexing="ij")
    cand = mesh.gid(ii.ravel(), jj.ravel(), kk.ravel()).astype(np.int64)
    vx, vy, vz = mesh.cell_centres(cand)
    f = maxwellian_density(vx, vy, vz, n, T, V, mass, T_aniso).astype(dtype)
    content = (f >= dtype(min_value)).any(axis=1)
    occ = np.zeros((L[2], L[1], L[0]), dtype=bool)
    ci, cj, ck = mesh.indices(cand[content])
    occ[ck, cj, ci] = True
    keep = _dilate(occ, add_width)
    kz, ky, kx = np.nonzero(keep)
    gids = np.sort(mesh.gid(kx, ky, kz).astype(np.int64))
    # the candidate box already spans one block beyond every content block,
    # so every kept block was evaluated above (cand is sorted by GID)
    order = np.argsort(cand)
    pos = order[np.searchsorted(cand[order], gids)]
    data = f[pos]
    return CellState(gids=gids.astype(np.uint32), data=np.ascontiguousarray(data.reshape(-1, WID3)), V=V.copy(),
                     n=n, T=T)


def larmor_cell(mesh: VelocityMesh | None = None) -> CellState:
    """The single-cell plain-acceleration case: n = 1e6 m^-3, T = 0.5 MK, V = 0,
    B = (0, 0, 10 nT), minValue 1e-15, on the +-4020 km/s, 30 km/s mesh."""
    mesh = mesh or VelocityMesh()
    c = maxwellian_cell(mesh, 1e6, 5e5, (0.0, 0.0, 0.0), 1e-15)
    c.B = np.array([0.0, 0.0, 1e-8])
    return c


def random_drifting_cells(n_cells: int, seed: int = 0, mesh: VelocityMesh | None = None, min_value: float = 1e-15):
    """Independent drifting Maxwellians of the batched-acceleration workload.

    Per cell: n log-uniform in [1e5, 1e7] m^-3, T log-uniform in [1e5, 1e7] K,
    |V| uniform in [0, 800] km/s along a uniform random direction, B along a
    uniform random direction with |B| uniform in [5, 50] nT.
    """
    mesh = mesh or VelocityMesh()
    rng = np.random.default_rng(seed)
    cells = []
    for _ in range(n_cells):
        n = 10.0 ** rng.uniform(5.0, 7.0)
        T = 10.0 ** rng.uniform(5.0, 7.0)
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        V = d * rng.uniform(0.0, 8.0e5)
        b = rng.normal(size=3)
        b /= np.linalg.norm(b)
        B = b * rng.uniform(5e-9, 50e-9)
        c = maxwellian_cell(mesh, n, T, V, min_value)
        c.B = B
        cells.append(c)
    return cells


def sinewave_grid(dims, mesh: VelocityMesh | None = None, n0: float = 1e6, amplitude: float = 0.5, T: float = 1e6,
                  V=(4e5, 0.0, 0.0), B=(0.0, 0.0, 5e-9), min_value: float = 1e-15):
    """The full-Vlasov-step workload on a uniform periodic grid (cells x
    fastest): a Maxwellian per cell with n = n0 (1 + amplitude sin(2 pi x / Lx)),
    temperature T, bulk velocity V and uniform B, as the sine-wave translation
    tests of the reference set it up (testpackage transtest_2_amr_sinewave, on
    a uniform grid).  Cells with equal density share one generated VDF."""
    mesh = mesh or VelocityMesh()
    nx, ny, nz = (int(v) for v in dims)
    by_x = []
    for x in range(nx):
        n = n0 * (1.0 + amplitude * np.sin(2.0 * np.pi * x / nx))
        c = maxwellian_cell(mesh, n, T, V, min_value=min_value)
        c.B = np.asarray(B, np.float64)
        by_x.append(c)
    return [by_x[c % nx] for c in range(nx * ny * nz)]


def _bimaxwellian_blocks(mesh: VelocityMesh, n: float, T_perp: float, T_par: float, min_value: float) -> float:
    """Estimated block count (content plus its +-1 halo) of a bi-Maxwellian."""
    peak = n * (MASS_PROTON / (2.0 * np.pi * K_B)) ** 1.5 / (T_perp * np.sqrt(T_par))
    if peak <= min_value:
        return 0.0
    lg = np.log(peak / min_value)
    r_perp = np.sqrt(2.0 * K_B * T_perp / MASS_PROTON * lg) / mesh.block_size[0]
    r_par = np.sqrt(2.0 * K_B * T_par / MASS_PROTON * lg) / mesh.block_size[0]
    return 4.0 / 3.0 * np.pi * (r_perp + 1.0) ** 2 * (r_par + 1.0)


def serving_requests(n_requests: int, seed: int = 0, mesh: VelocityMesh | None = None, max_steps: int = 100,
                     min_value: float = 1e-15):
    """Independent VDF-advance requests of the serving workload.

    Each: a drifting bi-Maxwellian (tri-Maxwellian of projects/project.h:66-73
    with T_x = T_y = T_perp in the magnetic-field frame), T_par / T_perp
    uniform in [0.5, 3], n = 1e6 m^-3, |V| uniform in [0, 800] km/s along a
    random direction; its block count drawn log-normal (median 5000, clipped
    to 500..60000) and met by choosing T_perp; B of random direction with |B|
    uniform in [5, 50] nT (E = -V x B enters through the gyration about V);
    dt = 0.01 gyroperiod; steps uniform in 1..max_steps.
    Returns dicts with keys cell (CellState), B, dt, steps."""
    from .mesh import CHARGE
    mesh = mesh or VelocityMesh()
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_requests):
        target = float(np.clip(np.exp(rng.normal(np.log(5000.0), 0.8)), 500.0, 60000.0))
        est = target / 1.35  # the ellipsoid-plus-halo estimate runs about 35% below the pruned count
        ratio = rng.uniform(0.5, 3.0)
        n = 1e6
        lo, hi = 1e3, 1e9
        for _ in range(60):  # bisection on T_perp for the target block count
            mid = np.sqrt(lo * hi)
            if _bimaxwellian_blocks(mesh, n, mid, ratio * mid, min_value) < est:
                lo = mid
            else:
                hi = mid
        T_perp = np.sqrt(lo * hi)
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        V = d * rng.uniform(0.0, 8.0e5)
        b = rng.normal(size=3)
        b /= np.linalg.norm(b)
        Bmag = rng.uniform(5e-9, 50e-9)
        e1 = np.cross(b, [1.0, 0.0, 0.0] if abs(b[0]) < 0.9 else [0.0, 1.0, 0.0])
        e1 /= np.linalg.norm(e1)
        e2 = np.cross(b, e1)
        R = np.stack([e1, e2, b])
        cell = maxwellian_cell(mesh, n, T_perp, V, min_value, T_aniso=(T_perp, T_perp, ratio * T_perp, R))
        cell.B = b * Bmag
        Tg = 2.0 * np.pi * MASS_PROTON / (CHARGE * Bmag)
        out.append({"cell": cell, "B": cell.B, "dt": 0.01 * Tg, "steps": int(rng.integers(1, max_steps + 1))})
    return out
