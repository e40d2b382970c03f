"""Several particle populations and acceleration subcycling on top of batches.

The reference keeps one velocity mesh per population and loops over the
populations in its drivers (vlasovmover.cpp:503-565, arch_moments.cpp:342-
499); here a population is one batch (its own mesh, mass and charge), and
these helpers do the per-cell bookkeeping that spans populations or
subcycles.
"""
from __future__ import annotations

import math

import numpy as np

# columns of a batch's 16-double moment record
N, NVX, NVY, NVZ, RHOM, VX, VY, VZ, RHOQ, P11, P22, P33, P23, P13, P12, MASS = range(16)


def combine_moments(records, masses, charges) -> np.ndarray:
    """Cell moments over populations as calculateMoments_V / _R form them
    (arch_moments.cpp:342-499): RHOM and RHOQ are sums over populations, the
    bulk velocity is mass-weighted, and each population's pressure is taken
    about the cell's (all-population) bulk velocity and summed.

    records: per population an (n_cells, 16) moment record of one batch, whose
    pressure is about the population's own bulk velocity.  Returns
    (n_cells, 11): RHOM, VX, VY, VZ, RHOQ, P11, P22, P33, P23, P13, P12."""
    recs = [np.asarray(r, np.float64) for r in records]
    n_cells = recs[0].shape[0]
    out = np.zeros((n_cells, 11))
    rhom = sum(r[:, N] * m for r, m in zip(recs, masses))
    mom = sum(r[:, NVX:NVZ + 1] * m for r, m in zip(recs, masses))
    with np.errstate(divide="ignore", invalid="ignore"):
        V = np.where(rhom[:, None] != 0, mom / rhom[:, None], 0.0)
    out[:, 0] = rhom
    out[:, 1:4] = V
    out[:, 4] = sum(r[:, N] * q for r, q in zip(recs, charges))
    # P about W = P about the population's own V + m n (V_p - W)(V_p - W)
    pairs = [(0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1)]
    for r, m in zip(recs, masses):
        d = r[:, VX:VZ + 1] - V
        for q, (a, b) in enumerate(pairs):
            out[:, 5 + q] += r[:, P11 + q] + m * r[:, N] * d[:, a] * d[:, b]
    return out


def cell_subcycles(dt: float, max_v_dt) -> np.ndarray:
    """Subcycles per cell, getAccelerationSubcycles (vlasovmover.cpp:398-401):
    max(ceil(dt / max_v_dt), 1), with dt signed as the reference passes it."""
    m = np.atleast_1d(np.asarray(max_v_dt, np.float64))
    return np.maximum(np.ceil(dt / m), 1).astype(np.int64)


def acceleration_subcycles(dt: float, max_v_dt) -> int:
    """Global subcycle count: the maximum over cells (vlasovmover.cpp:527-545)."""
    return int(cell_subcycles(dt, max_v_dt).max())


def subcycle_dt(step: int, dt: float, max_v_dt) -> np.ndarray:
    """Per-cell dt of subcycle `step` (calculateAcceleration, vlasovmover.cpp:
    428-456): max_v_dt on every step but the last, which takes the rest, with
    the sign of dt; zero for a cell whose subcycles are done (the reference
    leaves it out of the accelerated cells, vlasovmover.cpp:547-556)."""
    m = np.atleast_1d(np.asarray(max_v_dt, np.float64))
    this = np.where((step + 1) * m > abs(dt), np.maximum(abs(dt) - step * m, 0.0), m)
    this = np.where(step < cell_subcycles(dt, m), this, 0.0)
    return -this if dt < 0 else this


# std::minstd_rand0 (std::default_random_engine of the GNU C++ library):
# x <- 16807 x mod (2^31 - 1), seeded with s mod (2^31 - 1) (1 for 0)
_MINSTD_A, _MINSTD_M = 16807, 2147483647


def map_order_for_step(tstep: int) -> int:
    """The dimension order of every subcycle of time step `tstep`
    (calculateAcceleration, vlasovmover.cpp:422-426): one draw of
    uniform_int_distribution<>(0, 2) from a default_random_engine seeded with
    the step number.  The GNU C++ library's distribution scales down the
    engine's range [1, 2^31 - 2] by (range // 3), rejecting draws past 3 times
    that."""
    x = tstep % _MINSTD_M
    if x == 0:
        x = 1
    urange = _MINSTD_M - 2 - 1          # engine max - min
    scaling = urange // 3
    past = 3 * scaling
    while True:
        x = (_MINSTD_A * x) % _MINSTD_M
        r = x - 1
        if r < past:
            return r // scaling


def accelerate_subcycled(batch, B, dt: float, max_v_dt, map_order: int) -> int:
    """Acceleration of one population over dt in subcycles of at most max_v_dt
    per cell, as calculateAcceleration does it (vlasovmover.cpp:503-565): all
    subcycles of the step in one dimension order (map_order_for_step), each a
    full vlgpu_accelerate step (pivot moments, three sweeps, block adjustment,
    moments).  A cell whose subcycles are done gets dt = 0 and passes through
    unchanged; the adjustment that follows the last subcycle is the
    reference's final adjustVelocityBlocks of all cells, and adjusting an
    already adjusted cell changes nothing.  Returns the number of subcycles."""
    n = acceleration_subcycles(dt, max_v_dt)
    for s in range(n):
        batch.accelerate(B, subcycle_dt(s, dt, max_v_dt), map_order)
    return n
