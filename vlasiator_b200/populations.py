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


def acceleration_subcycles(dt: float, max_v_dt) -> int:
    """Global subcycle count (getAccelerationSubcycles, vlasovmover.cpp:398-401,
    maxed over cells as vlasovmover.cpp:527-545 does)."""
    return max(1, max(int(math.ceil(abs(dt) / float(m))) for m in np.atleast_1d(max_v_dt)))


def subcycle_dt(step: int, dt: float, max_v_dt) -> np.ndarray:
    """Per-cell dt of subcycle `step` (calculateAcceleration, vlasovmover.cpp:
    428-456): max_v_dt on every step but the last, which takes the rest;
    zero once a cell has covered |dt|; the sign of dt."""
    m = np.asarray(max_v_dt, np.float64)
    this = np.where((step + 1) * m > abs(dt), np.maximum(abs(dt) - step * m, 0.0), m)
    return -this if dt < 0 else this


def accelerate_subcycled(batch, B, dt: float, max_v_dt, map_orders) -> int:
    """Acceleration over dt in subcycles of at most max_v_dt per cell, each a
    full vlgpu_accelerate step (pivot moments, three sweeps, block adjustment,
    moments).  Cells that have covered dt before the last subcycle take dt = 0
    steps, where the reference leaves them out of the accelerated cells.
    Returns the number of subcycles."""
    n = acceleration_subcycles(dt, max_v_dt)
    for s in range(n):
        batch.accelerate(B, subcycle_dt(s, dt, max_v_dt), map_orders[s % len(map_orders)])
    return n
