"""The pressure tensor of the single-read moments launch, restated in numpy
(FP64, the order of the device's per-block sums does not matter here): the
second sums are taken about a reference velocity U that is not the bulk
velocity V (a previous step's, or zero), and the correction uses the first
sums about U, T_a = S_a - U_a S0, formed from first sums taken about 0.  The
two-pass reference (V first, then sum f (v-V)(v-V), arch_moments.h:83-155)
is matched to about eps (|U - V| / v_th)^2 and eps (|U| / v_th)^2, which is
what the kernel's comment claims."""
import numpy as np
import pytest

from vlasiator_b200.mesh import MASS_PROTON, VelocityMesh
from vlasiator_b200.projects import maxwellian_cell


def cell_velocities(mesh, gids):
    """Velocity of every phase-space cell of the blocks (64 per block, x fastest)."""
    g = gids.astype(np.int64)
    L0, L1 = mesh.length[0], mesh.length[1]
    bi, bj, bk = g % L0, (g // L0) % L1, g // (L0 * L1)
    dv = [mesh.block_size[d] / 4 for d in range(3)]
    c = np.arange(64)
    ci, cj, ck = c % 4, (c // 4) % 4, c // 16
    vx = mesh.vmin[0] + bi[:, None] * mesh.block_size[0] + (ci[None, :] + 0.5) * dv[0]
    vy = mesh.vmin[1] + bj[:, None] * mesh.block_size[1] + (cj[None, :] + 0.5) * dv[1]
    vz = mesh.vmin[2] + bk[:, None] * mesh.block_size[2] + (ck[None, :] + 0.5) * dv[2]
    return vx, vy, vz


def pressure_two_pass(f, v):
    S0 = f.sum()
    V = [(f * vi).sum() / S0 for vi in v]
    return np.array([(f * (v[a] - V[a]) * (v[b] - V[b])).sum() for a, b in
                     [(0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1)]]), V


def pressure_single_read(f, v, U):
    S0 = f.sum()
    S = [(f * vi).sum() for vi in v]                      # first sums about 0
    T = [S[a] - U[a] * S0 for a in range(3)]              # first sums about U
    w = [v[a] - U[a] for a in range(3)]
    out = []
    for a, b in [(0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1)]:
        Sab = (f * w[a] * w[b]).sum()                     # second sums about U
        out.append(Sab - T[a] * T[b] / S0)
    return np.array(out)


@pytest.mark.parametrize("T,V,shift", [(1e6, (4e5, 0, 0), "stale"), (1e6, (4e5, 0, 0), "zero"),
                                       (1e5, (8e5, -3e5, 2e5), "stale"), (1e5, (8e5, -3e5, 2e5), "zero"),
                                       (1e7, (0, 0, 0), "zero")])
def test_single_read_pressure_matches_two_pass(T, V, shift):
    mesh = VelocityMesh()
    c = maxwellian_cell(mesh, 1e6, T, V, dtype=np.float64)
    f = c.data.astype(np.float64)
    v = cell_velocities(mesh, c.gids)
    P_ref, Vb = pressure_two_pass(f, v)
    U = [0.9 * Vb[a] + 1e4 for a in range(3)] if shift == "stale" else [0.0, 0.0, 0.0]
    P = pressure_single_read(f, v, U)
    vth = np.sqrt(2 * 1.380649e-23 * T / MASS_PROTON)
    bound = 64 * np.finfo(np.float64).eps * (1 + (np.linalg.norm(np.subtract(U, Vb)) / vth) ** 2)
    scale = np.abs(P_ref[:3]).max()
    assert np.abs(P - P_ref).max() <= bound * scale
