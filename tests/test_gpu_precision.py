"""Precision study: the FP32 GPU Vlasov step (FP32 VDF, FP64 Kahan moments,
FP64 geometry) against an all-FP64 run of the oracle (Realf = double) on the
sine-wave periodic grid, step after step.

The workload is the precision-study configuration (sine-wave grid, dx = 300
km, T = 1 MK, V = (400, 0, 0) km/s, B = (0, 0, 5 nT), dt = 0.8 x the r-space
CFL limit, 200 steps) on a 6 x 2 x 2 grid instead of 32 x 32 x 8, so that the
FP64 oracle finishes in about a minute on the host cores; the error growth per
step does not depend on the grid size.  Reported per run (printed with -s):
the VDF max |error| relative to the grid's peak, the relative errors of n,
V and the pressure tensor, and the cumulative mass drift (sum f dv^3 plus the
mass removed by block adjustment) of the FP32 run and of the FP64 run.
"""
import os

import numpy as np
import pytest

from vlasiator_b200.mesh import CHARGE, MASS_PROTON, WID3
from vlasiator_b200.projects import sinewave_grid

pytestmark = pytest.mark.gpu

DIMS = (6, 2, 2)
DX = 3e5
STEPS = int(os.environ.get("VLGPU_PRECISION_STEPS", "200"))


def r_dt(mesh, cells):
    eps = np.finfo(np.float64).tiny * 1000
    bs = [(mesh.vmax[d] - mesh.vmin[d]) / mesh.length[d] for d in range(3)]
    best = np.inf
    for c in cells:
        g = c.gids.astype(np.int64)
        idx = [g % mesh.length[0], (g // mesh.length[0]) % mesh.length[1], g // (mesh.length[0] * mesh.length[1])]
        for i in (0, 3):
            V = [mesh.vmin[d] + idx[d] * bs[d] + (i + 0.5) * bs[d] / 4 + eps for d in range(3)]
            best = min(best, float(np.min([DX / np.abs(v) for v in V])))
    return best


def dv3(mesh):
    return np.prod([(mesh.vmax[d] - mesh.vmin[d]) / mesh.length[d] / 4 for d in range(3)])


@pytest.fixture(scope="module")
def fp64_run(mesh, orc_dp):
    cells = sinewave_grid(DIMS, mesh)
    dt = 0.8 * r_dt(mesh, cells)
    B = np.stack([c.B for c in cells])
    state = [(c.gids, c.data.astype(np.float64)) for c in cells]
    moms, loss_total = [], 0.0
    for s in range(STEPS):
        state, loss, _, mom_v, _ = orc_dp.vlasov_step(mesh, DIMS, state, B, dt, s % 3, (DX, DX, DX), MASS_PROTON,
                                                      CHARGE)
        loss_total += float(loss.sum())
        moms.append(mom_v)
    return dict(cells=cells, dt=dt, B=B, state=state, moments=np.stack(moms), loss=loss_total)


@pytest.mark.parametrize("exact", [False, True])
def test_fp32_gpu_against_fp64_oracle(vl_lib, mesh, fp64_run, exact):
    from vlasiator_b200 import vlgpu
    cells, dt, B = fp64_run["cells"], fp64_run["dt"], fp64_run["B"]
    total = sum(c.n_blocks for c in cells)
    moms = []
    with vlgpu.Batch(mesh, len(cells), 6 * total + 65536, exact=exact) as b:
        b.upload([c.gids for c in cells], [c.data for c in cells])
        b.set_grid(DIMS, DX)
        b.vlasov_step(B, dt, 0)
        moms.append(b.moments(second=True))
        for s in range(1, STEPS):
            b.vlasov_step_device(dt, s % 3)
            moms.append(b.moments(second=True))
        final = b.cells()
        loss32 = float(b.rho_loss().sum())
        b.sync()
        assert not b.status().any()
    moms = np.stack(moms)
    ref = fp64_run["moments"]
    # VDF error at the end, relative to the grid's peak; a block missing on
    # one side counts as zeros
    peak = max(float(np.abs(d).max()) for _, d in fp64_run["state"])
    vdf_err = 0.0
    for (g1, d1), (g2, d2) in zip(final, fp64_run["state"]):
        u = np.union1d(g1, g2)
        a = np.zeros((len(u), WID3))
        c = np.zeros((len(u), WID3))
        a[np.searchsorted(u, g1)] = d1
        c[np.searchsorted(u, g2)] = d2
        vdf_err = max(vdf_err, float(np.abs(a - c).max()))
    vdf_err /= peak
    n_err = np.abs(moms[:, :, 0] / ref[:, :, 0] - 1).max(axis=1)
    v_scale = np.abs(ref[:, :, 5:8]).max()
    v_err = (np.abs(moms[:, :, 5:8] - ref[:, :, 5:8]).max(axis=(1, 2))) / v_scale
    p_scale = np.abs(ref[:, :, 9:12]).max()
    p_err = (np.abs(moms[:, :, 9:15] - ref[:, :, 9:15]).max(axis=(1, 2))) / p_scale
    m0 = sum(float(c.data.astype(np.float64).sum()) for c in cells) * dv3(mesh)
    m32 = sum(float(d.astype(np.float64).sum()) for _, d in final) * dv3(mesh) + loss32
    m64 = sum(float(d.sum()) for _, d in fp64_run["state"]) * dv3(mesh) + fp64_run["loss"]
    drift32, drift64 = m32 / m0 - 1, m64 / m0 - 1
    mode = "exact" if exact else "fused"
    print(f"\nprecision study ({mode} mode: remap and translation, grid {DIMS}, {STEPS} steps, dt {dt:.4f} s):"
          f"\n  VDF max |err| / peak at the end: {vdf_err:.3e}"
          f"\n  n rel err: step 1 {n_err[0]:.2e}, step {STEPS} {n_err[-1]:.2e}, max {n_err.max():.2e}"
          f"\n  V err / max|V|: step 1 {v_err[0]:.2e}, step {STEPS} {v_err[-1]:.2e}"
          f"\n  P err / max|P_ii|: step 1 {p_err[0]:.2e}, step {STEPS} {p_err[-1]:.2e}"
          f"\n  cumulative mass drift: FP32 GPU {drift32:.3e}, FP64 oracle {drift64:.3e}")
    assert vdf_err < 1e-3
    assert n_err.max() < 1e-4 and v_err.max() < 1e-3 and p_err.max() < 1e-3
    assert abs(drift32 - drift64) < 1e-5


@pytest.fixture(scope="module")
def vl_lib():
    from vlasiator_b200 import vlgpu
    return vlgpu.load()
