"""Precision study: the FP32 GPU Vlasov step (FP32 VDF, FP64 Kahan moments,
FP64 geometry) against the reference's own all-FP64 build (Realf = double,
its translation, map_1d, block adjustment and moment templates, OpenMP over
the host cores) on the periodic sine-wave grid, step after step, with the
reference's own FP32 build beside it as the yardstick of what FP32 storage
costs in the reference itself.

The workload is the precision-study configuration: a 32 x 32 x 8 sine-wave
grid (n = 1e6 (1 + 0.5 sin 2 pi x/Lx), T = 1 MK, V = (400, 0, 0) km/s,
B = (0, 0, 5 nT)), dx = 300 km, dt = 0.8 x the r-space CFL limit, map order
s mod 3.  The recorded study runs 200 steps (VLGPU_PRECISION_STEPS=200,
about 20 minutes of the FP64 reference on 16 host cores); by default the test
takes 5 steps.  Reported per step (printed with -s, and written as a table to
$VLGPU_PRECISION_REPORT when set): the relative errors of n, V and the
pressure tensor against the FP64 run and the cumulative mass drift (sum of n
plus the mass removed by block adjustment); at the end the VDF max |error|
relative to the grid's peak.  The FP32 reference yardstick runs 5 steps
(VLGPU_PRECISION_YARDSTICK_STEPS to change it).
"""
import os

import numpy as np
import pytest

from oracle.oracle import ReferenceBuild, grid_neighbors, reference_available
from vlasiator_b200.mesh import CHARGE, MASS_PROTON, WID3
from vlasiator_b200.projects import sinewave_grid

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not reference_available(), reason="reference build missing")]

DIMS = (32, 32, 8)
DX = 3e5
STEPS = int(os.environ.get("VLGPU_PRECISION_STEPS", "5"))
YARDSTICK_STEPS = min(STEPS, int(os.environ.get("VLGPU_PRECISION_YARDSTICK_STEPS", "5")))


def r_dt(mesh, cells):
    """reduce_vlasov_dt (arch_dt.cpp:34-97) over the grid: dx / |v| at the
    centres of every block's first and last cells."""
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


def _dv3(mesh):
    return np.prod([(mesh.vmax[d] - mesh.vmin[d]) / mesh.length[d] / 4 for d in range(3)])


def _split(m):
    """(n, V, P) from the reference's per-cell (sum f dv3, sum f v dv3, sum f (v-V)(v-V) dv3)."""
    n = m[:, 0]
    return n, m[:, 1:4] / n[:, None], MASS_PROTON * m[:, 4:10]


def _reference_run(precision, mesh, cells, dt, steps):
    ref = ReferenceBuild(precision)
    ref.init(mesh)
    n_cells = len(cells)
    h = ref.create([c.gids for c in cells], [c.data for c in cells], [1e-15] * n_cells)
    B = np.stack([c.B for c in cells])
    nbrs = grid_neighbors(DIMS)
    n_s, v_s, p_s, mass, loss = [], [], [], [], 0.0
    try:
        for s in range(steps):
            m, dl = ref.vlasov_step(h, DIMS, (DX, DX, DX), B, dt, s % 3, CHARGE, MASS_PROTON, nbrs, moments=True)
            n, V, P = _split(m)
            loss += float(dl.sum())
            n_s.append(n), v_s.append(V), p_s.append(P), mass.append(float(n.sum()) + loss)
        state = [ref.extract(h, c) for c in range(n_cells)]
    finally:
        ref.destroy(h)
    assert ref.bailouts() == 0
    return dict(n=np.stack(n_s), V=np.stack(v_s), P=np.stack(p_s), mass=np.array(mass), state=state)


@pytest.fixture(scope="module")
def study(mesh):
    cells = sinewave_grid(DIMS, mesh)
    dt = 0.8 * r_dt(mesh, cells)
    m0 = float(sum(c.data.astype(np.float64).sum() for c in cells)) * _dv3(mesh)
    fp64 = _reference_run("dp", mesh, cells, dt, STEPS)
    fp32 = _reference_run("sp", mesh, cells, dt, YARDSTICK_STEPS)
    return dict(cells=cells, dt=dt, m0=m0, fp64=fp64, fp32=fp32, rows={})


def _errors(run, ref, steps):
    """Per step: n relative error, V error / max |V|, P error / max P_ii (max over cells)."""
    k = steps
    n_err = np.abs(run["n"][:k] / ref["n"][:k] - 1).max(axis=1)
    v_err = np.abs(run["V"][:k] - ref["V"][:k]).max(axis=(1, 2)) / np.abs(ref["V"][:k]).max()
    p_err = np.abs(run["P"][:k] - ref["P"][:k]).max(axis=(1, 2)) / np.abs(ref["P"][:k, :, :3]).max()
    return n_err, v_err, p_err


def _vdf_error(cells_a, cells_b):
    """Max |f_a - f_b| over the grid relative to the peak of b; a block that
    one side lacks counts as zeros."""
    peak = max(float(np.abs(d).max()) for _, d in cells_b)
    err = 0.0
    for (g1, d1), (g2, d2) in zip(cells_a, cells_b):
        u = np.union1d(g1, g2)
        a = np.zeros((len(u), WID3))
        c = np.zeros((len(u), WID3))
        a[np.searchsorted(u, g1)] = d1
        c[np.searchsorted(u, g2)] = d2
        err = max(err, float(np.abs(a - c).max()))
    return err / peak


def _report(study, label, run, steps):
    n_err, v_err, p_err = _errors(run, study["fp64"], steps)
    drift = run["mass"][:steps] / study["m0"] - 1
    study["rows"][label] = (n_err, v_err, p_err, drift)
    path = os.environ.get("VLGPU_PRECISION_REPORT")
    if path:
        ref_drift = study["fp64"]["mass"] / study["m0"] - 1
        with open(path, "a") as f:
            f.write(f"\n## {label}: grid {DIMS}, {steps} steps, dt {study['dt']:.4f} s\n\n")
            f.write("| step | n rel err | V err / max abs V | P err / max P_ii | mass drift | "
                    "FP64 reference mass drift |\n")
            f.write("|---|---|---|---|---|---|\n")
            for s in range(steps):
                f.write(f"| {s + 1} | {n_err[s]:.3e} | {v_err[s]:.3e} | {p_err[s]:.3e} | {drift[s]:.3e} | "
                        f"{ref_drift[s]:.3e} |\n")
            if "vdf" in run:
                f.write(f"\nVDF max abs error / peak after step {steps}: {run['vdf']:.3e}\n")
    print(f"\n{label}: n err step 1 {n_err[0]:.2e} last {n_err[-1]:.2e}; V err {v_err[0]:.2e} / {v_err[-1]:.2e}; "
          f"P err {p_err[0]:.2e} / {p_err[-1]:.2e}; mass drift {drift[-1]:.2e}"
          + (f"; VDF err / peak {run['vdf']:.2e}" if "vdf" in run else ""))
    return n_err, v_err, p_err, drift


def test_fp32_reference_yardstick(study):
    """The reference's own FP32 build against its FP64 build: the error that
    FP32 storage of the VDF costs the reference itself."""
    fp32 = study["fp32"]
    if YARDSTICK_STEPS == STEPS:
        fp32["vdf"] = _vdf_error(fp32["state"], study["fp64"]["state"])
    n_err, v_err, p_err, _ = _report(study, "reference FP32 build", fp32, YARDSTICK_STEPS)
    assert n_err.max() < 1e-4 and v_err.max() < 1e-3 and p_err.max() < 1e-3


@pytest.mark.parametrize("exact", [False, True])
def test_fp32_gpu_against_fp64_reference(study, mesh, exact):
    from vlasiator_b200 import vlgpu
    cells, dt = study["cells"], study["dt"]
    B = np.stack([c.B for c in cells])
    total = sum(c.n_blocks for c in cells)
    n_s, v_s, p_s, mass = [], [], [], []
    with vlgpu.Batch(mesh, len(cells), 6 * total + 65536, exact=exact) as b:
        b.upload([c.gids for c in cells], [c.data for c in cells])
        b.set_grid(DIMS, DX)
        for s in range(STEPS):
            if s == 0:
                b.vlasov_step(B, dt, 0)
            else:
                b.vlasov_step_device(dt, s % 3)
            m = b.moments(second=True)
            n_s.append(m[:, 0]), v_s.append(m[:, 5:8]), p_s.append(m[:, 9:15])
            mass.append(float(m[:, 0].sum()) + float(b.rho_loss().sum()))
        final = b.cells()
        b.sync()
        assert not b.status().any()
    run = dict(n=np.stack(n_s), V=np.stack(v_s), P=np.stack(p_s), mass=np.array(mass))
    run["vdf"] = _vdf_error(final, study["fp64"]["state"])
    label = "GPU FP32, " + ("exact mode" if exact else "fused mode (default)")
    n_err, v_err, p_err, drift = _report(study, label, run, STEPS)
    ref_drift = study["fp64"]["mass"] / study["m0"] - 1
    assert run["vdf"] < 1e-3
    assert n_err.max() < 1e-4 and v_err.max() < 1e-3 and p_err.max() < 1e-3
    assert abs(drift[-1] - ref_drift[-1]) < 1e-5
    # over the steps the reference's FP32 build ran, the GPU's moment errors
    # stay within a small factor of the reference's own
    yard = study["rows"].get("reference FP32 build")
    if yard is not None:
        k = YARDSTICK_STEPS
        for got, ref32 in zip((n_err, v_err, p_err), yard[:3]):
            assert got[:k].max() <= 10 * ref32[:k].max() + 1e-9
