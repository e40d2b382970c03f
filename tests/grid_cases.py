"""Cell sets of the grid tests and the numpy statement of the r-space time
step they are checked with."""
import numpy as np

from vlasiator_b200.projects import maxwellian_cell


def varied_grid(mesh, dims, seed):
    rng = np.random.default_rng(seed)
    cells = []
    for _ in range(int(np.prod(dims))):
        V = rng.uniform(-3e5, 3e5, 3)
        cells.append(maxwellian_cell(mesh, 10 ** rng.uniform(5.5, 6.5), rng.uniform(1.5e5, 4e5), V))
    return cells


def r_dt_restated(mesh, cells, dx):
    """reduce_vlasov_dt for one population, in numpy (arch_dt.cpp:34-97)."""
    eps = np.finfo(np.float64).tiny * 1000
    bs = [(mesh.vmax[d] - mesh.vmin[d]) / mesh.length[d] for d in range(3)]
    dv = [bs[d] / 4 for d in range(3)]
    out = []
    for c in cells:
        g = c.gids.astype(np.int64)
        idx = [g % mesh.length[0], (g // mesh.length[0]) % mesh.length[1], g // (mesh.length[0] * mesh.length[1])]
        best = np.inf
        for i in (0, 3):
            V = [mesh.vmin[d] + idx[d] * bs[d] + (i + 0.5) * dv[d] + eps for d in range(3)]
            t = np.minimum(np.minimum(dx[0] / np.abs(V[0]), dx[1] / np.abs(V[1])), dx[2] / np.abs(V[2]))
            best = min(best, float(t.min()))
        out.append(best)
    return np.array(out)
