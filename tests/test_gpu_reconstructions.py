"""The PLM and PQM acceleration reconstructions (the reference's
ACC_SEMILAG_PLM / ACC_SEMILAG_PQM builds of map_1d) against fixtures made by
the reference's own code (tests/golden/make_golden.py).

Each sweep starts from the reference's previous output, so errors do not
compound: identical block sets, values within 1e-5 of the cell's peak, mass
to 1e-6 per sweep.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
ORDERS = [[0, 1, 2], [1, 2, 0], [2, 0, 1]]


@pytest.fixture(scope="module")
def vl():
    from vlasiator_b200 import vlgpu
    vlgpu.load()
    return vlgpu


@pytest.mark.parametrize("recon", ["pqm", "plm"])
def test_reconstruction_matches_reference(vl, mesh, recon):
    z = np.load(os.path.join(GOLDEN, f"map1d_sp_{recon}.npz"))
    names = sorted({k.split("/")[0] for k in z.files})
    worst = 0.0
    for name in names:
        g, d = z[f"{name}/gids_in"], z[f"{name}/data_in"]
        isect = z[f"{name}/isect"]
        mo = int(z[f"{name}/map_order"])
        with vl.Batch(mesh, 1, 4 * len(g) + 4096, recon=recon) as b:
            for s, dim in enumerate(ORDERS[mo]):
                b.upload([g], [d])
                b.map_1d(isect[4 * dim:4 * dim + 4][None, :], dim)
                (gg, dd), = b.cells()
                rg, rd = z[f"{name}/sweep{s}_gids"], z[f"{name}/sweep{s}_data"]
                np.testing.assert_array_equal(gg, rg, err_msg=f"{recon} {name} sweep {s}")
                peak = float(np.abs(rd).max())
                err = float(np.abs(dd - rd).max()) / peak
                worst = max(worst, err)
                assert err <= 1e-5, f"{recon} {name} sweep {s}: {err:.2e} of peak"
                m1, m0 = float(dd.astype(np.float64).sum()), float(rd.astype(np.float64).sum())
                assert abs(m1 / m0 - 1.0) <= 1e-6
                assert not b.status().any()
                g, d = rg, rd
    print(f"{recon}: worst {worst:.2e} of peak")


def test_exact_mode_is_ppm_only(vl, mesh):
    with vl.Batch(mesh, 1, 4096, recon="pqm") as b:
        with pytest.raises(vl.VlgpuError):
            b.set_exact(True)
    with vl.Batch(mesh, 1, 4096, exact=True) as b:
        with pytest.raises(vl.VlgpuError):
            b.set_reconstruction("plm")
