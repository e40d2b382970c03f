"""VLSV output (no GPU): the layout of the VLSV2 specification
(doc/vlsv2/documentation.lyx in the reference tree) and the arrays
iowrite.cpp writes for a population, read back exactly."""
import struct
import xml.etree.ElementTree as ET

import numpy as np

from vlasiator_b200.mesh import WID3, VelocityMesh
from vlasiator_b200.projects import maxwellian_cell
from vlasiator_b200.vlsv import VlsvReader, write_vlasov_file


def test_vlasov_file_round_trip(tmp_path):
    mesh = VelocityMesh()
    cells = [maxwellian_cell(mesh, 1e6, 3e5, (1e5 * k, 0, 0)) for k in range(3)]
    cells.insert(1, type(cells[0])(gids=np.zeros(0, np.uint32), data=np.zeros((0, WID3), np.float32)))
    mom = np.random.default_rng(0).normal(size=(4, 16))
    path = str(tmp_path / "bulk.vlsv")
    write_vlasov_file(path, mesh, [(c.gids, c.data) for c in cells], grid_dims=(2, 2, 1), moments=mom)
    raw = open(path, "rb").read()
    (footer,) = struct.unpack("<Q", raw[:8])
    root = ET.fromstring(raw[footer:])
    assert root.tag == "VLSV"
    for el in root:  # mandatory attributes and an offset inside the array region
        for a in ("arraysize", "vectorsize", "datatype", "datasize"):
            assert el.get(a) is not None, (el.tag, a)
        assert 8 <= int(el.text) <= footer
    r = VlsvReader(path)
    np.testing.assert_array_equal(r.read("MESH", name="SpatialGrid"), np.arange(1, 5))
    np.testing.assert_array_equal(r.read("BLOCKSPERCELL", name="proton"), [len(c.gids) for c in cells])
    np.testing.assert_array_equal(r.read("BLOCKIDS", name="proton"), np.concatenate([c.gids for c in cells]))
    avgs = r.read("BLOCKVARIABLE", name="proton")
    assert avgs.shape == (sum(len(c.gids) for c in cells), WID3) and avgs.dtype == np.float32
    np.testing.assert_array_equal(avgs, np.concatenate([c.data for c in cells]))
    assert r.find("BLOCKVARIABLE", name="proton").get("mesh") == "SpatialGrid"
    np.testing.assert_array_equal(r.read("MESH_BBOX", mesh="proton"), [67, 67, 67, 4, 4, 4])
    crd = r.read("MESH_NODE_CRDS_X", mesh="proton")
    assert len(crd) == 67 * 4 + 1 and crd[0] == mesh.vmin[0]
    # what the reference's restart reader looks up first (ioread.cpp:170-200, 1162-1194)
    np.testing.assert_array_equal(r.read("VARIABLE", name="CellID", mesh="SpatialGrid"), np.arange(1, 5))
    assert r.find("VARIABLE", name="CellID").get("vectorsize") == "1"
    for name, want, kind, size in (("time", 0.0, "float", "8"), ("timestep", 0, "uint", "4"),
                                   ("xmax", 6e5, "float", "8"), ("ycells_ini", 2, "uint", "4"),
                                   ("zcells_ini", 1, "uint", "4")):
        el = r.find("PARAMETER", name=name)
        assert (el.get("datatype"), el.get("datasize"), el.get("arraysize")) == (kind, size, "1"), name
        assert r.read("PARAMETER", name=name)[0] == want, name
    np.testing.assert_allclose(r.read("VARIABLE", name="vg_v"), mom[:, 5:8])
    np.testing.assert_allclose(r.read("VARIABLE", name="vg_pressure"), mom[:, 9:12].mean(1))
