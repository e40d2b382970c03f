"""VLSV output of the VDF and its moments (the arrays iowrite.cpp writes).

The layout follows the VLSV2 specification in the reference tree
(doc/vlsv2/documentation.lyx): the file starts with an 8-byte unsigned
offset of the footer, the arrays follow in binary (vectors of fixed size,
native little-endian components), and the footer is an XML tree under a
<VLSV> root with one tag per array, whose value is the array's byte offset
and whose mandatory attributes are arraysize, vectorsize, datatype
(int / uint / float) and datasize.  The vlsv library the reference links is
not part of its tree, so files are checked against that specification and by
reading them back, not against the library's reader.

Arrays of a Vlasov file (iowrite.cpp:141-320, 485-555, 690-715;
datareducer.cpp): the CellID variable and the scalar PARAMETER arrays
(time, dt, timestep, the grid's extent and cell counts) that the
reference's restart reader looks up (ioread.cpp:170-200, 1162-1194);
MESH / MESH_BBOX / MESH_NODE_CRDS_{X,Y,Z} of the spatial grid
("SpatialGrid"), the same for each population's velocity mesh, and per
population CELLSWITHBLOCKS, BLOCKSPERCELL, BLOCKIDS and BLOCKVARIABLE (the
64 phase-space densities of every block, float), plus VARIABLE arrays
vg_rhom, vg_rhoq, vg_v, vg_pressure and populations_vg_blocks.
"""
from __future__ import annotations

import struct
import xml.etree.ElementTree as ET

import numpy as np

from .mesh import WID, WID3, VelocityMesh

_KIND = {"f": "float", "u": "uint", "i": "int"}


class VlsvWriter:
    """Writes arrays one after another and the XML footer on close."""

    def __init__(self, path: str):
        self.f = open(path, "wb")
        self.f.write(struct.pack("<Q", 0))  # footer offset, patched on close
        self.tags = []

    def write_array(self, tag: str, attribs: dict, data) -> None:
        a = np.ascontiguousarray(data)
        if a.ndim == 1:
            a = a.reshape(-1, 1)
        kind = _KIND[a.dtype.kind]
        a = a.astype(a.dtype.newbyteorder("<"), copy=False)
        offset = self.f.tell()
        self.f.write(a.tobytes())
        attrs = dict(attribs)
        attrs.update(arraysize=str(a.shape[0]), vectorsize=str(a.shape[1]), datatype=kind,
                     datasize=str(a.dtype.itemsize))
        self.tags.append((tag, attrs, offset))

    def close(self) -> None:
        root = ET.Element("VLSV")
        for tag, attrs, offset in self.tags:
            el = ET.SubElement(root, tag, attrs)
            el.text = str(offset)
        footer = self.f.tell()
        self.f.write(ET.tostring(root))
        self.f.seek(0)
        self.f.write(struct.pack("<Q", footer))
        self.f.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class VlsvReader:
    """Reads the arrays of a file written in that layout."""

    def __init__(self, path: str):
        with open(path, "rb") as f:
            raw = f.read()
        (footer,) = struct.unpack("<Q", raw[:8])
        self.raw = raw
        self.root = ET.fromstring(raw[footer:])

    def find(self, tag: str, **attribs):
        for el in self.root:
            if el.tag == tag and all(el.get(k) == v for k, v in attribs.items()):
                return el
        raise KeyError((tag, attribs))

    def read(self, tag: str, **attribs) -> np.ndarray:
        el = self.find(tag, **attribs)
        n, v, size = int(el.get("arraysize")), int(el.get("vectorsize")), int(el.get("datasize"))
        dt = np.dtype({"float": "f", "uint": "u", "int": "i"}[el.get("datatype")] + str(size)).newbyteorder("<")
        a = np.frombuffer(self.raw, dtype=dt, count=n * v, offset=int(el.text))
        return a.reshape(n, v) if v > 1 else a


def _node_coords(vmin, cell, n_cells):
    return vmin + np.arange(n_cells + 1, dtype=np.float64) * cell


def write_vlasov_file(path: str, mesh: VelocityMesh, cells, grid_dims=None, dx=(3e5, 3e5, 3e5),
                      grid_min=(0.0, 0.0, 0.0), moments=None, pop: str = "proton", mass: float | None = None,
                      charge: float | None = None, time: float = 0.0, dt: float = 0.0, timestep: int = 0,
                      file_index: int = 0) -> None:
    """One population's VDF and moments.  cells: [(gids, data)] per spatial
    cell, x fastest (cell ID = index + 1, as dccrg numbers a uniform grid);
    moments: the batch's (n_cells, 16) record (vlgpu_batch_moments); time,
    dt, timestep and file_index: the run's scalar parameters."""
    n = len(cells)
    dims = tuple(grid_dims) if grid_dims is not None else (n, 1, 1)
    ids = np.arange(1, n + 1, dtype=np.uint64)
    with VlsvWriter(path) as w:
        # the cell IDs and the run's scalar parameters (writeCommonGridData,
        # iowrite.cpp:485-514): Real parameters as float64, uint ones as uint32
        w.write_array("VARIABLE", {"name": "CellID", "mesh": "SpatialGrid"}, ids)
        lo = np.asarray(grid_min, np.float64)
        hi = lo + np.asarray(dx, np.float64) * np.asarray(dims, np.float64)
        for name, value, dtype in (("time", time, np.float64), ("dt", dt, np.float64),
                                   ("timestep", timestep, np.uint32), ("fieldSolverSubcycles", 1, np.uint32),
                                   ("fileIndex", file_index, np.uint32),
                                   ("xmin", lo[0], np.float64), ("xmax", hi[0], np.float64),
                                   ("ymin", lo[1], np.float64), ("ymax", hi[1], np.float64),
                                   ("zmin", lo[2], np.float64), ("zmax", hi[2], np.float64),
                                   ("xcells_ini", dims[0], np.uint32), ("ycells_ini", dims[1], np.uint32),
                                   ("zcells_ini", dims[2], np.uint32)):
            w.write_array("PARAMETER", {"name": name}, np.array([value], dtype))
        sg = {"name": "SpatialGrid", "type": "amr_ucd", "max_refinement_level": "0",
              "xperiodic": "yes", "yperiodic": "yes", "zperiodic": "yes"}
        w.write_array("MESH", sg, ids)
        w.write_array("MESH_BBOX", {"mesh": "SpatialGrid"},
                      np.array([dims[0], dims[1], dims[2], 1, 1, 1], np.uint64))
        for c, tag in enumerate(("MESH_NODE_CRDS_X", "MESH_NODE_CRDS_Y", "MESH_NODE_CRDS_Z")):
            w.write_array(tag, {"mesh": "SpatialGrid"}, _node_coords(grid_min[c], dx[c], dims[c]))
        # the population's velocity mesh (iowrite.cpp:178-215)
        vm = {"mesh": pop, "type": "amr_ucd", "max_velocity_ref_level": "0"}
        w.write_array("MESH_BBOX", vm, np.array([*mesh.length, WID, WID, WID], np.uint64))
        for c, tag in enumerate(("MESH_NODE_CRDS_X", "MESH_NODE_CRDS_Y", "MESH_NODE_CRDS_Z")):
            w.write_array(tag, vm, _node_coords(mesh.vmin[c], mesh.block_size[c] / WID, mesh.length[c] * WID))
        per_cell = np.array([len(g) for g, _ in cells], np.uint32)
        popattr = {"name": pop, "mesh": "SpatialGrid"}
        w.write_array("CELLSWITHBLOCKS", popattr, ids)
        w.write_array("BLOCKSPERCELL", popattr, per_cell)
        gids = np.concatenate([np.asarray(g, np.uint32) for g, _ in cells]) if n else np.zeros(0, np.uint32)
        data = (np.concatenate([np.asarray(d, np.float32).reshape(-1, WID3) for _, d in cells])
                if n else np.zeros((0, WID3), np.float32))
        w.write_array("BLOCKIDS", popattr, gids)
        w.write_array("BLOCKVARIABLE", popattr, data)
        w.write_array("VARIABLE", {"name": "populations_vg_blocks", "mesh": "SpatialGrid"}, per_cell)
        if moments is not None:
            m = np.asarray(moments, np.float64)
            w.write_array("VARIABLE", {"name": "vg_rhom", "mesh": "SpatialGrid", "unit": "kg/m^3"}, m[:, 4])
            w.write_array("VARIABLE", {"name": "vg_rhoq", "mesh": "SpatialGrid", "unit": "C/m^3"}, m[:, 8])
            w.write_array("VARIABLE", {"name": "vg_v", "mesh": "SpatialGrid", "unit": "m/s"}, m[:, 5:8])
            # scalar pressure: a third of the trace (VariablePressureSolver)
            w.write_array("VARIABLE", {"name": "vg_pressure", "mesh": "SpatialGrid", "unit": "Pa"},
                          (m[:, 9] + m[:, 10] + m[:, 11]) / 3.0)
            w.write_array("VARIABLE", {"name": "vg_ptensor_diagonal", "mesh": "SpatialGrid", "unit": "Pa"},
                          m[:, 9:12])
            w.write_array("VARIABLE", {"name": "vg_ptensor_offdiagonal", "mesh": "SpatialGrid", "unit": "Pa"},
                          m[:, 12:15])


def write_batch(path: str, batch, grid_dims=None, dx=(3e5, 3e5, 3e5), pop: str = "proton", **params) -> None:
    """Downloads a batch (blocks sorted by ID per cell) and its moments and
    writes them; params: write_vlasov_file's time, dt, timestep, file_index."""
    write_vlasov_file(path, batch.mesh, batch.cells(), grid_dims=grid_dims, dx=dx,
                      moments=batch.moments(second=True), pop=pop, **params)
