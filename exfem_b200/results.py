"""Result output for ParaView: VTK XML unstructured grids (.vtu) and time-series
collections (.pvd), the format of the reference's writer (gfem/io/vtk.py:24-71).

The files follow the VTK XML specification, which fixes their layout: binary
DataArrays, base64 of a UInt64 byte count followed by the little-endian values;
cells given by connectivity, offsets and type ids (VTK_HEXAHEDRON = 12 for C3D8,
VTK_QUADRATIC_TETRA = 24 for C3D10, whose mid-edge order 0-1, 1-2, 2-0, 0-3, 1-3, 2-3
is the element's own).  Node arrays (length nn) go to PointData, element arrays
(length of all cells) to CellData.  ``frame`` gathers the usual result fields —
displacement, and per element the volume-averaged von Mises stress and equivalent
plastic strain (``Model.stresses``, gfem/model.py:530-539).
"""
import base64

import numpy as np

VTK_CELL = {"C3D8": 12, "C3D10": 24}
_TYPES = {"Float64": np.float64, "Float32": np.float32, "Int64": np.int64, "UInt8": np.uint8}


def _array(name, values, vtk_type="Float64", ncomp=None):
    a = np.ascontiguousarray(values, dtype=_TYPES[vtk_type]).ravel()
    raw = a.tobytes()
    payload = base64.b64encode(np.uint64(len(raw)).tobytes() + raw).decode("ascii")
    comps = f' NumberOfComponents="{ncomp}"' if ncomp else ""
    return f'<DataArray type="{vtk_type}" Name="{name}"{comps} format="binary">{payload}</DataArray>'


def write_vtu(path, X, blocks, point_data=None, cell_data=None):
    """Mesh X (nn, 3) with blocks (objects with ``conn`` and ``etype``) and result
    arrays (name -> array) to one .vtu file."""
    X = np.asarray(X, dtype=np.float64)
    conns = [np.asarray(b.conn, dtype=np.int64) for b in blocks]
    types = np.concatenate([np.full(len(c), VTK_CELL[b.etype.name], np.uint8) for b, c in zip(blocks, conns)]) \
        if conns else np.zeros(0, np.uint8)
    flat = np.concatenate([c.ravel() for c in conns]) if conns else np.zeros(0, np.int64)
    offsets = np.cumsum(np.concatenate([np.full(len(c), c.shape[1]) for c in conns])) if conns else np.zeros(0)
    pd, cd = [], []
    for name, v in (point_data or {}).items():
        v = np.asarray(v, dtype=np.float64)
        if len(v) != len(X):
            raise ValueError(f"point array {name} has {len(v)} rows, the mesh {len(X)} nodes")
        pd.append(_array(name, v, "Float64", v.shape[1] if v.ndim > 1 else None))
    for name, v in (cell_data or {}).items():
        v = np.asarray(v, dtype=np.float64)
        if len(v) != len(types):
            raise ValueError(f"cell array {name} has {len(v)} rows, the mesh {len(types)} cells")
        cd.append(_array(name, v, "Float64", v.shape[1] if v.ndim > 1 else None))
    with open(path, "w") as f:
        f.write('<?xml version="1.0"?>\n'
                '<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64">\n'
                f'<UnstructuredGrid>\n<Piece NumberOfPoints="{len(X)}" NumberOfCells="{len(types)}">\n'
                f'<Points>{_array("Points", X, "Float64", 3)}</Points>\n'
                f'<Cells>{_array("connectivity", flat, "Int64")}{_array("offsets", offsets, "Int64")}'
                f'{_array("types", types, "UInt8")}</Cells>\n'
                f'<PointData>{"".join(pd)}</PointData>\n<CellData>{"".join(cd)}</CellData>\n'
                '</Piece>\n</UnstructuredGrid>\n</VTKFile>\n')


def write_pvd(path, entries):
    """Time series: entries [(time, .vtu file name), ...]."""
    with open(path, "w") as f:
        f.write('<?xml version="1.0"?>\n<VTKFile type="Collection" version="0.1">\n<Collection>\n')
        for t, name in entries:
            f.write(f'<DataSet timestep="{t:.9g}" file="{name}"/>\n')
        f.write('</Collection>\n</VTKFile>\n')


def frame(model, u, states):
    """{"U": (nn, 3), "MISES": (ne,), "PEEQ": (ne,)} of a solution (element values in
    block order)."""
    host = lambda t: np.asarray(t.detach().cpu() if hasattr(t, "detach") else t, dtype=np.float64)
    st = model.stresses(u, states)
    return dict(U=host(u).reshape(-1, 3), MISES=np.concatenate([host(s["MISES"]) for s in st]),
                PEEQ=np.concatenate([host(s["PEEQ"]) for s in st]))


def write_frame(path, model, u, states):
    """Displacement, von Mises and equivalent plastic strain of a solution to .vtu."""
    fr = frame(model, u, states)
    write_vtu(path, model.X, model.blocks, point_data={"U": fr["U"]},
              cell_data={"MISES": fr["MISES"], "PEEQ": fr["PEEQ"]})
