"""Structured mesh generators with the reference's node and element numbering.

Drop-in for ``gfem.mesh`` (gfem/mesh.py:5-42).  The numbering is a format the
hot path depends on (``dofs = 3*node + d``, the gather plan, the tile maps), so
it is kept identical to the reference and checked bit for bit against fixtures
generated from the reference's own ``mesh.py``:

  * ``box_hex``: node id ``(i*(ny+1) + j)*(nz+1) + k`` with i along x; elements in
    (i, j, k) lexicographic order, Abaqus C3D8 corner order (gfem/mesh.py:5-16).
  * ``hex_to_tet4``: 6 Kuhn tetrahedra per hexahedron around the 0-6 diagonal,
    local nodes 1 and 2 swapped where the signed volume is negative (mesh.py:19-29).
  * ``tet4_to_tet10``: one mid-node per distinct edge, numbered after the corner
    nodes in lexicographic order of the sorted (lo, hi) edge, edge order
    (0,1) (1,2) (2,0) (0,3) (1,3) (2,3) per element (mesh.py:32-38).
"""
import numpy as np

KUHN = np.array([[0, 1, 2, 6], [0, 2, 3, 6], [0, 3, 7, 6],
                 [0, 7, 4, 6], [0, 4, 5, 6], [0, 5, 1, 6]])
TET10_EDGES = ((0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3))


def box_hex(L, H, W, nx, ny, nz, origin=(0, 0, 0)):
    gx = np.linspace(0, L, nx + 1) + origin[0]
    gy = np.linspace(0, H, ny + 1) + origin[1]
    gz = np.linspace(0, W, nz + 1) + origin[2]
    X = np.empty(((nx + 1) * (ny + 1) * (nz + 1), 3))
    X[:, 0] = np.repeat(gx, (ny + 1) * (nz + 1))
    X[:, 1] = np.tile(np.repeat(gy, nz + 1), nx + 1)
    X[:, 2] = np.tile(gz, (nx + 1) * (ny + 1))
    base = (np.arange(nx)[:, None, None] * (ny + 1) + np.arange(ny)[None, :, None]) * (nz + 1) \
        + np.arange(nz)[None, None, :]
    base = base.reshape(-1)
    sx, sy = (ny + 1) * (nz + 1), nz + 1
    off = np.array([0, sx, sx + sy, sy, 1, sx + 1, sx + sy + 1, sy + 1])
    return X, base[:, None] + off[None, :]


def hex_to_tet4(X, conn):
    X = np.asarray(X)
    t = np.asarray(conn)[:, KUHN].reshape(-1, 4)
    a, b, c, d = (X[t[:, k]] for k in range(4))
    vol = np.einsum("ij,ij->i", np.cross(b - a, c - a), d - a)
    neg = vol < 0
    t[neg, 1], t[neg, 2] = t[neg, 2].copy(), t[neg, 1].copy()
    return X, t


def tet4_to_tet10(X, conn):
    X = np.asarray(X)
    conn = np.asarray(conn)
    nn = len(X)
    pairs = np.stack([conn[:, list(e)] for e in TET10_EDGES], 0)        # (6, ne, 2)
    lo, hi = pairs.min(-1).astype(np.int64), pairs.max(-1).astype(np.int64)
    key = lo * nn + hi
    uk, inv = np.unique(key.reshape(-1), return_inverse=True)
    mids = 0.5 * (X[uk // nn] + X[uk % nn])
    mid_id = inv.reshape(len(TET10_EDGES), -1).T + nn
    return np.vstack([X, mids]), np.hstack([conn, mid_id])


def nodes_where(X, fn):
    X = np.asarray(X)
    return np.nonzero(fn(X[:, 0], X[:, 1], X[:, 2]))[0]


def jitter_interior(X, h, frac, seed, box_lo=None, box_hi=None):
    """Move every node that is not on the bounding box by U(-frac*h, frac*h) per axis.
    Boundary nodes stay put, so face selections by coordinate remain exact."""
    X = np.array(X, dtype=np.float64)
    lo = X.min(0) if box_lo is None else np.asarray(box_lo, float)
    hi = X.max(0) if box_hi is None else np.asarray(box_hi, float)
    tol = 1e-9 * max(float(np.max(hi - lo)), 1.0)
    interior = np.all((X > lo + tol) & (X < hi - tol), axis=1)
    h = np.broadcast_to(np.asarray(h, float), (3,))
    rng = np.random.default_rng(seed)
    d = rng.uniform(-1.0, 1.0, size=X.shape) * frac * h
    X[interior] += d[interior]
    return X
