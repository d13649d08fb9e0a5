"""Oracle: structured mesh generation of the reference, restated on the CPU.

Test infrastructure only (see ``oracle/__init__.py``); also the mesh source of the
CPU reference arm of ``bench.py``, which must not load the CUDA library.

  * gfem/mesh.py:5-16   ``box_hex``: grid nodes with x slowest and z fastest, node id
                        (i (ny+1) + j) (nz+1) + k; elements in (i, j, k) order with
                        Abaqus C3D8 corner order (bottom face counter-clockwise, then top)
  * gfem/mesh.py:19-29  ``hex_to_tet4``: six tetrahedra per hexahedron around its 0-6
                        diagonal (Kuhn split), nodes 1 and 2 swapped where the signed
                        volume is negative
  * gfem/mesh.py:32-38  ``tet4_to_tet10``: one mid-node per distinct edge at the edge
                        midpoint, numbered after the corners in ascending (lo, hi) order,
                        local edges (0,1) (1,2) (2,0) (0,3) (1,3) (2,3)

Pinned bit for bit to the reference's own output (``tests/golden/mesh_fixtures.npz``,
``tests/test_oracle.py``).  ``jitter_interior`` is the synthetic workloads' node
perturbation (uniform, interior nodes only, one seeded generator), the same draw as
the product's mesh module so both build the same meshes.
"""
import numpy as np

# the six Kuhn tetrahedra of a hexahedron, as local corner indices (gfem/mesh.py:19-21)
_KUHN_SPLIT = ((0, 1, 2, 6), (0, 2, 3, 6), (0, 3, 7, 6), (0, 7, 4, 6), (0, 4, 5, 6), (0, 5, 1, 6))
# local edges of a tetrahedron in the order of its mid-nodes 4..9 (gfem/mesh.py:33)
_TET_EDGES = ((0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3))


def box_hex(L, H, W, nx, ny, nz, origin=(0.0, 0.0, 0.0)):
    axes = [np.linspace(0.0, ext, n + 1) + o for ext, n, o in zip((L, H, W), (nx, ny, nz), origin)]
    gi, gj, gk = np.indices((nx + 1, ny + 1, nz + 1)).reshape(3, -1)
    X = np.stack([axes[0][gi], axes[1][gj], axes[2][gk]], axis=1)
    ei, ej, ek = np.indices((nx, ny, nz)).reshape(3, -1)

    def node(a, b, c):
        return (a * (ny + 1) + b) * (nz + 1) + c
    corners = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
    conn = np.stack([node(ei + di, ej + dj, ek + dk) for di, dj, dk in corners], axis=1)
    return X, conn


def hex_to_tet4(X, conn):
    X = np.asarray(X)
    conn = np.asarray(conn)
    tets = np.stack([conn[:, list(t)] for t in _KUHN_SPLIT], axis=1).reshape(-1, 4)
    p0, p1, p2, p3 = (X[tets[:, a]] for a in range(4))
    vol = np.sum(np.cross(p1 - p0, p2 - p0) * (p3 - p0), axis=1)
    flip = vol < 0
    tets[flip] = tets[flip][:, [0, 2, 1, 3]]
    return X, tets


def tet4_to_tet10(X, conn):
    X = np.asarray(X)
    conn = np.asarray(conn)
    ne = len(conn)
    ends = np.concatenate([np.sort(conn[:, list(e)], axis=1) for e in _TET_EDGES])   # (6 ne, 2), edge-major
    order = np.lexsort((ends[:, 1], ends[:, 0]))
    srt = ends[order]
    new = np.ones(len(srt), bool)
    new[1:] = np.any(srt[1:] != srt[:-1], axis=1)
    rank = np.cumsum(new) - 1                                      # distinct-edge number in sorted order
    edge_id = np.empty(len(ends), np.int64)
    edge_id[order] = rank
    distinct = srt[new]
    mids = 0.5 * (X[distinct[:, 0]] + X[distinct[:, 1]])
    mid_nodes = edge_id.reshape(len(_TET_EDGES), ne).T + len(X)
    return np.concatenate([X, mids]), np.concatenate([conn, mid_nodes], axis=1)


def nodes_where(X, fn):                                            # gfem/mesh.py:41-42
    X = np.asarray(X)
    return np.flatnonzero(fn(X[:, 0], X[:, 1], X[:, 2]))


def jitter_interior(X, h, frac, seed):
    """Nodes strictly inside the bounding box move by U(-1, 1) * frac * h per axis
    (one ``default_rng(seed)`` draw of shape X.shape); boundary nodes stay."""
    X = np.array(X, dtype=np.float64)
    lo, hi = X.min(0), X.max(0)
    tol = 1e-9 * max(float(np.max(hi - lo)), 1.0)
    inside = np.all((X > lo + tol) & (X < hi - tol), axis=1)
    step = np.random.default_rng(seed).uniform(-1.0, 1.0, size=X.shape) * frac * np.broadcast_to(
        np.asarray(h, float), (3,))
    X[inside] += step[inside]
    return X
