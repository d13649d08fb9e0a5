"""Element-face surfaces of solid blocks: the names of ``gfem.surfaces`` that the
load set-up of the hot path uses (host side, NumPy + the library's C++ index code).

The config-3 right-hand side is ``pressure_vector(X, sub_surface(skin(X, blocks),
top_nodes), -1)``.  What is here:

  * ``FacetType`` — facet shape functions in closed form (TRI6: the faces of
    C3D10, 3-point rule; QUAD4: the faces of C3D8, 2x2 Gauss rule) and the node
    permutation that reverses a facet's orientation (gfem/elements.py:40-101
    defines the same facet types);
  * ``Surface`` — facets grouped by facet type (gfem/surfaces.py:10-32) with
    ``nodes`` and ``integrate`` (103-120: nodal weights int N_a dA, area, and the
    area-weighted normal sum);
  * ``skin`` (gfem/surfaces.py:182-221): faces that belong to exactly one element;
  * ``orient_outward`` (150-162) and ``sub_surface`` (234-242).

How ``skin`` works here: every face of every element is keyed by its corner nodes
in ascending order (triangles padded in front with -1, so triangles and quads share
one key width); the library counts equal keys in a hash table
(``exfem_host_face_once``) and a face is on the boundary when its key occurs once.
Each boundary face is oriented by the sign of its area vector (the sum of the fan
triangles of its corner polygon, taken from corner 0) against the direction to its
element's corner centroid, and reversed when that points inward.  The facets are
listed by facet type in order of first appearance, and inside a type by block,
local face index and element — the order of the reference's surfaces, which the
tests compare against bit for bit (``tests/golden/ref_index_fixtures.npz``).
"""
import ctypes as C

import numpy as np

from ._lib import check, lib

_G2 = 1.0 / np.sqrt(3.0)


class FacetType:
    """A surface facet: ``ncorner`` corner nodes (counter-clockwise seen from the
    outward side), then one mid-side node per edge for quadratic facets."""

    def __init__(self, name, nnode, ncorner, points, weights):
        self.name, self.nnode, self.ncorner = name, nnode, ncorner
        self.gp = np.asarray(points, float)
        self.gw = np.asarray(weights, float)
        self.N = np.stack([self.shape(s, t) for s, t in self.gp])            # (ngp, nnode)
        self.dN = np.stack([self.shape_grad(s, t) for s, t in self.gp])      # (ngp, nnode, 2)
        # reversed orientation: corner 0 stays, the corner cycle runs backwards, and
        # the mid-side nodes follow their edges (edge k joins corners k and k+1)
        k = ncorner
        self.reverse = [0] + list(range(k - 1, 0, -1)) + list(range(nnode - 1, k - 1, -1))

    def shape(self, s, t):
        if self.name == "TRI6":
            b = np.array([1.0 - s - t, s, t])                                 # barycentric
            edges = [(0, 1), (1, 2), (2, 0)]
            return np.concatenate([b * (2.0 * b - 1.0), [4.0 * b[i] * b[j] for i, j in edges]])
        xs, ys = np.array([-1.0, 1.0, 1.0, -1.0]), np.array([-1.0, -1.0, 1.0, 1.0])
        return 0.25 * (1.0 + xs * s) * (1.0 + ys * t)

    def shape_grad(self, s, t):
        if self.name == "TRI6":
            b = np.array([1.0 - s - t, s, t])
            db = np.array([[-1.0, -1.0], [1.0, 0.0], [0.0, 1.0]])             # d b_i / d(s, t)
            rows = [(4.0 * b[i] - 1.0) * db[i] for i in range(3)]
            rows += [4.0 * (db[i] * b[j] + b[i] * db[j]) for i, j in [(0, 1), (1, 2), (2, 0)]]
            return np.stack(rows)
        xs, ys = np.array([-1.0, 1.0, 1.0, -1.0]), np.array([-1.0, -1.0, 1.0, 1.0])
        return np.stack([0.25 * xs * (1.0 + ys * t), 0.25 * ys * (1.0 + xs * s)], axis=1)

    def flip(self, facets):
        """The same facets with reversed orientation."""
        return np.asarray(facets)[:, self.reverse]

    def area_vectors(self, X, facets):
        """Quadrature-weighted normals dx/ds x dx/dt * w_g of each facet at each
        point: (nf, ngp, 3); their length is the area element."""
        xe = np.asarray(X)[np.asarray(facets)]                                # (nf, nnode, 3)
        ts = np.matmul(self.dN[:, :, 0], xe)                                  # (nf, ngp, 3)
        tt = np.matmul(self.dN[:, :, 1], xe)
        return np.cross(ts, tt) * self.gw[:, None]

    def __repr__(self):
        return f"<FacetType {self.name}>"


TRI6 = FacetType("TRI6", 6, 3, [[1 / 6, 1 / 6], [2 / 3, 1 / 6], [1 / 6, 2 / 3]], [1 / 6] * 3)
QUAD4 = FacetType("QUAD4", 4, 4, [[-_G2, -_G2], [_G2, -_G2], [_G2, _G2], [-_G2, _G2]], [1.0] * 4)
FACETS = {6: TRI6, 4: QUAD4}


class Surface:
    """Facets grouped by type: ``groups`` is a list of (FacetType, facets (nf, nnode))."""

    def __init__(self, groups=None, name="surface"):
        self.name = name
        self.groups = []
        for ft, f in groups or []:
            self.add(ft, f)

    def add(self, ft, facets):
        facets = np.asarray(facets, dtype=np.int64).reshape(-1, ft.nnode)
        if len(facets) == 0:
            return
        types = [g for g, _ in self.groups]
        if ft in types:
            i = types.index(ft)
            self.groups[i] = (ft, np.concatenate([self.groups[i][1], facets]))
        else:
            self.groups.append((ft, facets))

    def __len__(self):
        return int(sum(len(f) for _, f in self.groups))

    def nodes(self):
        """Sorted distinct nodes of all facets."""
        if not self.groups:
            return np.zeros(0, np.int64)
        return np.unique(np.concatenate([f.reshape(-1) for _, f in self.groups]))

    def integrate(self, X, field=None):
        """(nodal weights int N_a dA (nn,), area, area-weighted normal sum); ``field``
        optionally scales each facet (constant over the facet)."""
        nn = len(X)
        w = np.zeros(nn)
        area, nsum = 0.0, np.zeros(3)
        for ft, f in self.groups:
            n = ft.area_vectors(X, f)                                        # (nf, ngp, 3)
            da = np.sqrt(np.sum(n * n, axis=-1))                              # (nf, ngp)
            if field is not None:
                da = da * np.asarray(field, float)[:, None]
            w += np.bincount(f.reshape(-1), weights=(da @ ft.N).reshape(-1), minlength=nn)
            area += float(da.sum())
            nsum += n.reshape(-1, 3).sum(0)
        return w, area, nsum


def _area_vector(X, ft, facets):
    """Area vector of each facet's corner polygon: sum of its fan triangles from
    corner 0 (for a triangle, (c1 - c0) x (c2 - c0); for a quad, both halves)."""
    c = np.asarray(X)[np.asarray(facets)[:, :ft.ncorner]]
    e = c[:, 1:] - c[:, :1]                                                   # edges from corner 0
    return np.cross(e[:, :-1], e[:, 1:]).sum(1)


def orient_outward(X, ft, facets, centroids):
    """Reverse the facets whose area vector points toward their element's centroid."""
    facets = np.asarray(facets)
    c = np.asarray(X)[facets[:, :ft.ncorner]]
    towards = np.asarray(centroids) - c.mean(1)
    inward = np.sum(_area_vector(X, ft, facets) * towards, axis=1) > 0
    out = facets.copy()
    out[inward] = ft.flip(facets[inward])
    return out


def _conn(b):
    c = b.conn
    return np.asarray(c.cpu() if hasattr(c, "cpu") else c, dtype=np.int64)


def skin(X, blocks):
    """Faces of the blocks' elements that no other element shares, outward oriented."""
    X = np.asarray(X)
    faces = []                                # (block, local face, facet type, face nodes, element ids)
    for bi, b in enumerate(blocks):
        conn = _conn(b)
        for k, loc in enumerate(b.etype.faces):
            faces.append((bi, k, FACETS[len(loc)], conn[:, loc], np.arange(len(conn))))
    s = Surface(name="skin")
    if not faces:
        return s
    keys = []
    for _, _, ft, f, _ in faces:
        key = np.full((len(f), 4), -1, np.int64)
        key[:, 4 - ft.ncorner:] = np.sort(f[:, :ft.ncorner], axis=1)
        keys.append(key)
    keys = np.ascontiguousarray(np.concatenate(keys))
    once = np.zeros(len(keys), np.uint8)
    check(lib.exfem_host_face_once(C.c_int64(len(keys)), keys.ctypes.data, once.ctypes.data))
    pos = 0
    for bi, k, ft, f, el in faces:
        sel = once[pos:pos + len(f)].astype(bool)
        pos += len(f)
        if not sel.any():
            continue
        b = blocks[bi]
        cen = X[_conn(b)[el[sel], :b.etype.ncorner]].mean(1)
        s.add(ft, orient_outward(X, ft, f[sel], cen))
    return s


def sub_surface(surface, node_set):
    """The facets of ``surface`` whose corner nodes all belong to ``node_set``."""
    nodes = np.asarray(list(node_set) if not isinstance(node_set, np.ndarray) else node_set, dtype=np.int64)
    out = Surface(name="sub")
    for ft, f in surface.groups:
        out.add(ft, f[np.isin(f[:, :ft.ncorner], nodes).all(1)])
    return out
