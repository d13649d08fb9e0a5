"""Boundary surfaces of solid blocks (drop-in names of ``gfem.surfaces``), host set-up.

Covers what the load set-up of the hot path needs (the config-3 traction on the
z = 1 face is ``pressure_vector(X, sub_surface(skin(X, blocks), top_nodes), -1)``):

  * ``FacetType`` ``TRI6`` (faces of C3D10, 3-point rule) and ``QUAD4`` (faces of
    C3D8, 2x2 Gauss rule), shape functions and their parametric derivatives in
    closed form (gfem/elements.py:40-101);
  * ``Surface`` — facet groups by type (gfem/surfaces.py:10-32, 103-120);
  * ``orient_outward`` (gfem/surfaces.py:150-161), ``skin`` (182-221: faces owned by
    exactly one element, grouped per block and local face, outward oriented),
    ``sub_surface`` (234-242).
"""
import numpy as np

_G2 = 1.0 / np.sqrt(3.0)


class FacetType:
    def __init__(self, name, nnode, ncorner, gp, gw, flip):
        self.name, self.nnode, self.ncorner = name, nnode, ncorner
        self.gp, self.gw = np.asarray(gp, float), np.asarray(gw, float)
        self._flip = list(flip)
        self.N, self.dN = self._tabulate()                   # (ngp, nnode), (ngp, nnode, 2)

    def _tabulate(self):
        N, dN = [], []
        for s, t in self.gp:
            if self.name == "TRI6":
                L = np.array([1 - s - t, s, t])
                dL = np.array([[-1.0, -1.0], [1.0, 0.0], [0.0, 1.0]])       # dL_i / d(s, t)
                n = list(L * (2 * L - 1))
                d = [(4 * L[i] - 1) * dL[i] for i in range(3)]
                for i, j in ((0, 1), (1, 2), (2, 0)):
                    n.append(4 * L[i] * L[j])
                    d.append(4 * (dL[i] * L[j] + L[i] * dL[j]))
            else:                                                           # QUAD4
                C = np.array([[-1, -1], [1, -1], [1, 1], [-1, 1]], float)
                n = 0.25 * (1 + C[:, 0] * s) * (1 + C[:, 1] * t)
                d = np.stack([0.25 * C[:, 0] * (1 + C[:, 1] * t), 0.25 * C[:, 1] * (1 + C[:, 0] * s)], 1)
            N.append(np.asarray(n))
            dN.append(np.asarray(d))
        return np.array(N), np.array(dN)

    def flip(self, f):
        return np.asarray(f)[:, self._flip]

    def __repr__(self):
        return f"<FacetType {self.name}>"


TRI6 = FacetType("TRI6", 6, 3, [[1 / 6, 1 / 6], [2 / 3, 1 / 6], [1 / 6, 2 / 3]], [1 / 6] * 3, [0, 2, 1, 5, 4, 3])
QUAD4 = FacetType("QUAD4", 4, 4, [[-_G2, -_G2], [_G2, -_G2], [_G2, _G2], [-_G2, _G2]], [1.0] * 4, [0, 3, 2, 1])
FACETS = {6: TRI6, 4: QUAD4}


class Surface:
    def __init__(self, groups=None, name="surface"):
        self.name = name
        self.groups = []                                    # [(FacetType, facets (nf, nnode))]
        for ft, f in groups or []:
            self.add(ft, f)

    def add(self, ft, f):
        f = np.asarray(f, dtype=np.int64).reshape(-1, ft.nnode)
        if not len(f):
            return
        for i, (g, a) in enumerate(self.groups):
            if g is ft:
                self.groups[i] = (g, np.vstack([a, f]))
                return
        self.groups.append((ft, f))

    def __len__(self):
        return sum(len(f) for _, f in self.groups)

    def nodes(self):
        if not self.groups:
            return np.zeros(0, np.int64)
        return np.unique(np.concatenate([f.ravel() for _, f in self.groups]))

    def _jacobians(self, X, ft, f):
        xe = np.asarray(X)[f]                                         # (nf, nnode, 3)
        a1 = np.einsum("fai,ga->fgi", xe, ft.dN[:, :, 0])
        a2 = np.einsum("fai,ga->fgi", xe, ft.dN[:, :, 1])
        return np.cross(a1, a2) * ft.gw[None, :, None]               # weighted normals (nf, ngp, 3)

    def integrate(self, X, field=None):
        """(nodal weights int N_a dA (nn,), area, area-weighted normal sum)."""
        w = np.zeros(len(X))
        area, nsum = 0.0, np.zeros(3)
        for ft, f in self.groups:
            n = self._jacobians(X, ft, f)
            da = np.linalg.norm(n, axis=-1)
            mult = 1.0 if field is None else np.asarray(field)[:, None]
            np.add.at(w, f, np.einsum("fg,ga->fa", da * mult, ft.N))
            area += da.sum()
            nsum += n.sum((0, 1))
        return w, area, nsum


def orient_outward(X, ft, facets, centroids):
    """Flip the facets whose right-hand normal points toward their element's centroid."""
    c = np.asarray(X)[facets[:, :ft.ncorner]]
    if ft.ncorner == 3:
        n = np.cross(c[:, 1] - c[:, 0], c[:, 2] - c[:, 0])
    else:
        n = np.cross(c[:, 2] - c[:, 0], c[:, 3] - c[:, 1])
    inward = np.einsum("fi,fi->f", n, centroids - c.mean(1)) > 0
    out = facets.copy()
    out[inward] = ft.flip(facets[inward])
    return out


def skin(X, blocks):
    """Faces of the blocks' elements that no other element shares, outward oriented,
    grouped by block then local face index, elements ascending inside a group."""
    X = np.asarray(X)
    keys, owners = [], []
    for bi, b in enumerate(blocks):
        conn = np.asarray(b.conn.cpu() if hasattr(b.conn, "cpu") else b.conn, dtype=np.int64)
        et = b.etype
        for k, loc in enumerate(et.faces):
            ft = FACETS[len(loc)]
            corners = np.sort(conn[:, loc[:ft.ncorner]], axis=1)
            if ft.ncorner == 3:                              # one key width for triangles and quads
                corners = np.hstack([np.full((len(conn), 1), -1), corners])
            keys.append(corners)
            owners.append(np.stack([np.full(len(conn), bi), np.arange(len(conn)), np.full(len(conn), k)], 1))
    s = Surface(name="skin")
    if not keys:
        return s
    keys, owners = np.concatenate(keys), np.concatenate(owners)
    _, inv, cnt = np.unique(keys, axis=0, return_inverse=True, return_counts=True)
    own = owners[cnt[inv.ravel()] == 1]
    for bi in np.unique(own[:, 0]):
        b = blocks[bi]
        conn = np.asarray(b.conn.cpu() if hasattr(b.conn, "cpu") else b.conn, dtype=np.int64)
        sel = own[own[:, 0] == bi]
        for k in np.unique(sel[:, 2]):
            el = sel[sel[:, 2] == k, 1]
            loc = b.etype.faces[k]
            ft = FACETS[len(loc)]
            cen = X[conn[el, :b.etype.ncorner]].mean(1)
            s.add(ft, orient_outward(X, ft, conn[el][:, loc], cen))
    return s


def sub_surface(surface, node_set):
    """Facets of ``surface`` whose corner nodes all belong to ``node_set``."""
    nodes = np.asarray(list(node_set), dtype=np.int64)
    size = int(max(surface.nodes().max(initial=0), nodes.max(initial=0))) + 1
    mask = np.zeros(size, bool)
    mask[nodes] = True
    out = Surface(name="sub")
    for ft, f in surface.groups:
        out.add(ft, f[mask[f[:, :ft.ncorner]].all(1)])
    return out
