"""Oracle: element library, materials, element kernels, index maps, global operators.

Test infrastructure only (see ``oracle/__init__.py``).  CPU, FP64, torch.func AD.

Restates, in order:
  * gfem/elements.py:11-39   ``_tabulate`` / ``ElementType`` (N, dN by AD at set-up)
  * gfem/elements.py:76-92   TRI6 facet (config 3 pressure load)
  * gfem/elements.py:113-125 HEX8 = C3D8 with ``fbar=True`` (B-bar for small strain)
  * gfem/elements.py:166-179 TET10 = C3D10, 4-point rule a/b, w = 1/24
  * gfem/materials.py:18-19, 56-68       ``lame``, ``LinearElastic``
  * gfem/materials.py:224-302            ``_safe_norm``, ``J2Plasticity``
  * gfem/model.py:28-111, 129-137        geom, B-bar defgrad, stress, force, stiff, cauchy
  * gfem/model.py:157-158, 162-192       dofs, ops_matvec, ops_diagonal, ops_assemble
  * gfem/model.py:241-267                gather_plan, gather_matvec
  * gfem/model.py:449-490, 530-539       fields/scale, internal_force, element_stiffness,
                                          stiffness_ops, tangent_jvp, stresses
plus two index maps that the reference does not have but the CUDA path uses and
which are checked bit for bit: the greedy element colouring and the element-tile
node maps.
"""
import numpy as np
import torch
from torch.func import jacfwd, jvp, vjp, vmap

DT = torch.float64
I3 = torch.eye(3, dtype=DT)


def _t(a):
    return torch.as_tensor(np.asarray(a, dtype=np.float64))


# ---------------------------------------------------------------- shape functions
_H = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
               [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], float)   # elements.py:114-115
_HT = torch.as_tensor(_H)
_EDGES10 = [(0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3)]             # elements.py:167
_TA, _TB = 0.5854101966249685, 0.1381966011250105                        # elements.py:175


def _hexN(p):                                                          # elements.py:120-121
    return 0.125 * (1 + _HT[:, 0] * p[0]) * (1 + _HT[:, 1] * p[1]) * (1 + _HT[:, 2] * p[2])


def _L(p):                                                             # elements.py:160-161
    return torch.stack([1 - p[0] - p[1] - p[2], p[0], p[1], p[2]])


def _tet10N(p):                                                        # elements.py:170-172
    L = _L(p)
    return torch.cat([L * (2 * L - 1), torch.stack([4 * L[i] * L[j] for i, j in _EDGES10])])


def _tri6N(p):                                                         # elements.py:86-92
    L = torch.stack([1 - p[0] - p[1], p[0], p[1]])
    return torch.cat([L * (2 * L - 1), torch.stack([4 * L[0] * L[1], 4 * L[1] * L[2], 4 * L[2] * L[0]])])


def _tabulate(Nfun, pts):                                              # elements.py:11-15
    pts = torch.as_tensor(np.asarray(pts, float))
    N = torch.stack([Nfun(p) for p in pts])
    dN = torch.stack([jacfwd(Nfun)(p) for p in pts])
    return N, dN


class ElementType:
    """Volume element: N (ngp, nn) and dN (ngp, nn, 3) tabulated by AD (elements.py:18-39)."""

    def __init__(self, name, nnode, gp, gw, Nfun, fbar=False, center=None, ncorner=None):
        self.name, self.nnode = name, nnode
        self.gp, self.gw = np.asarray(gp, float), np.asarray(gw, float)
        self.ngp = len(self.gw)
        self.Nfun = Nfun
        self.N, self.dN = _tabulate(Nfun, self.gp)
        self.w = torch.as_tensor(self.gw)
        self.fbar = fbar
        self.dN0 = _tabulate(Nfun, [center])[1][0] if center is not None else None
        self.ncorner = ncorner or nnode


class FacetType:
    """Surface facet: N (ngp, nn), dN (ngp, nn, 2) (elements.py:42-49)."""

    def __init__(self, name, nnode, gp, gw, Nfun):
        self.name, self.nnode = name, nnode
        self.gp, self.gw = np.asarray(gp, float), np.asarray(gw, float)
        N, dN = _tabulate(Nfun, self.gp)
        self.N, self.dN = N.numpy(), dN.numpy()


HEX8 = ElementType("C3D8", 8, _H / np.sqrt(3), np.ones(8), _hexN, fbar=True, center=[0, 0, 0])
HEX8_PLAIN = ElementType("C3D8_FULL", 8, _H / np.sqrt(3), np.ones(8), _hexN)
TET10 = ElementType("C3D10", 10, [[_TB, _TB, _TB], [_TA, _TB, _TB], [_TB, _TA, _TB], [_TB, _TB, _TA]],
                    [1 / 24] * 4, _tet10N, ncorner=4)
TRI6 = FacetType("TRI6", 6, [[1 / 6, 1 / 6], [2 / 3, 1 / 6], [1 / 6, 2 / 3]], [1 / 6] * 3, _tri6N)
ELEMENTS = {"C3D8": HEX8, "C3D8_FULL": HEX8_PLAIN, "C3D10": TET10}


# ---------------------------------------------------------------- materials
def lame(E, nu):                                                       # materials.py:18-19
    return E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))


class LinearElastic:
    """materials.py:56-68: sigma = lam tr(eps) I + 2 mu eps, eps = sym(F) - I."""
    nstate = 1
    small_strain = True

    def __init__(self, E, nu, density=1.0):
        self.E, self.nu, self.density = float(E), float(nu), float(density)
        self.mu, self.lam = lame(self.E, self.nu)

    def pk1(self, F, s):
        eps = 0.5 * (F + F.T) - I3
        return self.lam * torch.trace(eps) * I3 + 2 * self.mu * eps, s

    def eqps(self, s):
        return 0.0 * s[..., 0]


def _interp(x, xp, fp):
    """np.interp semantics as used by ``jnp.interp`` in materials.py:260: segment
    i = clip(#(xp <= x), 1, n-1), linear inside, clamped to the end values outside."""
    n = xp.shape[0]
    c = (xp <= x).to(torch.int64).sum()
    i = torch.clamp(c, 1, n - 1)
    ar = torch.arange(n)
    hi, lo = (ar == i).to(DT), (ar == i - 1).to(DT)
    x0, x1 = (lo * xp).sum(), (hi * xp).sum()
    f0, f1 = (lo * fp).sum(), (hi * fp).sum()
    dx, df = x1 - x0, f1 - f0
    eps = float(np.spacing(np.finfo(np.float64).eps))
    dx0 = torch.abs(dx) <= eps
    f = torch.where(dx0, f0, f0 + ((x - x0) / torch.where(dx0, torch.ones_like(dx), dx)) * df)
    f = torch.where(x < xp[0], fp[0], f)
    f = torch.where(x > xp[-1], fp[-1], f)
    return f


def _interp_slope(x, xp, fp):
    """d/dx of ``_interp`` (what ``jax.grad(self.sy)`` returns in materials.py:282):
    the segment slope inside the table, 0 where the value is clamped."""
    n = xp.shape[0]
    c = (xp <= x).to(torch.int64).sum()
    i = torch.clamp(c, 1, n - 1)
    ar = torch.arange(n)
    hi, lo = (ar == i).to(DT), (ar == i - 1).to(DT)
    dx = (hi * xp).sum() - (lo * xp).sum()
    df = (hi * fp).sum() - (lo * fp).sum()
    eps = float(np.spacing(np.finfo(np.float64).eps))
    dx0 = torch.abs(dx) <= eps
    s = torch.where(dx0, torch.zeros_like(dx), df / torch.where(dx0, torch.ones_like(dx), dx))
    s = torch.where(x < xp[0], torch.zeros_like(s), s)
    s = torch.where(x > xp[-1], torch.zeros_like(s), s)
    return s


def _safe_norm(a):                                                     # materials.py:224-225
    return torch.sqrt(torch.sum(a * a) + 1e-30)


class J2Plasticity:
    """materials.py:228-302: small-strain von Mises, table isotropic hardening
    (linearly extended to eps_p = 1e6), linear kinematic Hk, radial return with a
    fixed 25-iteration local Newton.  State = [eps_p (9), alpha, beta (9)]."""
    nstate = 19
    small_strain = True

    def __init__(self, E, nu, table, Hk=0.0):
        self.E, self.nu = float(E), float(nu)
        self.mu, self.lam = lame(self.E, self.nu)
        self.K = self.lam + 2 * self.mu / 3
        self.Hk = float(Hk)
        t = np.asarray(table, dtype=np.float64).reshape(-1, 2)
        if t.shape[0] == 1:
            t = np.array([[t[0, 0], 0.0], [t[0, 0], 1e3]])
        sy_tab, ep_tab = t[:, 0], t[:, 1]
        slope = (sy_tab[-1] - sy_tab[-2]) / max(ep_tab[-1] - ep_tab[-2], 1e-30)
        self.ep_tab_np = np.append(ep_tab, 1e6)
        self.sy_tab_np = np.append(sy_tab, sy_tab[-1] + slope * (1e6 - ep_tab[-1]))
        self.ep_tab = torch.as_tensor(self.ep_tab_np)
        self.sy_tab = torch.as_tensor(self.sy_tab_np)
        self.table = t
        self.sy0 = float(t[0, 0])

    def sy(self, a):
        return _interp(a, self.ep_tab, self.sy_tab)

    def dsy(self, a):
        return _interp_slope(a, self.ep_tab, self.sy_tab)

    def eqps(self, s):
        return s[..., 9]

    def _return(self, eps, s):                                         # materials.py:270-296
        mu = self.mu
        ep = s[:9].reshape(3, 3)
        a0 = s[9]
        beta = s[10:19].reshape(3, 3)
        ee = eps - ep
        tr = torch.trace(ee)
        dev = ee - tr / 3 * I3
        s_tr = 2 * mu * dev
        xi = s_tr - beta
        q_tr = np.sqrt(1.5) * _safe_norm(xi)
        f_tr = q_tr - self.sy(a0)
        H3 = 3 * mu + self.Hk
        dg = torch.zeros((), dtype=DT)
        for _ in range(25):
            g = q_tr - H3 * dg - self.sy(a0 + dg)
            dg = torch.clamp(dg + g / (H3 + self.dsy(a0 + dg)), min=0.0)
        dg = torch.where(f_tr > 0, dg, torch.zeros_like(dg))
        n = 1.5 * xi / (q_tr + 1e-30)
        s_dev = s_tr - 2 * mu * dg * n
        sig = s_dev + self.K * tr * I3
        ep_new = ep + dg * n
        beta_new = beta + (2.0 / 3.0) * self.Hk * dg * n
        s_new = torch.cat([ep_new.reshape(-1), (a0 + dg).reshape(1), beta_new.reshape(-1)])
        return sig, s_new

    def pk1(self, F, s):
        return self._return(0.5 * (F + F.T) - I3, s)


# ---------------------------------------------------------------- element kernels
class Block:
    """One element type + one material (model.py:21-158).  Kernels are vmapped over
    the leading element axis; ``chunk`` bounds the working set of the AD tangents."""

    def __init__(self, conn, etype, material, chunk=4096):
        self.conn = np.asarray(conn, dtype=np.int64)
        self.etype, self.material = etype, material
        self.ne = int(self.conn.shape[0])
        self.chunk = chunk
        self._build()

    def _build(self):
        et, mat = self.etype, self.material
        dN, w, N = et.dN, et.w, et.N
        dN0 = et.dN0 if et.fbar else None

        def geom(Xe):                                                  # model.py:35-38
            Jac = torch.einsum("an,gai->gni", Xe, dN)
            dNdX = torch.einsum("gai,gij->gaj", dN, torch.linalg.inv(Jac))
            return dNdX, w * torch.linalg.det(Jac)

        def defgrad(Xe, ue, dNdX):                                     # model.py:40-52
            F = I3 + torch.einsum("ai,gaj->gij", ue, dNdX)
            if et.fbar:                                                # B-bar (small strain)
                J0inv = torch.linalg.inv(Xe.T @ dN0)
                F0 = I3 + ue.T @ (dN0 @ J0inv)
                tr0 = torch.trace(F0) - 3.0
                tr = torch.diagonal(F, dim1=1, dim2=2).sum(-1) - 3.0
                F = F + ((tr0 - tr) / 3.0)[:, None, None] * I3
            return F

        def stress(F, se, eig):                                        # model.py:54-68 (T = T0)
            return vmap(lambda f, s: mat.pk1(f - eig, s))(F, se)

        def force(Xe, ue, se, scv):                                    # model.py:70-81
            sc, eig = scv[0], scv[1:10].reshape(3, 3)
            dNdX, vol = geom(Xe)
            if et.fbar:
                F, pullback = vjp(lambda u: defgrad(Xe, u, dNdX), ue)
                P, snew = stress(F, se, eig)
                fe = pullback(P * (sc * vol)[:, None, None])[0]
            else:
                F = defgrad(Xe, ue, dNdX)
                P, snew = stress(F, se, eig)
                fe = torch.einsum("gij,gaj,g->ai", P, dNdX, sc * vol)
            return fe, snew

        def stiff(Xe, ue, se, scv):                                    # model.py:83-111
            nn = ue.shape[0]
            sc, eig = scv[0], scv[1:10].reshape(3, 3)
            dNdX, vol = geom(Xe)
            stress_P = lambda f, s: mat.pk1(f - eig, s)[0]
            if et.fbar:
                Fmap = lambda u: defgrad(Xe, u, dNdX)
                F = Fmap(ue)
                G = jacfwd(Fmap)(ue)                                   # (ngp, 3, 3, nn, 3)
                A = vmap(jacfwd(stress_P))(F, se)                      # (ngp, 3, 3, 3, 3)
                K = torch.einsum("gijak,gijlm,glmbn,g->akbn", G, A, G, sc * vol)
                return K.reshape(nn * 3, nn * 3)
            F = defgrad(Xe, ue, dNdX)
            A = vmap(jacfwd(stress_P))(F, se)
            K = torch.einsum("gaj,gijkl,gbl,g->aibk", dNdX, A, dNdX, sc * vol)
            return K.reshape(nn * 3, nn * 3)

        def cauchy(Xe, ue, se, scv):                                   # model.py:129-137
            dNdX, vol = geom(Xe)
            F = defgrad(Xe, ue, dNdX)
            P, snew = stress(F, se, scv[1:10].reshape(3, 3))
            wv = vol / vol.sum()
            return (torch.einsum("g,gij->ij", wv, P), torch.einsum("g,g->", wv, mat.eqps(snew)),
                    torch.einsum("g,gij->ij", wv, F))

        def geo_stiff(Xe, sig):                                        # model.py:113-117
            dNdX, vol = geom(Xe)
            k = torch.einsum("gai,ij,gbj,g->ab", dNdX, sig, dNdX, vol)
            n = k.shape[0]
            return torch.einsum("ab,ij->aibj", k, I3).reshape(n * 3, n * 3)

        self._geom, self._defgrad = geom, defgrad
        self._force, self._stiff, self._cauchy = vmap(force), vmap(stiff), vmap(cauchy)
        self._geo_stiff = vmap(geo_stiff)

    def _chunks(self, fn, *args):
        outs = []
        for a in range(0, self.ne, self.chunk):
            outs.append(fn(*[x[a:a + self.chunk] for x in args]))
        if isinstance(outs[0], tuple):
            return tuple(torch.cat([o[k] for o in outs]) for k in range(len(outs[0])))
        return torch.cat(outs)

    def force(self, Xe, ue, se, scv):
        return self._chunks(self._force, Xe, ue, se, scv)

    def stiff(self, Xe, ue, se, scv):
        return self._chunks(self._stiff, Xe, ue, se, scv)

    def cauchy(self, Xe, ue, se, scv):
        return self._chunks(self._cauchy, Xe, ue, se, scv)

    def geo_stiff(self, Xe, sig):
        return self._chunks(self._geo_stiff, Xe, sig)

    def init_state(self):                                              # model.py:154-155
        return torch.zeros((self.ne, self.etype.ngp, self.material.nstate), dtype=DT)

    def dofs(self):                                                    # model.py:157-158
        return (self.conn[:, :, None] * 3 + np.arange(3)).reshape(self.ne, -1)


# ---------------------------------------------------------------- EbE operators
def ops_matvec(ops, v, ndof):                                          # model.py:162-166
    out = torch.zeros(ndof, dtype=v.dtype)
    for d, K in ops:
        d = torch.as_tensor(d)
        out.index_add_(0, d.reshape(-1), torch.einsum("eij,ej->ei", K, v[d]).reshape(-1))
    return out


def ops_diagonal(ops, ndof):                                           # model.py:169-173
    out = torch.zeros(ndof, dtype=DT)
    for d, K in ops:
        d = torch.as_tensor(d)
        out.index_add_(0, d.reshape(-1), torch.diagonal(K, dim1=1, dim2=2).reshape(-1))
    return out


def ops_assemble(ops, ndof):                                           # model.py:176-192
    import scipy.sparse as sp
    rows, cols, vals = [], [], []
    for d, K in ops:
        d = np.asarray(d)
        K = np.asarray(K)
        nd = d.shape[1]
        rows.append(np.repeat(d, nd, axis=1).ravel())
        cols.append(np.tile(d, (1, nd)).ravel())
        vals.append(K.reshape(len(d), -1).ravel())
    if not rows:
        return sp.csr_matrix((ndof, ndof))
    A = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(ndof, ndof)).tocsr()
    A.sum_duplicates()
    return A


def gather_plan(conns, nn):                                            # model.py:241-261
    """For every node the stable-sorted list of flat element slots elem*nnode+local
    that touch it, padded to the max valence with the sentinel ``off`` (a zero row)."""
    slots, nodes = [], []
    off = 0
    for c in conns:
        c = np.asarray(c)
        nodes.append(c.ravel())
        slots.append(off + np.arange(c.size))
        off += c.size
    nodes, slots = np.concatenate(nodes), np.concatenate(slots)
    order = np.argsort(nodes, kind="stable")
    nodes, slots = nodes[order], slots[order]
    cnt = np.bincount(nodes, minlength=nn)
    vmax = max(int(cnt.max()), 1)
    start = np.concatenate([[0], np.cumsum(cnt)[:-1]])
    pos = np.arange(len(nodes)) - start[nodes]
    g = np.full((nn, vmax), off, np.int64)
    g[nodes, pos] = slots
    return g.astype(np.int32 if off < 2 ** 31 else np.int64)


def gather_matvec(plan, ops, v, ndof):                                 # model.py:264-267
    parts = [torch.einsum("eij,ej->ei", K, v[torch.as_tensor(d)]).reshape(-1, 3) for d, K in ops]
    ys = torch.cat(parts + [torch.zeros((1, 3), dtype=v.dtype)])
    return torch.sum(ys[torch.as_tensor(plan, dtype=torch.int64)], dim=1).reshape(-1)


def greedy_colouring(conn, nn):
    """Element colouring used by the deterministic scatter (no counterpart in the
    reference, which assembles with ``gather_plan``).  Elements are visited in
    index order; each takes the smallest colour not yet used by any element that
    shares a node with it.  Returns int32 colours (ne,)."""
    conn = np.asarray(conn)
    used = [0] * nn                       # per node: bitmask of colours already taken
    col = np.empty(len(conn), np.int32)
    for e, row in enumerate(conn.tolist()):
        m = 0
        for a in row:
            m |= used[a]
        c = 0
        while (m >> c) & 1:
            c += 1
        col[e] = c
        bit = 1 << c
        for a in row:
            used[a] |= bit
    return col


def tile_order(X, conn, ncorner):
    """Tile order of the matrix-free product (no counterpart in the reference),
    position -> element.  Elements are grouped by connected component (elements
    sharing nodes), components in the order of their first element; inside a
    component they follow a Morton curve of the corner-coordinate sums s_e (corner
    nodes summed in local order), quantised per axis as
    min(floor((s - lo) / (hi - lo) * 2^21), 2^21 - 1) over the extent [lo, hi] of
    all sums, bits interleaved x lowest; ties by element index."""
    X = np.asarray(X, dtype=np.float64)
    conn = np.asarray(conn, dtype=np.int64)
    ne, nnode = conn.shape
    if ne == 0:
        return np.zeros(0, np.int32)
    import scipy.sparse as sps
    from scipy.sparse.csgraph import connected_components
    nn = len(X)
    rows = np.repeat(np.arange(ne), nnode)
    G = sps.csr_matrix((np.ones(ne * nnode), (rows, ne + conn.reshape(-1))), shape=(ne + nn, ne + nn))
    _, lab = connected_components(G, directed=False)
    first = np.full(lab.max() + 1, ne, np.int64)
    np.minimum.at(first, lab[:ne], np.arange(ne))
    comp = first[lab[:ne]]
    s = X[conn[:, 0]].copy()
    for a in range(1, ncorner):
        s = s + X[conn[:, a]]
    lo, hi = s.min(0), s.max(0)
    key = np.zeros(ne, np.uint64)
    for d in range(3):
        if hi[d] > lo[d]:
            f = np.floor((s[:, d] - lo[d]) / (hi[d] - lo[d]) * 2097152.0)
            q = np.minimum(np.maximum(f, 0.0), 2097151.0).astype(np.uint64)
        else:
            q = np.zeros(ne, np.uint64)
        for b in range(21):
            key |= ((q >> np.uint64(b)) & np.uint64(1)) << np.uint64(3 * b + d)
    return np.lexsort((np.arange(ne), key, comp)).astype(np.int32)


_TET_EDGES = ((0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3))


def _even(p):
    return sum(p[i] > p[j] for i in range(4) for j in range(i + 1, 4)) % 2 == 0


def _tet10_permuted(c, pi):
    out = [c[pi[i]] for i in range(4)]
    for a, b in _TET_EDGES:
        k = next(k for k, (x, y) in enumerate(_TET_EDGES) if {x, y} == {pi[a], pi[b]})
        out.append(c[4 + k])
    return out


def tile_pairs(order, conn, window=16):
    """Face pairs of a C3D10 tile order (no counterpart in the reference).  Walking
    the order, each element not yet placed takes the first unplaced element among
    the next `window` positions that shares three corners with it; pairs and the
    remaining singles keep the order of their first element and consecutive singles
    go side by side.  A pair (e, f) sharing face corners p, q, r gets local corners
    (p, q, r, s) for e -- the first even permutation (lexicographic) of e's corners
    with its off-face corner s last -- and (q, p, r, t) for f when that is an even
    permutation of f's corners (else both keep their numbering); mid-edge nodes
    follow their corners.  Returns (order, conn_tile)."""
    import itertools
    conn = np.asarray(conn, dtype=np.int64)
    order = [int(e) for e in order]
    ne = len(order)
    used = np.zeros(conn.shape[0], bool)
    units = []
    for k, e in enumerate(order):
        if used[e]:
            continue
        used[e] = True
        mate = -1
        for m in range(k + 1, min(ne, k + window + 1)):
            f = order[m]
            if not used[f] and len(set(conn[e, :4]) & set(conn[f, :4])) == 3:
                mate = f
                break
        if mate >= 0:
            used[mate] = True
        units.append((e, mate))
    out_o, out_c = [], []

    def emit(e, pi=None):
        out_o.append(e)
        out_c.append(list(conn[e]) if pi is None else _tet10_permuted(list(conn[e]), pi))

    pending = -1
    for e, f in units:
        if f < 0:
            if pending < 0:
                pending = e
            else:
                emit(pending)
                emit(e)
                pending = -1
            continue
        ce, cf = list(conn[e, :4]), list(conn[f, :4])
        se = next(i for i in range(4) if ce[i] not in cf)
        tf = next(i for i in range(4) if cf[i] not in ce)
        pe = next((list(p) for p in itertools.permutations(range(4)) if p[3] == se and _even(p)), None)
        pf = None
        if pe is not None:
            want = [ce[pe[1]], ce[pe[0]], ce[pe[2]], cf[tf]]
            pf = [cf.index(w) for w in want]
            if not _even(pf):
                pf = None
        if pf is not None:
            emit(e, pe)
            emit(f, pf)
        else:
            emit(e)
            emit(f)
    if pending >= 0:
        emit(pending)
    return np.asarray(out_o, np.int32), np.asarray(out_c, np.int32).reshape(-1, conn.shape[1])


def tile_maps(conn, tile):
    """Element-tile maps used by the matrix-free product (no counterpart in the
    reference), for conn given in tile order.  Positions [t*tile, (t+1)*tile) form
    tile t; slot s = a*tile + p is local node a of the element at tile position p.
    Per tile: the sorted distinct nodes; for each node (in that order) its slots in
    increasing order, concatenated into perm (padded with zeros to nnode*tile per
    tile); nend = end of each node's run.
    Returns (ptr (ntile+1,), nodes, nend, perm (ntile, nnode*tile))."""
    conn = np.asarray(conn, dtype=np.int64)
    ne, nnode = conn.shape
    ntile = -(-ne // tile)
    ptr, nodes, nend = [0], [], []
    perm = np.zeros((ntile, nnode * tile), np.uint16)
    for t in range(ntile):
        blk = conn[t * tile:(t + 1) * tile]
        u = np.unique(blk)
        slot_node = np.searchsorted(u, blk.T.reshape(-1))        # slot order a*tile + p (valid p only)
        la = np.arange(blk.shape[0])
        slots = (np.arange(nnode)[:, None] * tile + la[None, :]).reshape(-1)
        order = np.argsort(slot_node, kind="stable")
        perm[t, :len(order)] = slots[order]
        nend.append(np.cumsum(np.bincount(slot_node, minlength=len(u))))
        nodes.append(u)
        ptr.append(ptr[-1] + len(u))
    cat = (lambda xs, dt: np.concatenate(xs).astype(dt) if xs else np.zeros(0, dt))
    return np.asarray(ptr, np.int32), cat(nodes, np.int32), cat(nend, np.uint16), perm


# ---------------------------------------------------------------- model
class Model:
    """Nodes + element blocks with the reference's global operators (model.py:270-539)."""

    def __init__(self, nodes):
        self.X = torch.as_tensor(np.asarray(nodes, dtype=np.float64))
        self.nn = int(self.X.shape[0])
        self.ndof = 3 * self.nn
        self.blocks = []
        self._plan = None

    def add_block(self, conn, etype, material, chunk=4096):
        b = Block(conn, etype, material, chunk)
        self.blocks.append(b)
        self._plan = None
        return b

    def init_state(self):
        return [b.init_state() for b in self.blocks]

    def gather(self):
        if self._plan is None:
            self._plan = gather_plan([b.conn for b in self.blocks], self.nn)
        return self._plan

    def _scv(self, scale):                                             # model.py:449-463
        out = []
        sc = scale or [None] * len(self.blocks)
        for b, s in zip(self.blocks, sc):
            s = torch.ones(b.ne, dtype=DT) if s is None else torch.as_tensor(np.asarray(s, np.float64))
            out.append(torch.cat([s[:, None], torch.zeros((b.ne, 9), dtype=DT)], 1))
        return out

    def element_forces(self, u, states, scale=None):
        U = torch.as_tensor(u).reshape(-1, 3)
        return [b.force(self.X[b.conn], U[b.conn], s, c)
                for b, s, c in zip(self.blocks, states, self._scv(scale))]

    def internal_force(self, u, states, scale=None):                   # model.py:466-477
        new, parts = [], []
        for fe, sn in self.element_forces(u, states, scale):
            parts.append(fe.reshape(-1, 3))
            new.append(sn)
        if not parts:
            return torch.zeros(self.ndof, dtype=DT), new
        ys = torch.cat(parts + [torch.zeros((1, 3), dtype=parts[0].dtype)])
        plan = torch.as_tensor(self.gather(), dtype=torch.int64)
        return torch.sum(ys[plan], dim=1).reshape(-1), new

    def element_stiffness(self, u, states, scale=None):                # model.py:479-483
        U = torch.as_tensor(u).reshape(-1, 3)
        return [b.stiff(self.X[b.conn], U[b.conn], s, c)
                for b, s, c in zip(self.blocks, states, self._scv(scale))]

    def stiffness_ops(self, u, states, scale=None):                    # model.py:485-486
        return list(zip([b.dofs() for b in self.blocks], self.element_stiffness(u, states, scale)))

    def tangent_jvp(self, u, states, v, scale=None):                   # model.py:488-490
        u = torch.as_tensor(u)
        return jvp(lambda x: self.internal_force(x, states, scale)[0], (u,), (torch.as_tensor(v),))[1]

    def geometric_ops(self, stresses):                                 # model.py:541-553
        return [(b.dofs(), b.geo_stiff(self.X[b.conn], st["S"])) for b, st in zip(self.blocks, stresses)]

    def stresses(self, u, states, scale=None):                         # model.py:530-539
        U = torch.as_tensor(u).reshape(-1, 3)
        out = []
        for b, s, c in zip(self.blocks, states, self._scv(scale)):
            sig, ep, F = b.cauchy(self.X[b.conn], U[b.conn], s, c)
            dev = sig - (torch.diagonal(sig, dim1=1, dim2=2).sum(-1) / 3)[:, None, None] * I3
            mises = torch.sqrt(1.5 * torch.sum(dev * dev, dim=(1, 2)))
            out.append(dict(S=sig, MISES=mises, PEEQ=ep, F=F))
        return out


def lumped_mass(model):                                                # model.py:120-124, 501-510
    """HRZ diagonal lumping per element, d_a = rho sum_g vol_g N_a(g)^2 scaled to
    rho * element volume, summed at the nodes and repeated for the 3 DOFs."""
    m = np.zeros(model.nn)
    for b in model.blocks:
        et, rho = b.etype, float(getattr(b.material, "density", 1.0))
        Xe = model.X[torch.as_tensor(b.conn)]                           # (ne, nnode, 3)
        Jac = torch.einsum("ean,gai->egni", Xe, et.dN)
        vol = et.w[None, :] * torch.linalg.det(Jac)                     # (ne, ngp)
        d = rho * torch.einsum("eg,ga->ea", vol, et.N * et.N)
        d = d * (rho * vol.sum(1))[:, None] / d.sum(1)[:, None]
        np.add.at(m, b.conn, d.numpy())
    return np.repeat(m, 3)
