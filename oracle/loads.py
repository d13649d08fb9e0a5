"""Oracle: boundary skin and uniform-pressure load vector (config-3 right-hand side).

Test infrastructure only (see ``oracle/__init__.py``).

  * gfem/elements.py:176       TET10 faces as TRI6 facets (corner nodes first)
  * gfem/surfaces.py:155-168   ``orient_outward`` (flip facets whose normal points
                               toward the owning element's centroid; TRI6 flip order)
  * gfem/surfaces.py:182-221   ``skin`` (faces owned by exactly one element)
  * gfem/surfaces.py:234-242   ``sub_surface`` (facets whose corners are all in a node set)
  * gfem/loads.py:39-51        ``pressure_vector`` f_a = -p int N_a n dA, reference config.
"""
import numpy as np

from .fem import TRI6

TET10_FACES = [[0, 1, 2, 4, 5, 6], [0, 3, 1, 7, 8, 4], [1, 3, 2, 8, 9, 5], [2, 3, 0, 9, 7, 6]]


def skin_tet10(X, conn):
    X = np.asarray(X)
    conn = np.asarray(conn)
    faces = np.concatenate([conn[:, loc] for loc in TET10_FACES])
    owner = np.concatenate([np.arange(len(conn))] * len(TET10_FACES))
    keys = np.sort(faces[:, :3], axis=1)
    _, inv, cnt = np.unique(keys, axis=0, return_inverse=True, return_counts=True)
    bnd = cnt[inv.ravel()] == 1
    f, own = faces[bnd], owner[bnd]
    cen = X[conn[own, :4]].mean(1)
    c = X[f[:, :3]]
    n = np.cross(c[:, 1] - c[:, 0], c[:, 2] - c[:, 0])
    inward = np.einsum("fi,fi->f", n, cen - c.mean(1)) > 0
    out = f.copy()
    out[inward] = f[inward][:, [0, 2, 1, 5, 4, 3]]
    return out


def sub_surface(facets, node_set, nn):
    mask = np.zeros(nn, bool)
    mask[np.asarray(node_set, dtype=np.int64)] = True
    return facets[mask[facets[:, :3]].all(1)]


def pressure_vector(X, facets, p):
    X = np.asarray(X)
    f = np.zeros_like(X)
    xe = X[facets]
    a1 = np.einsum("fai,ga->fgi", xe, TRI6.dN[:, :, 0])
    a2 = np.einsum("fai,ga->fgi", xe, TRI6.dN[:, :, 1])
    n = np.cross(a1, a2) * TRI6.gw[None, :, None]
    fe = -p * np.einsum("fgi,ga->fai", n, TRI6.N)
    np.add.at(f, facets, fe)
    return f.ravel()
