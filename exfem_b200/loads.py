"""Dead-load vectors (drop-in names of ``gfem.loads``), host set-up.

  * ``cload_vector`` — concentrated nodal loads (gfem/loads.py:31-34);
  * ``pressure_vector`` — equivalent nodal forces of a uniform pressure p
    (positive into the surface) on the reference configuration,
    f_a = -p sum_g w_g N_a(g) (dx/ds x dx/dt)(g) (gfem/loads.py:37-49);
  * ``traction_vector`` — a uniform traction t on a surface, f_a = t int N_a dA
    (gfem/loads.py:52-56).

Vectors are (ndof,) FP64 NumPy arrays, node-interleaved (dof = 3 node + c).
"""
import numpy as np


def cload_vector(ndof, nodes, dof, value):
    f = np.zeros(ndof)
    np.add.at(f, np.asarray(nodes, dtype=np.int64) * 3 + dof, value)
    return f


def pressure_vector(X, surface, p):
    X = np.asarray(X)
    nn = len(X)
    f = np.zeros((nn, 3))
    for ft, fac in surface.groups:
        n = ft.area_vectors(X, fac)                                   # (nf, ngp, 3)
        fe = -p * np.matmul(ft.N.T, n)                                # (nf, nnode, 3)
        for c in range(3):
            f[:, c] += np.bincount(fac.reshape(-1), weights=fe[..., c].reshape(-1), minlength=nn)
    return f.ravel()


def traction_vector(X, surface, t):
    w, _, _ = surface.integrate(X)
    return (w[:, None] * np.asarray(t, float)[None]).ravel()
