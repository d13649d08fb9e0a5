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
    f = np.zeros_like(X, dtype=np.float64)
    for ft, fac in surface.groups:
        n = surface._jacobians(X, ft, fac)                           # (nf, ngp, 3)
        np.add.at(f, fac, -p * np.einsum("fgi,ga->fai", n, ft.N))
    return f.ravel()


def traction_vector(X, surface, t):
    w, _, _ = surface.integrate(X)
    return (w[:, None] * np.asarray(t, float)[None]).ravel()
