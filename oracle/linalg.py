"""Oracle: linear algebra of the reference, restated in NumPy/SciPy FP64.

Test infrastructure only (see ``oracle/__init__.py``).

  * gfem/linalg.py:21-47    ``pcg`` (x0 = 0, stop when r.r <= tol^2 b.b or k >= maxiter,
                             returns (x, k, sqrt(r.r / b.b)))
  * gfem/linalg.py:51-77    ``csr_to_device`` ELL-or-CSR rule and ``csr_mv``
  * gfem/linalg.py:80-98    ``rigid_body_modes``
  * gfem/linalg.py:138-146  ``AMG._rho`` power iteration (seed 0, 15 iterations, x1.1)
  * gfem/linalg.py:126-133  coarse dense Cholesky with 1e-13 regularisation
  * gfem/linalg.py:156-195  ``AMG.make``: Chebyshev smoother on D^-1 A over [rho/30, rho]
                             and the V-cycle (level 0 may use the current fine operator)
  * gfem/linalg.py:199-217  ``Direct`` (SuperLU, COLAMD) and ``bc_matrix``
"""
import numpy as np
import scipy.linalg
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def pcg(A, b, M=None, x0=None, tol=1e-8, maxiter=2000):                # linalg.py:21-47
    M = M or (lambda r: r)
    b = np.asarray(b, dtype=np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)
    r = b - A(x)
    z = M(r)
    p = z
    rz = float(np.dot(r, z))
    bn2 = max(float(np.dot(b, b)), 1e-300)
    tol2 = tol * tol * bn2
    k = 0
    rr = float(np.dot(r, r))
    while rr > tol2 and k < maxiter:
        Ap = A(p)
        alpha = rz / float(np.dot(p, Ap))
        x = x + alpha * p
        r = r - alpha * Ap
        rr = float(np.dot(r, r))
        z = M(r)
        rz_new = float(np.dot(r, z))
        p = z + (rz_new / rz) * p
        rz = rz_new
        k += 1
    return x, k, np.sqrt(rr / bn2)


def csr_to_device(A, ell_max_ratio=2.0):                               # linalg.py:51-70
    """Returns ('ell', data, cols) when the longest row is <= 2x the mean, else ('csr', A)."""
    A = A.tocsr()
    A.sort_indices()
    cnt = np.diff(A.indptr)
    n = A.shape[0]
    w = int(cnt.max()) if n else 0
    if n and w <= ell_max_ratio * max(cnt.mean(), 1.0):
        pos = np.arange(A.nnz) - np.repeat(A.indptr[:-1], cnt)
        rows = np.repeat(np.arange(n), cnt)
        cols = np.zeros((n, w), np.int32)
        data = np.zeros((n, w), A.data.dtype)
        cols[rows, pos] = A.indices
        data[rows, pos] = A.data
        return dict(kind="ell", ell_data=data, ell_cols=cols, n=n)
    return dict(kind="csr", A=A, n=n)


def csr_mv(M, x):                                                      # linalg.py:73-77
    if M["kind"] == "ell":
        return np.sum(M["ell_data"] * x[M["ell_cols"]], axis=1)
    return M["A"] @ x


def rigid_body_modes(X):                                               # linalg.py:80-98
    X = np.asarray(X)
    n = len(X)
    t = np.ones(n)
    c = (X - X[t > 0].mean(0)) * t[:, None]
    B = np.zeros((3 * n, 6))
    for i in range(3):
        B[i::3, i] = t
    x, y, z = c[:, 0], c[:, 1], c[:, 2]
    B[0::3, 3], B[1::3, 3] = -y, x
    B[1::3, 4], B[2::3, 4] = -z, y
    B[0::3, 5], B[2::3, 5] = z, -x
    return B


def rho_power(A, dinv, it=15):                                         # linalg.py:138-146
    x = np.random.default_rng(0).standard_normal(A.shape[0])
    lam = 1.0
    for _ in range(it):
        y = dinv * (A @ x)
        lam = np.linalg.norm(y) / max(np.linalg.norm(x), 1e-300)
        x = y / max(np.linalg.norm(y), 1e-300)
    return 1.1 * lam


def coarse_cholesky(Ac):                                               # linalg.py:126-133
    Ac = np.asarray(Ac, dtype=np.float64)
    Ac = 0.5 * (Ac + Ac.T)
    try:
        return np.linalg.cholesky(Ac + 1e-13 * np.abs(Ac).max() * np.eye(len(Ac)))
    except np.linalg.LinAlgError:
        w, V = np.linalg.eigh(Ac)
        return np.linalg.cholesky(V @ np.diag(np.maximum(w, 1e-12 * w.max())) @ V.T)


def level_dinv(A):                                                     # linalg.py:120-121
    d = A.diagonal()
    return np.where(np.abs(d) > 0, 1.0 / np.where(d == 0, 1, d), 0.0)


def cheb(Amv, dinv, rho, x, b, deg=2):                                 # linalg.py:161-175
    lmax, lmin = rho, rho / 30.0
    theta, delta = 0.5 * (lmax + lmin), 0.5 * (lmax - lmin)
    sigma = theta / delta
    rh = 1.0 / sigma
    r = dinv * (b - Amv(x))
    d = r / theta
    for _ in range(deg):
        x = x + d
        r = r - dinv * Amv(d)
        rh_new = 1.0 / (2 * sigma - rh)
        d = rh_new * rh * d + 2 * rh_new / delta * r
        rh = rh_new
    return x + d


def vcycle(levels, L, b, lvl=0, A0=None, dinv0=None, deg=2):           # linalg.py:177-192
    """``levels``: list of dict(A, dinv, rho, P, R) (scipy CSR); ``L``: coarse Cholesky factor."""
    if lvl == len(levels):
        y = scipy.linalg.solve_triangular(L, b, lower=True)
        return scipy.linalg.solve_triangular(L.T, y, lower=False)
    lv = levels[lvl]
    if lvl == 0 and A0 is not None:
        Amv, dinv = A0, dinv0
    else:
        Amv, dinv = (lambda v, A=lv["A"]: A @ v), lv["dinv"]
    x = cheb(Amv, dinv, lv["rho"], np.zeros_like(b), b, deg)
    r = b - Amv(x)
    xc = vcycle(levels, L, lv["R"] @ r, lvl + 1, deg=deg)
    x = x + lv["P"] @ xc
    return cheb(Amv, dinv, lv["rho"], x, b, deg)


def cheby_lmax(Amv, dinv, free, it=25):                               # solvers.py:328-342
    """Bound of the spectrum of D^-1 A by power iteration: start sin(0.37 i + 0.1)
    on the free DOFs plus 1e-3, 25 iterations, the last |w| / |v| times 1.1."""
    n = len(dinv)
    v = np.sin(np.arange(n) * 0.37 + 0.1) * free + 1e-3
    lam = 1.0
    for _ in range(it):
        w = dinv * Amv(v)
        lam = np.linalg.norm(w) / np.linalg.norm(v)
        v = w / np.linalg.norm(w)
    return 1.1 * lam


def cheby_precond(Amv, dinv, lmax, r, deg=6):                          # solvers.py:289-306
    """Chebyshev-Jacobi polynomial z = M(r) over [lmax/30, lmax], degree 6."""
    lo, hi = lmax / 30.0, lmax
    th, de = 0.5 * (hi + lo), 0.5 * (hi - lo)
    sg = th / de
    rh = 1.0 / sg
    res = dinv * r
    d = res / th
    x = np.zeros_like(r)
    for _ in range(deg):
        x = x + d
        res = res - dinv * Amv(d)
        rn = 1.0 / (2 * sg - rh)
        d = rn * rh * d + 2 * rn / de * res
        rh = rn
    return x + d


def bc_matrix(A, free):                                                # linalg.py:213-217
    D = sp.diags(np.asarray(free, float))
    return (D @ A @ D + sp.diags(1.0 - np.asarray(free, float))).tocsr()


class Direct:                                                          # linalg.py:199-210
    def __init__(self, A, permc_spec="COLAMD"):
        """``permc_spec``: SuperLU's column ordering (the reference's COLAMD by
        default; "MMD_AT_PLUS_A" factors large 3D stiffness matrices with far less
        fill, same solution to rounding)."""
        self.n = A.shape[0]
        try:
            self.lu = spla.splu(A.tocsc(), permc_spec=permc_spec)
            self._solve = self.lu.solve
        except RuntimeError:
            self._solve = spla.factorized(A.tocsc())

    def solve(self, b):
        return self._solve(np.asarray(b))
