"""Linear algebra of the hot path (drop-in for ``gfem.linalg``).

* ``pcg(A, b, M, x0, tol, maxiter) -> (x, k, relres)`` (gfem/linalg.py:21-47).
  With ``A`` a :class:`NativeSolver` the whole loop runs in the library (device
  scalars, graph-captured iteration chunks); with plain callables it runs the
  same recurrence over torch device vectors.
* ``rigid_body_modes`` (linalg.py:80-98), ``bc_matrix`` (213-217), ``Direct``
  (199-210, SuperLU on the host, a reference solver for parity), ``csr_to_device``
  / ``csr_mv`` (51-77).
* ``AMG(A, X, max_coarse=300, degree=2, presmooth=1, rot_mask=None)``
  (linalg.py:102-195).  The hierarchy is set up once on the host, as in the
  reference, then copied to HBM (FP64 and FP32 values) and applied by the
  library's device V-cycle.  The reference calls PyAMG's
  ``smoothed_aggregation_solver`` with a BSR matrix, rigid-body near-null space,
  symmetric strength with theta = 0, standard aggregation, Jacobi prolongation
  smoothing with omega = 4/3 and local (Gershgorin row-sum) weighting, and
  ``max_coarse = 300``.  PyAMG is not available here, so this module contains a
  project-written smoothed-aggregation set-up with those same choices (Vanek,
  Mandel & Brezina 1996): nodal-block strength graph, 3-pass standard
  aggregation (native, ``exfem_host_standard_aggregation``), tentative
  prolongator by per-aggregate orthonormalisation of the near-null space,
  one Jacobi smoothing step, Galerkin coarse operators R A P with R = P^T.  The
  reference's own per-level data follow unchanged: inverse diagonal, spectral
  bound by 15 power iterations from a seed-0 Gaussian vector times 1.1, and a
  dense Cholesky coarse solve with 1e-13 regularisation.
"""
import ctypes as C
import time

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

from . import _lib
from ._lib import check, lib, ptr, stream_ptr


# ------------------------------------------------------------------ PCG
def pcg(A, b, M=None, x0=None, tol=1e-8, maxiter=2000):
    """Preconditioned CG (gfem/linalg.py:21-47).  ``A`` may be a NativeSolver."""
    if isinstance(A, NativeSolver):
        return A.pcg(b, tol=tol, maxiter=maxiter)
    M = M or (lambda r: r)
    x = torch.zeros_like(b) if x0 is None else x0.clone()
    r = b - A(x)
    z = M(r)
    p = z.clone()
    rz = torch.dot(r, z)
    bn2 = torch.clamp(torch.dot(b, b), min=1e-300)
    tol2 = tol * tol * bn2
    rr = torch.dot(r, r)
    k = 0
    while bool(rr > tol2) and k < maxiter:
        Ap = A(p)
        alpha = rz / torch.dot(p, Ap)
        x = x + alpha * p
        r = r - alpha * Ap
        rr = torch.dot(r, r)
        z = M(r)
        rz_new = torch.dot(r, z)
        p = z + (rz_new / rz) * p
        rz = rz_new
        k += 1
    return x, k, torch.sqrt(rr / bn2)


# ------------------------------------------------------------------ CSR helpers
def csr_to_device(A, ell_max_ratio=2.0):
    """Device CSR (torch sparse) of a host matrix; the ELL/CSR choice of the
    reference (linalg.py:51-70) is a JAX gather strategy and has no effect here."""
    A = A.tocsr()
    A.sort_indices()
    t = torch.sparse_csr_tensor(torch.as_tensor(A.indptr, dtype=torch.int64), torch.as_tensor(A.indices, dtype=torch.int64),
                                torch.as_tensor(A.data), size=A.shape, device="cuda")
    return dict(csr=t, n=A.shape[0])


def csr_mv(M, x, n=None):
    return (M["csr"] @ x.reshape(-1, 1)).reshape(-1)


def rigid_body_modes(X, rot_mask=None):                                # linalg.py:80-98
    X = np.asarray(X)
    n = len(X)
    t = np.ones(n) if rot_mask is None else (~np.asarray(rot_mask)).astype(float)
    c = (X - X[t > 0].mean(0)) * t[:, None]
    B = np.zeros((3 * n, 6))
    for i in range(3):
        B[i::3, i] = t
    x, y, z = c[:, 0], c[:, 1], c[:, 2]
    B[0::3, 3], B[1::3, 3] = -y, x
    B[1::3, 4], B[2::3, 4] = -z, y
    B[0::3, 5], B[2::3, 5] = z, -x
    return B


def bc_matrix(A, free):                                                # linalg.py:213-217
    D = sp.diags(np.asarray(free, float))
    return (D @ A @ D + sp.diags(1.0 - np.asarray(free, float))).tocsr()


class Direct:                                                          # linalg.py:199-210
    """Host sparse direct solve (SuperLU); a parity reference, not the hot path."""

    def __init__(self, A):
        self.n = A.shape[0]
        try:
            self.lu = spla.splu(A.tocsc(), permc_spec="COLAMD")
            self._solve = self.lu.solve
        except RuntimeError:
            self._solve = spla.factorized(A.tocsc())

    def solve(self, b):
        return self._solve(np.asarray(b))


def ops_assemble(ops, ndof):
    """Host CSR of element operators [(dofs, Ke)] (gfem/model.py:176-192)."""
    rows, cols, vals = [], [], []
    for d, K in ops:
        d = np.asarray(d.cpu() if isinstance(d, torch.Tensor) else d, dtype=np.int64)
        K = np.asarray(K.detach().cpu().double() if isinstance(K, torch.Tensor) else K)
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


# ------------------------------------------------------------------ smoothed aggregation (host set-up)
def _strength_graph(A, bs):
    """Nodal strength graph of A with bs x bs blocks; theta = 0 keeps every block
    with a nonzero entry (explicit zeros removed first)."""
    A = A.tocoo()
    keep = A.data != 0
    r, c = A.row[keep] // bs, A.col[keep] // bs
    nb = A.shape[0] // bs
    S = sp.csr_matrix((np.ones(len(r)), (r, c)), shape=(nb, nb))
    S.sum_duplicates()
    S.sort_indices()
    return S


def _aggregate(S):
    n = S.shape[0]
    ptr_ = np.ascontiguousarray(S.indptr.astype(np.int64))
    idx = np.ascontiguousarray(S.indices.astype(np.int32))
    agg = np.empty(n, np.int32)
    nagg = C.c_int64()
    check(lib.exfem_host_standard_aggregation(n, ptr_.ctypes.data, idx.ctypes.data, agg.ctypes.data, C.byref(nagg)))
    return agg, int(nagg.value)


def _fit_candidates(agg, nagg, B, bs, drop=1e-10):
    """Tentative prolongator T (n x nagg*K) and coarse near-null space Bc (nagg*K x K):
    per aggregate, modified Gram-Schmidt of the near-null-space rows of its DOFs;
    columns that vanish (relative norm < drop) are zeroed."""
    n, K = B.shape
    node = np.arange(n) // bs
    a_of = agg[node]
    member = a_of >= 0
    dofs = np.nonzero(member)[0]
    order = np.argsort(a_of[dofs], kind="stable")
    dofs = dofs[order]
    a_sorted = a_of[dofs]
    counts = np.bincount(a_sorted, minlength=nagg)
    starts = np.concatenate([[0], np.cumsum(counts)[:-1]])
    Bc = np.zeros((nagg * K, K))
    Ti, Tj, Tv = [], [], []
    for m in np.unique(counts[counts > 0]):
        aggs = np.nonzero(counts == m)[0]
        rows = dofs[starts[aggs][:, None] + np.arange(m)[None, :]]          # (g, m)
        Q = B[rows].copy()                                                  # (g, m, K)
        R = np.zeros((len(aggs), K, K))
        n0 = np.linalg.norm(Q, axis=1) + 1e-300                             # (g, K)
        for j in range(K):
            for i in range(j):
                rij = np.einsum("gm,gm->g", Q[:, :, i], Q[:, :, j])
                R[:, i, j] = rij
                Q[:, :, j] -= rij[:, None] * Q[:, :, i]
            nj = np.linalg.norm(Q[:, :, j], axis=1)
            ok = nj > drop * n0[:, j]
            R[:, j, j] = np.where(ok, nj, 0.0)
            Q[:, :, j] = np.where(ok[:, None], Q[:, :, j] / np.where(ok, nj, 1.0)[:, None], 0.0)
        for g, a in enumerate(aggs):
            Bc[a * K:(a + 1) * K] = R[g]
        Ti.append(np.repeat(rows, K, axis=1).ravel())
        Tj.append((aggs[:, None, None] * K + np.arange(K)[None, None, :]).repeat(m, axis=1).reshape(len(aggs), -1).ravel())
        Tv.append(Q.reshape(len(aggs), -1).ravel())
    T = sp.csr_matrix((np.concatenate(Tv), (np.concatenate(Ti), np.concatenate(Tj))), shape=(n, nagg * K))
    T.eliminate_zeros()
    return T, Bc


def sa_hierarchy(A, B, bs=3, max_coarse=300, max_levels=10, omega=4.0 / 3.0):
    """Smoothed-aggregation hierarchy: list of (A, P) and the coarsest matrix."""
    A = A.tocsr()
    A.eliminate_zeros()
    levels = []
    while A.shape[0] > max_coarse and len(levels) < max_levels - 1:
        S = _strength_graph(A, bs)
        agg, nagg = _aggregate(S)
        if nagg == 0:
            break
        T, Bc = _fit_candidates(agg, nagg, B, bs)
        D = np.asarray(abs(A).sum(axis=1)).ravel()
        Dinv = np.where(D != 0, 1.0 / np.where(D != 0, D, 1.0), 0.0)
        P = (T - omega * (sp.diags(Dinv) @ (A @ T))).tocsr()
        P.eliminate_zeros()
        R = P.T.tocsr()
        Ac = (R @ A @ P).tocsr()
        Ac.eliminate_zeros()
        levels.append((A, P))
        if Ac.shape[0] >= A.shape[0]:
            A = Ac
            break
        A, B, bs = Ac, Bc, B.shape[1]
    return levels, A


def _rho(A, dinv, it=15):                                              # linalg.py:138-146
    x = np.random.default_rng(0).standard_normal(A.shape[0])
    lam = 1.0
    for _ in range(it):
        y = dinv * (A @ x)
        lam = np.linalg.norm(y) / max(np.linalg.norm(x), 1e-300)
        x = y / max(np.linalg.norm(y), 1e-300)
    return 1.1 * lam


def _csr_parts(M):
    M = M.tocsr()
    M.sort_indices()
    return (np.ascontiguousarray(M.indptr.astype(np.int64)), np.ascontiguousarray(M.indices.astype(np.int32)),
            np.ascontiguousarray(M.data.astype(np.float64)))


def amg_setup(A, X=None, max_coarse=300, rot_mask=None):
    """Host part of :class:`AMG`: dict with ``levels`` (list of dicts A, P, R, dinv,
    rho, n, nc), ``coarse`` (regularised Cholesky factor of the coarsest matrix),
    ``coarse_inv`` (its dense inverse product) and ``nnz`` per level
    (gfem/linalg.py:102-146).
    Needs no GPU, so many independent set-ups can run in worker processes."""
    A = A.tocsr()
    n = A.shape[0]
    if X is not None and n == 3 * len(X):
        B, bs = rigid_body_modes(X, rot_mask), 3
    else:
        B, bs = np.ones((n, 1)), 1
    sa_levels, Ac = sa_hierarchy(A, B, bs, max_coarse)
    levels = []
    for Al, P in sa_levels:
        d = Al.diagonal()
        dinv = np.where(np.abs(d) > 0, 1.0 / np.where(d == 0, 1, d), 0.0)
        levels.append(dict(A=Al, P=P, R=P.T.tocsr(), dinv=dinv, rho=float(_rho(Al, dinv)),
                           n=Al.shape[0], nc=P.shape[1]))
    Acd = Ac.toarray()
    Acd = 0.5 * (Acd + Acd.T)
    try:
        Lc = np.linalg.cholesky(Acd + 1e-13 * np.abs(Acd).max() * np.eye(len(Acd)))
    except np.linalg.LinAlgError:
        w, V = np.linalg.eigh(Acd)
        Lc = np.linalg.cholesky(V @ np.diag(np.maximum(w, 1e-12 * w.max())) @ V.T)
    Linv = np.linalg.inv(Lc)
    nnz = [lv["A"].nnz for lv in levels] + [int(np.count_nonzero(Acd))]
    return dict(levels=levels, coarse=Lc, coarse_inv=np.ascontiguousarray(Linv.T @ Linv), nnz=nnz)


class AMG:
    """Smoothed-aggregation AMG: host set-up, device V-cycle (gfem/linalg.py:102-195)."""

    def __init__(self, A, X=None, max_coarse=300, degree=2, presmooth=1, rot_mask=None, setup=None):
        t0 = time.time()
        h = setup if setup is not None else amg_setup(A, X, max_coarse, rot_mask)
        self.levels, self.coarse, self.coarse_inv, nnz = h["levels"], h["coarse"], h["coarse_inv"], h["nnz"]
        self.degree, self.presmooth = degree, presmooth
        self.sizes = [lv["n"] for lv in self.levels] + [self.coarse_inv.shape[0]]
        self.complexity = float(sum(nnz) / max(nnz[0], 1))
        self.nlevels = len(self.sizes)
        self.setup_time = time.time() - t0
        self._upload()

    @classmethod
    def from_setup(cls, setup, degree=2, presmooth=1):
        """Upload a hierarchy made by :func:`amg_setup` (for instance in a worker
        process).  A level whose ``A`` is None stores no matrix: it is smoothed
        with the solver's level-0 operator (the matrix-free product)."""
        return cls(None, setup=setup, degree=degree, presmooth=presmooth)

    def _upload(self):
        _lib.require_cuda()
        h = C.c_void_p()
        check(lib.exfem_amg_create(C.byref(h)))
        self._h = h
        for lv in self.levels:
            Al = lv["A"] if lv["A"] is not None else sp.csr_matrix((lv["n"], lv["n"]))
            Ap, Ai, Av = _csr_parts(Al)
            Pp, Pi, Pv = _csr_parts(lv["P"])
            Rp, Ri, Rv = _csr_parts(lv["R"])
            dinv = np.ascontiguousarray(lv["dinv"], dtype=np.float64)
            check(lib.exfem_amg_add_level(h, lv["n"], lv["nc"], Ap.ctypes.data, Ai.ctypes.data, Av.ctypes.data,
                                          Pp.ctypes.data, Pi.ctypes.data, Pv.ctypes.data, Rp.ctypes.data,
                                          Ri.ctypes.data, Rv.ctypes.data, dinv.ctypes.data, lv["rho"]))
        check(lib.exfem_amg_set_coarse(h, self.coarse_inv.shape[0], self.coarse_inv.ctypes.data))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:
            lib.exfem_amg_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def info(self):
        return f"AMG levels={self.nlevels} sizes={self.sizes} op.complexity={self.complexity:.2f}"

    def params(self):
        return dict(handle=self._h)

    def vcycle(self, r, level0=None, dinv0=None):
        """z = M(r): one device V-cycle in r's precision (FP64 or FP32); ``level0``
        is an optional Block whose matrix-free tangent smooths level 0 with the
        inverse diagonal ``dinv0`` (gfem/solvers.py:311-314)."""
        r = r.contiguous()
        code = _lib.F64 if r.dtype == torch.float64 else _lib.F32
        z = torch.empty_like(r)
        check(lib.exfem_amg_vcycle(self._h, code, ptr(r), ptr(z), level0.handle if level0 is not None else None,
                                   ptr(dinv0.to(r.dtype).contiguous()) if dinv0 is not None else None, stream_ptr()))
        return z

    def make(self):
        """precond(params, r, A0=None, dinv0=None) as in gfem/linalg.py:156-195;
        ``A0`` may be a Block (matrix-free level 0) or None (stored level-0 matrix)."""
        def precond(p, r, A0=None, dinv0=None):
            if A0 is not None and not hasattr(A0, "handle"):
                raise NotImplementedError("level-0 override must be a Block (matrix-free tangent)")
            return self.vcycle(r, A0, dinv0)
        return precond


class DeviceAMG(AMG):
    """Smoothed-aggregation AMG set up on the GPU (no counterpart in the reference,
    whose set-up runs PyAMG on the host, gfem/linalg.py:103-136).

    ``block``: a :class:`model.Block` with its prescribed DOFs set
    (``Block.set_fixed``); ``Ke``: its FP64 element matrices (ne, 3 nnode, 3 nnode),
    e.g. ``block.stiffness(u, state)``.  The same set-up as :func:`amg_setup` (rigid
    body modes of the block's coordinates, standard aggregation on the theta = 0
    strength graph, Jacobi-smoothed prolongator, Galerkin coarse operators), with
    the assembly of A and every matrix product on the device; only the graph work
    (adjacency, aggregates, sparsity patterns, per-aggregate orthonormalisation)
    runs on the host.  For meshes whose assembled matrix is too large for the
    host set-up.  The mesh level keeps no stored matrix unless ``keep_level0``:
    the solvers smooth it with the block's matrix-free product."""

    def __init__(self, block, Ke, max_coarse=300, degree=2, presmooth=1, keep_level0=False):
        """``block``, ``Ke``: one block and its element matrices, or lists of the
        blocks of a model over one node set and their element matrices (A_0 is then
        the sum over the blocks, with the first block's prescribed DOFs)."""
        t0 = time.time()
        _lib.require_cuda()
        h = C.c_void_p()
        check(lib.exfem_amg_create(C.byref(h)))
        self._h = h
        blocks = list(block) if isinstance(block, (list, tuple)) else [block]
        Kes = list(Ke) if isinstance(Ke, (list, tuple)) else [Ke]
        if len(blocks) != len(Kes):
            raise ValueError(f"{len(blocks)} blocks but {len(Kes)} element-matrix arrays")
        Kes = [K.to(torch.float64).contiguous() for K in Kes]
        hb = (C.c_void_p * len(blocks))(*[b.handle.value for b in blocks])
        hk = (C.c_void_p * len(Kes))(*[K.data_ptr() for K in Kes])
        check(lib.exfem_amg_setup_blocks(h, len(blocks), hb, hk, int(max_coarse), 1 if keep_level0 else 0,
                                         stream_ptr()))
        cap = 16
        nl, rows, nnz = C.c_int(), (C.c_int64 * cap)(), (C.c_int64 * cap)()
        check(lib.exfem_amg_info(h, cap, C.byref(nl), rows, nnz))
        self.sizes = [int(rows[i]) for i in range(min(nl.value, cap))]
        self.nnz = [int(nnz[i]) for i in range(min(nl.value, cap))]
        self.levels, self.coarse, self.coarse_inv = None, None, None
        self.degree, self.presmooth = degree, presmooth
        self.complexity = float(sum(self.nnz) / max(self.nnz[0], 1))
        self.nlevels = nl.value
        self.keep_level0 = keep_level0
        self.setup_time = time.time() - t0

    def _export(self, level, what):
        rows, cols, nnz, rho = C.c_int64(), C.c_int64(), C.c_int64(), C.c_double()
        check(lib.exfem_amg_export_level(self._h, level, what, C.byref(rows), C.byref(cols), C.byref(nnz), None, None,
                                         None, C.byref(rho)))
        if what == 3:
            v = np.zeros(rows.value)
            check(lib.exfem_amg_export_level(self._h, level, 3, C.byref(rows), C.byref(cols), C.byref(nnz), None,
                                             None, v.ctypes.data, None))
            return v, rho.value
        ptr_ = np.zeros(rows.value + 1, np.int64)
        idx = np.zeros(max(nnz.value, 1), np.int32)
        val = np.zeros(max(nnz.value, 1))
        check(lib.exfem_amg_export_level(self._h, level, what, C.byref(rows), C.byref(cols), C.byref(nnz),
                                         ptr_.ctypes.data, idx.ctypes.data, val.ctypes.data, None))
        return sp.csr_matrix((val[:nnz.value], idx[:nnz.value], ptr_), shape=(rows.value, cols.value)), rho.value

    def to_setup(self):
        """The hierarchy as the dict :func:`amg_setup` returns (levels with A — None
        where no matrix is stored —, P, R, dinv, rho, n, nc; coarse_inv), e.g. to
        merge it into a batched union (``batch.union_hierarchy``)."""
        levels = []
        for l in range(len(self.sizes) - 1):
            A, _ = self._export(l, 0)
            P, _ = self._export(l, 1)
            R, _ = self._export(l, 2)
            dinv, rho = self._export(l, 3)
            levels.append(dict(A=A if A.nnz else None, P=P, R=R, dinv=dinv, rho=rho, n=P.shape[0], nc=P.shape[1]))
        nc = C.c_int64()
        check(lib.exfem_amg_export_coarse(self._h, C.byref(nc), None))
        Ainv = np.zeros((nc.value, nc.value))
        check(lib.exfem_amg_export_coarse(self._h, C.byref(nc), Ainv.ctypes.data))
        return dict(levels=levels, coarse=None, coarse_inv=Ainv, nnz=list(self.nnz))


# ------------------------------------------------------------------ native solver
class NativeSolver:
    """PCG / mixed-precision refinement in the library for one block, or for the
    blocks of a model (a list over one node set: every operator is the sum over the
    blocks, gfem/model.py:466-486, with the first block's prescribed DOFs).

    op: "ebe64" (stored Ke, FP64), "csr64" (the stored Ke assembled on the device
    into one FP64 CSR matrix, gfem/model.py:195-238), "mf64" (matrix-free FP64),
    "mf32" (matrix-free FP32); pc: "none", "jacobi", "amg", "cheby" (Chebyshev-Jacobi
    polynomial, gfem/solvers.py:289-306).  The stored-Ke operators
    take their element matrices from :meth:`set_ke` (one array per block)."""

    OPS = {"ebe64": _lib.OP_EBE_F64, "mf64": _lib.OP_MF_F64, "mf32": _lib.OP_MF_F32, "csr64": _lib.OP_CSR_F64}
    PCS = {"none": _lib.PC_NONE, "jacobi": _lib.PC_JACOBI, "amg": _lib.PC_AMG, "cheby": _lib.PC_CHEBY}

    def __init__(self, block, op="mf32", pc="amg", amg=None, graph=True, chunk=8, mixed_mode="reliable",
                 mixed_delta=0.1, device_loop=True):
        """mixed_mode: how :meth:`mixed` runs its FP32 work — "reliable" (one FP32
        recursion whose residual is replaced by the FP64 one after each reduction by
        mixed_delta) or "restart" (the reference's restarted refinement,
        gfem/solvers.py:344-384).  device_loop (with graph): the PCG loop runs to its
        stopping test inside one graph launch (conditional while node); False
        launches graphs of `chunk` iterations from the host."""
        self.blocks = list(block) if isinstance(block, (list, tuple)) else [block]
        self.block, self.amg = self.blocks[0], amg
        self.op, self.pc = op, pc
        h = C.c_void_p()
        check(lib.exfem_solver_create(self.block.handle, self.OPS[op], self.PCS[pc],
                                      amg.handle if amg is not None else None, C.byref(h)))
        self._h = h
        for b in self.blocks[1:]:
            check(lib.exfem_solver_add_block(h, b.handle))
        check(lib.exfem_solver_set_graph(h, 1 if graph else 0, chunk))
        check(lib.exfem_solver_set_loop(h, 1 if device_loop else 0))
        check(lib.exfem_solver_set_mixed_mode(h, {"reliable": 1, "restart": 0}[mixed_mode], float(mixed_delta)))
        self._Ke = None
        self.last_iters = 0
        self.last_passes = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:
            lib.exfem_solver_destroy(h)
            self._h = None

    def set_ke(self, Ke):
        """Element matrices of the block (a tensor) or of every block (a list)."""
        Kes = list(Ke) if isinstance(Ke, (list, tuple)) else [Ke]
        if len(Kes) != len(self.blocks):
            raise ValueError(f"{len(self.blocks)} blocks but {len(Kes)} element-matrix arrays")
        self._Ke = [K.contiguous() for K in Kes]
        for i, K in enumerate(self._Ke):
            check(lib.exfem_solver_set_ke_block(self._h, i, ptr(K)))

    def cheby_bound(self):
        """The Chebyshev-Jacobi preconditioner's bound on the spectrum of D^-1 A."""
        v = C.c_double()
        check(lib.exfem_solver_cheby_bound(self._h, C.byref(v)))
        return v.value

    def pcg(self, b, tol=1e-8, maxiter=2000):
        b = b.to(torch.float64).contiguous()
        x = torch.empty_like(b)
        k, rr = C.c_int(), C.c_double()
        check(lib.exfem_solver_pcg(self._h, ptr(b), ptr(x), float(tol), int(maxiter), C.byref(k), C.byref(rr),
                                   stream_ptr()))
        self.last_iters = k.value
        return x, k.value, rr.value

    def newton_increment(self, u, states, fext, start, qref, rtol, max_iter, line_search, cg_tol, cg_maxiter):
        """One Newton increment (predictor and corrections, gfem/solvers.py:607-683)
        as one graph launch on this solver (FP32 matrix-free operator, AMG, reliable
        updates; one or several blocks).  states: per block its J2 state tensor or
        None (elastic).  Returns (converged, corrections, u, states, qref, ratios)."""
        if len(states) != len(self.blocks):
            raise ValueError(f"one state entry per block: got {len(states)} for {len(self.blocks)} blocks")
        for b, st in zip(self.blocks, states):
            want = b.ne * b.etype.ngp * b.material.nstate
            if b.material.nstate > 1 and (st is None or st.numel() != want or st.dtype != torch.float64):
                raise ValueError(f"block {b.name}: J2 states need {want} FP64 values (ne, ngp, nstate)")
        u = u.to(torch.float64).contiguous()
        fext = fext.to(torch.float64).contiguous()
        start = start.to(torch.float64).contiguous()
        s_old = [s.contiguous() if s is not None else None for s in states]
        s_out = [torch.empty_like(s) if s is not None else None for s in s_old]
        arr_old = (C.c_void_p * max(len(s_old), 1))(*[ptr(s) for s in s_old])
        arr_out = (C.c_void_p * max(len(s_out), 1))(*[ptr(s) for s in s_out])
        u_out = torch.empty_like(u)
        q = C.c_double(float(qref))
        k, ok = C.c_int(), C.c_int()
        ratios = np.zeros(max(int(max_iter), 1))
        lin = np.zeros(2, np.int32)
        check(lib.exfem_newton_increment(self._h, ptr(u), arr_old, ptr(fext), ptr(start), float(rtol), int(max_iter),
                                         1 if line_search else 0, float(cg_tol), int(cg_maxiter), C.byref(q),
                                         ptr(u_out), arr_out, C.byref(k), C.byref(ok), ratios.ctypes.data,
                                         lin.ctypes.data, stream_ptr()))
        self.last_iters, self.last_passes = int(lin[0]), int(lin[1])
        n_it = k.value + 1 if ok.value else int(max_iter)
        return bool(ok.value), k.value, u_out, s_out, q.value, ratios[:n_it]

    def mixed(self, b, tol=1e-8, inner_tol=2e-5, max_pass=12, maxiter=20000):
        b = b.to(torch.float64).contiguous()
        x = torch.empty_like(b)
        k, p, rr = C.c_int(), C.c_int(), C.c_double()
        check(lib.exfem_solver_mixed(self._h, ptr(b), ptr(x), float(tol), float(inner_tol), int(max_pass),
                                     int(maxiter), C.byref(k), C.byref(p), C.byref(rr), stream_ptr()))
        self.last_iters, self.last_passes = k.value, p.value
        return x, k.value, p.value, rr.value
