"""Batched solves: many independent linear-elastic problems of uneven sizes, with
several right-hand sides each, solved together in one set of launches.

The reference solves one ``Model`` at a time; its multi-right-hand-side entry point
``optimize.multi_load_cases(model, step, F, cg_tol)`` (gfem/optimize.py:116-143)
runs a vmapped Jacobi-PCG over the rows of F for one mesh, every lane until the
slowest converges.  Here a batch spans meshes as well as load cases:

* every (problem, right-hand side) pair is an *instance*; the instances' meshes
  are concatenated into one union element block (per-element Lame parameters,
  one prescribed-DOF mask), so one launch of the matrix-free product covers all
  of them (``exfem_batch_create``);
* each problem's smoothed-aggregation hierarchy is set up once on the host, as
  for a single solve (``linalg.amg_setup``, in worker processes), and the
  hierarchies are merged level by level into one block-diagonal hierarchy.
  Problems with fewer levels are relayed by identity levels whose smoother is
  switched off, so each instance sees exactly its own V-cycle; the right-hand
  sides of one problem share its stored matrices (``exfem_amg_replicate``);
* ``exfem_batch_solve`` runs FP32 matrix-free AMG-PCG per instance inside FP64
  iterative refinement, each instance with its own scalars, reductions (one
  thread block per instance, fixed order) and stopping test
  ||b_i - A x_i|| <= tol ||b_i||; converged instances are frozen while the
  others continue.
"""
import ctypes as C
import multiprocessing as mp
import os
import time
from concurrent.futures import ProcessPoolExecutor

import numpy as np
import scipy.sparse as sp
import torch

from . import _lib, linalg
from ._lib import check, lib, ptr, stream_ptr
from .materials import LinearElastic, lame
from .model import Block


class Problem:
    """One mesh with its linear-elastic material, prescribed DOFs and loads.

    X (nn, 3) coordinates, conn (ne, nnode) connectivity, etype HEX8 or TET10,
    material :class:`LinearElastic`, fixed (3 nn,) bool mask of prescribed DOFs
    (prescribed value zero), rhs (nrhs, 3 nn) nodal forces."""

    def __init__(self, X, conn, etype, material, fixed, rhs):
        if not isinstance(material, LinearElastic):
            raise TypeError("batched solves cover linear-elastic materials")
        self.X = np.ascontiguousarray(np.asarray(X, dtype=np.float64))
        self.conn = np.ascontiguousarray(np.asarray(conn, dtype=np.int32))
        self.etype, self.material = etype, material
        self.ndof = 3 * len(self.X)
        self.fixed = np.asarray(fixed, dtype=bool).reshape(-1)
        rhs = np.asarray(rhs, dtype=np.float64)
        self.rhs = rhs.reshape(-1, self.ndof)
        if self.fixed.size != self.ndof:
            raise ValueError("fixed mask must hold 3 entries per node")


def _setup_worker(args):
    """Host AMG set-up of one problem from its element stiffness matrices (runs in
    a worker process; needs no GPU)."""
    dofs, Ke, ndof, free, X, max_coarse = args
    A = linalg.bc_matrix(linalg.ops_assemble([(dofs, Ke)], ndof), free)
    h = linalg.amg_setup(A, X, max_coarse)
    if h["levels"]:
        h["levels"][0]["A"] = None       # level 0 is smoothed with the matrix-free product
    return h


def _element_stiffness(p):
    blk = Block(p.conn, p.etype, p.material, X=p.X)
    Ke = blk.stiffness(torch.zeros(p.ndof, dtype=torch.float64, device="cuda"), blk.init_state())
    dofs = (p.conn.astype(np.int64)[:, :, None] * 3 + np.arange(3)).reshape(len(p.conn), -1)
    return dofs, Ke.cpu().numpy()


def device_setups(problems, max_coarse=300):
    """Per-problem hierarchies set up on the device (linalg.DeviceAMG, the host
    set-up's algorithm with the assembly and the products on the GPU), copied to the
    host in the form :func:`host_setups` returns, one problem after the other."""
    out = []
    for p in problems:
        blk = Block(p.conn, p.etype, p.material, X=p.X)
        blk.set_fixed(p.fixed)
        Ke = blk.stiffness(torch.zeros(p.ndof, dtype=torch.float64, device="cuda"), blk.init_state())
        amg = linalg.DeviceAMG(blk, Ke, max_coarse)
        out.append(amg.to_setup())
        del amg, Ke, blk
    return out


def host_setups(problems, max_coarse=300, workers=None, stiffness=None):
    """Per-problem host hierarchies.  Element stiffness matrices (``stiffness``, a
    list of (dofs, Ke) per problem) come from the GPU unless given; assembly and
    smoothed aggregation run in ``workers`` spawned processes (None: one per host
    core, up to 16; 0: in this process)."""
    if workers is None:
        workers = min(16, os.cpu_count() or 1)
    jobs = []
    for i, p in enumerate(problems):
        dofs, Ke = stiffness[i] if stiffness is not None else _element_stiffness(p)
        jobs.append((dofs, Ke, p.ndof, (~p.fixed).astype(np.float64), p.X, max_coarse))
    if workers <= 1 or len(jobs) == 1:
        return [_setup_worker(j) for j in jobs]
    with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_setup_worker, jobs, chunksize=max(1, len(jobs) // (4 * workers))))


def _canonical(M):
    """M as CSR with sorted, summed entries (a copy where M is not, so that the
    caller's matrix is left as it was)."""
    M = M.tocsr()
    if not M.has_canonical_format:
        M = M.copy()
        M.sum_duplicates()
    return M


def _block_diag_csr(blocks):
    """Block-diagonal CSR arrays (indptr int64, indices int32, data float64) of
    ``blocks`` (sparse matrices or ``(rows, cols)`` for an all-zero block), written
    by shifting each block's CSR arrays: the rows of a block-diagonal matrix are its
    blocks' rows with the column indices moved by the block's column offset."""
    ncols = sum(b[1] if isinstance(b, tuple) else b.shape[1] for b in blocks)
    if ncols >= 2 ** 31:
        raise ValueError(f"union level of {ncols} columns exceeds 32-bit column indices")
    ptrs, idx, val = [np.zeros(1, np.int64)], [], []
    nnz = col0 = 0
    for b in blocks:
        if isinstance(b, tuple):
            ptrs.append(np.full(b[0], nnz, np.int64))
            col0 += b[1]
            continue
        b = _canonical(b)
        ptrs.append(b.indptr[1:].astype(np.int64) + nnz)
        idx.append(b.indices.astype(np.int32, copy=False) + np.int32(col0))
        val.append(b.data.astype(np.float64, copy=False))
        nnz += b.nnz
        col0 += b.shape[1]
    indices = np.concatenate(idx) if idx else np.zeros(0, np.int32)
    data = np.concatenate(val) if val else np.zeros(0, np.float64)
    return np.concatenate(ptrs), indices, data


def union_hierarchy(setups):
    """Block-diagonal union of per-problem hierarchies, uploaded to a new library
    AMG handle.  Returns (handle, level_offsets (levels+1, nprob+1), sizes)."""
    nprob = len(setups)
    L = max(len(h["levels"]) for h in setups)
    coarse_n = [h["coarse_inv"].shape[0] for h in setups]
    h_amg = C.c_void_p()
    check(lib.exfem_amg_create(C.byref(h_amg)))
    offsets = []
    for l in range(L):
        As, Ps, dinv, rho = [], [], [], []
        for h, nc in zip(setups, coarse_n):
            lv = h["levels"][l] if l < len(h["levels"]) else None
            if lv is None:                                   # relay level of a shallower hierarchy
                I = sp.identity(nc, format="csr")
                As.append(I if l else None)
                Ps.append(I)
                dinv.append(np.ones(nc))
                rho.append(np.zeros(nc))
            else:
                As.append(lv["A"] if l else None)
                Ps.append(lv["P"])
                dinv.append(lv["dinv"])
                rho.append(np.full(lv["n"], lv["rho"]))
        sizes = [P.shape[0] for P in Ps]
        offsets.append(np.concatenate([[0], np.cumsum(sizes)]))
        n, nc = int(sum(sizes)), int(sum(P.shape[1] for P in Ps))
        # no stored level-0 matrix: level 0 is smoothed with the matrix-free product
        Ap, Ai, Av = _block_diag_csr([(P.shape[0], P.shape[0]) for P in Ps] if l == 0 else As)
        Pp, Pi, Pv = _block_diag_csr(Ps)
        Rp, Ri, Rv = _block_diag_csr([P.T for P in Ps])
        d = np.ascontiguousarray(np.concatenate(dinv))
        r = np.ascontiguousarray(np.concatenate(rho))
        check(lib.exfem_amg_add_level(h_amg, n, nc, Ap.ctypes.data, Ai.ctypes.data, Av.ctypes.data, Pp.ctypes.data,
                                      Pi.ctypes.data, Pv.ctypes.data, Rp.ctypes.data, Ri.ctypes.data, Rv.ctypes.data,
                                      d.ctypes.data, float(max(r.max(), 1.0))))
        check(lib.exfem_amg_set_level_rows(h_amg, l, r.ctypes.data))
    coff = np.concatenate([[0], np.cumsum(coarse_n)]).astype(np.int64)
    offsets.append(coff)
    blocks = np.ascontiguousarray(np.concatenate([h["coarse_inv"].ravel() for h in setups]))
    check(lib.exfem_amg_set_coarse_blocks(h_amg, nprob, coff.ctypes.data, blocks.ctypes.data))
    return h_amg, np.ascontiguousarray(np.stack(offsets).astype(np.int64))


class BatchSolver:
    """Solver for a fixed set of problems; ``solve()`` returns every instance's
    displacement.  Instances are ordered problem by problem, right-hand side by
    right-hand side."""

    def __init__(self, problems, max_coarse=300, workers=None, setups=None, amg_setup="device"):
        """amg_setup: "device" (per-problem hierarchies set up on the GPU, the
        default) or "host" (assembled CSR and host set-up in ``workers`` processes)."""
        _lib.require_cuda()
        t0 = time.time()
        self.problems = list(problems)
        if not self.problems:
            raise ValueError("empty batch")
        et = {p.etype.name for p in self.problems}
        if len(et) != 1:
            raise ValueError(f"one element type per batch, got {sorted(et)}")
        self.etype = self.problems[0].etype
        if setups is not None:
            self.setups = setups
        elif amg_setup == "device":
            self.setups = device_setups(self.problems, max_coarse)
        elif amg_setup == "host":
            self.setups = host_setups(self.problems, max_coarse, workers)
        else:
            raise ValueError(f"unknown AMG set-up {amg_setup!r}")
        self.t_host = time.time() - t0
        # instances: one per (problem, right-hand side)
        self.inst = [(k, r) for k, p in enumerate(self.problems) for r in range(len(p.rhs))]
        self.ninst = len(self.inst)
        Xs, cs, lams, mus, fixed = [], [], [], [], []
        node0 = 0
        for k, r in self.inst:
            p = self.problems[k]
            Xs.append(p.X)
            cs.append(p.conn + node0)
            mu, lam = lame(p.material.E, p.material.nu)
            lams.append(np.full(len(p.conn), lam))
            mus.append(np.full(len(p.conn), mu))
            fixed.append(p.fixed)
            node0 += len(p.X)
        self.block = Block(np.concatenate(cs), self.etype, self.problems[0].material, X=np.concatenate(Xs))
        self.block.set_lame(np.concatenate(lams), np.concatenate(mus))
        self.fixed = np.concatenate(fixed)
        self.block.set_fixed(self.fixed)
        self.ndof = 3 * node0
        self.dof_off = np.concatenate([[0], np.cumsum([self.problems[k].ndof for k, _ in self.inst])]).astype(np.int64)
        self._amg, lev_off = union_hierarchy(self.setups)
        inst_blk = np.array([k for k, _ in self.inst], np.int32)
        check(lib.exfem_amg_replicate(self._amg, len(self.problems), lev_off.ctypes.data, self.ninst,
                                      inst_blk.ctypes.data))
        h = C.c_void_p()
        check(lib.exfem_batch_create(self.block.handle, self._amg, self.ninst, self.dof_off.ctypes.data, C.byref(h)))
        self._h = h
        self.nlevels = lev_off.shape[0]
        self.rhs = self.union_rhs()
        self.t_setup = time.time() - t0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib.exfem_batch_destroy(h)
            self._h = None
        a = getattr(self, "_amg", None)
        if a is not None and a.value:
            lib.exfem_amg_destroy(a)
            self._amg = None

    def union_rhs(self, pin=False):
        """The instances' right-hand sides as one FP64 vector (host; pinned on request)."""
        b = np.concatenate([self.problems[k].rhs[r] for k, r in self.inst])
        t = torch.from_numpy(b)
        return t.pin_memory() if pin else t

    def split(self, x):
        """Per-instance views of a union vector."""
        return [x[self.dof_off[i]:self.dof_off[i + 1]] for i in range(self.ninst)]

    def solve(self, b=None, tol=1e-8, inner_tol=2e-5, max_pass=12, maxiter=20000):
        """x (union FP64 on the device) and info (per-instance iterations and
        relative residuals, refinement passes, status)."""
        if b is None:
            b = self.rhs
        b = b.to(device="cuda", dtype=torch.float64, non_blocking=True).contiguous()
        x = torch.empty_like(b)
        iters = np.zeros(self.ninst, np.int32)
        rel = np.zeros(self.ninst, np.float64)
        passes = C.c_int()
        st = lib.exfem_batch_solve(self._h, ptr(b), ptr(x), tol, inner_tol, max_pass, maxiter, iters.ctypes.data,
                                   C.byref(passes), rel.ctypes.data, stream_ptr())
        if st < 0:
            check(st)
        return x, dict(iters=iters, relres=rel, passes=passes.value, converged=(st == 0))


def cantilever(nx, ny, nz, h, material, tip_forces, etype=None):
    """Problem: a box cantilever of nx*ny*nz hexahedra (or 6 C3D10 each) of size h,
    x=0 face clamped, each right-hand side a total tip force vector (3,) split
    evenly over the nodes of the x = nx*h face."""
    from . import elements, mesh
    etype = etype or elements.HEX8
    X, c = mesh.box_hex(nx * h, ny * h, nz * h, nx, ny, nz)
    if etype.name == "C3D10":
        X, c = mesh.tet4_to_tet10(*mesh.hex_to_tet4(X, c))
    L = nx * h
    fix = mesh.nodes_where(X, lambda x, y, z: x < 1e-9 * L)
    tip = mesh.nodes_where(X, lambda x, y, z: x > L * (1 - 1e-9))
    fixed = np.zeros(3 * len(X), bool)
    for d in range(3):
        fixed[3 * fix + d] = True
    F = np.asarray(tip_forces, dtype=np.float64).reshape(-1, 3)
    rhs = np.zeros((len(F), 3 * len(X)))
    for k, f in enumerate(F):
        for d in range(3):
            rhs[k, 3 * tip + d] = f[d] / len(tip)
    return Problem(X, c, etype, material, fixed, rhs)


def random_cantilevers(count, seed=0, nx=(4, 64), nyz=(2, 16), h=5.0, E=(70e3, 210e3), nu=(0.25, 0.35),
                       force=(100.0, 1000.0)):
    """Seeded batch of C3D8 steel/aluminium-like cantilevers (mm, N, MPa): element
    counts uniform integers nx in [4, 64], ny, nz in [2, 16], element size 5 mm,
    E uniform in [70, 210] GPa, nu uniform in [0.25, 0.35], four right-hand sides
    each, tip forces along +x, +y, -y, -z with magnitudes uniform in [100, 1000] N."""
    rng = np.random.default_rng(seed)
    dirs = np.array([[1.0, 0, 0], [0, 1.0, 0], [0, -1.0, 0], [0, 0, -1.0]])
    out = []
    for _ in range(count):
        n = (int(rng.integers(nx[0], nx[1] + 1)), int(rng.integers(nyz[0], nyz[1] + 1)),
             int(rng.integers(nyz[0], nyz[1] + 1)))
        mat = LinearElastic(rng.uniform(*E), rng.uniform(*nu))
        mags = rng.uniform(*force, size=len(dirs))
        out.append(cantilever(*n, h, mat, dirs * mags[:, None]))
    return out
