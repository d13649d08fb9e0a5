"""Modal and buckling analysis by block LOBPCG on the device operators (drop-in for
``gfem.eigen.lobpcg`` / ``modal_lobpcg`` / ``buckling_lobpcg``, gfem/eigen.py:32-151,
and the linear buckling procedure of gfem/solvers.py:1074-1110).

Buckling: K0 phi = -lambda KG phi through the smallest mu of KG phi = mu K0 phi
(A = the initial-stress stiffness KG of the stresses of the linear response to the
step's loads, element matrices from the library's geometric-stiffness kernel; B =
the stiffness K0 at u = 0; T = a device V-cycle of K0), lambda = -1/mu.

K phi = w^2 M phi for the smallest eigenvalues: A = the stiffness (prescribed DOFs
held at zero) from the stored FP64 element matrices, or the FP64 matrix-free product
column by column, B = the HRZ-lumped mass matrix (gfem/model.py:120-124, 501-510),
T = one smoothed-aggregation V-cycle of the stiffness (hierarchy set up on the
device).  Every T application is a call of the library per column; the stored-Ke
operators (the modal A, the buckling A and B) apply one multi-right-hand-side
product per 16 columns, so each Ke is read once per block step; the block
Rayleigh-Ritz steps are small dense products on
the device and a small symmetric eigenproblem on the host, as in the reference
(Knyazev's LOBPCG with SVQB orthonormalisation).
"""
import numpy as np
import torch

from . import linalg
from .solvers import State, _Setup

_A, _B = 0.5854101966249685, 0.1381966011250105


def _tables(etype):
    """Shape functions N (ngp, nnode), their parametric derivatives dN (ngp, nnode, 3)
    and weights (ngp,) of the element's rule (gfem/elements.py:113-125, 166-179)."""
    if etype.name == "C3D8":
        H = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                      [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], float)
        gp, gw = H / np.sqrt(3.0), np.ones(8)
        N, dN = [], []
        for x in gp:
            f = 1 + H * x[None, :]                                   # (8, 3) factors
            N.append(0.125 * f.prod(1))
            dN.append(0.125 * np.stack([H[:, 0] * f[:, 1] * f[:, 2], H[:, 1] * f[:, 0] * f[:, 2],
                                        H[:, 2] * f[:, 0] * f[:, 1]], 1))
        return np.array(N), np.array(dN), gw
    gp = np.array([[_B, _B, _B], [_A, _B, _B], [_B, _A, _B], [_B, _B, _A]])
    gw = np.full(4, 1.0 / 24.0)
    dL = np.array([[-1.0, -1.0, -1.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])
    edges = [(0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3)]
    N, dN = [], []
    for x in gp:
        L = np.array([1 - x.sum(), x[0], x[1], x[2]])
        n = list(L * (2 * L - 1))
        d = [(4 * L[i] - 1) * dL[i] for i in range(4)]
        for i, j in edges:
            n.append(4 * L[i] * L[j])
            d.append(4 * (dL[i] * L[j] + L[i] * dL[j]))
        N.append(n)
        dN.append(d)
    return np.array(N), np.array(dN), gw


def lumped_mass(model):
    """Diagonal HRZ-lumped mass (ndof,) on the device: per element d_a = sum_g vol_g
    N_a(g)^2 scaled to density x element volume (gfem/model.py:120-124), added at the
    nodes (501-510)."""
    return torch.as_tensor(lumped_mass_host(model.X, model.blocks), device="cuda")


def lumped_mass_host(X, blocks):
    """:func:`lumped_mass` of nodes X (nn, 3) and blocks (conn, etype, material) as a
    host array (set-up work, done once per analysis)."""
    X = np.asarray(X, dtype=np.float64)
    m = np.zeros(len(X))
    for b in blocks:
        N, dN, gw = _tables(b.etype)
        rho = float(getattr(b.material, "density", 1.0))
        conn = np.asarray(b.conn, dtype=np.int64)
        Xe = X[conn]                                                  # (ne, nnode, 3)
        J = np.einsum("ean,gai->egni", Xe, dN)
        vol = gw[None, :] * np.linalg.det(J)                          # (ne, ngp)
        d = np.einsum("eg,ga->ea", vol, N * N)
        d = d * (rho * vol.sum(1))[:, None] / d.sum(1)[:, None]
        np.add.at(m, conn, d)
    return np.repeat(m, 3)


def _svqb(B, S):
    BS = B(S)
    G = (S.T @ BS).cpu().numpy()
    G = 0.5 * (G + G.T)
    d = np.sqrt(np.maximum(np.diag(G), 1e-300))
    w, V = np.linalg.eigh(G / d[:, None] / d[None, :])
    return w, V, d


def lobpcg(A, B, T, X0, k, tol=1e-6, maxiter=500, log=None):
    """Smallest k eigenpairs of A x = lam B x (gfem/eigen.py:32-84).  A, B, T: maps
    of (n, m) device blocks; X0 (n, m >= k).  Returns (eigenvalues (k,) NumPy,
    eigenvectors (n, k) device, iterations)."""
    dev = X0.device

    def orth(S):
        w, V, d = _svqb(B, S)
        keep = w > 1e-12 * w.max()
        Vk = V[:, keep] / np.sqrt(w[keep])[None, :]
        return (S / torch.as_tensor(d, device=dev)[None, :]) @ torch.as_tensor(Vk, device=dev)

    def rr(S, m):
        AS = A(S)
        Ga = (S.T @ AS).cpu().numpy()
        lam, C = np.linalg.eigh(0.5 * (Ga + Ga.T))
        return lam[:m], torch.as_tensor(C[:, :m], device=dev), AS

    X = orth(X0)
    m = X.shape[1]
    lam, C, AS = rr(X, m)
    X, AX = X @ C, AS @ C
    BX = B(X)
    P = None
    it = 0
    for it in range(1, maxiter + 1):
        lt = torch.as_tensor(lam, device=dev)
        R = AX - BX * lt[None, :]
        rn = (torch.linalg.norm(R, dim=0) / torch.clamp(lt.abs() * torch.linalg.norm(BX, dim=0), min=1e-300))
        res = float(rn[:k].max())
        if log and it % 10 == 1:
            log(f"    LOBPCG it {it:4d}: max rel. residual {res:.2e}")
        if res < tol:
            break
        W = T(R)
        W = W - X @ (BX.T @ W)
        parts = [X, W] if P is None else [X, W, P - X @ (BX.T @ P)]
        S = orth(torch.cat(parts, 1))
        lam, C, AS = rr(S, m)
        Xn = S @ C
        P = Xn - X @ (BX.T @ Xn)
        X, AX = Xn, AS @ C
        BX = B(X)
    return np.asarray(lam[:k]), X[:, :k], it


def modal_lobpcg(model, step, nmodes, state=None, tol=1e-6, maxiter=500, log=None, operator="stored"):
    """(w^2 (nmodes,), modes (nmodes, ndof)) of a model under the step's prescribed
    DOFs (gfem/eigen.py:99-124; ``nmodes`` is the reference step's ``nmodes``); the
    stiffness of a model of several blocks is the sum over its blocks.  operator:
    "stored" (default) keeps the FP64 element matrices the hierarchy is set up from
    and applies them to up to 16 columns per product (the reference's block EbE
    operator, gfem/eigen.py:97-110), each Ke read once per block step; "mf" applies
    the FP64 matrix-free product column by column and keeps no element matrices
    (ne x nd^2 doubles less on the device, about 13% slower)."""
    if operator not in ("mf", "stored"):
        raise ValueError(f"unknown modal operator {operator!r}")
    setup = _Setup(model, step, state or State(model))
    free = setup.free
    for blk in model.blocks:
        blk.set_fixed(setup.fixed)
    nd = model.ndof
    zero = torch.zeros(nd, dtype=torch.float64, device="cuda")
    Kes = [blk.stiffness(zero, blk.init_state()) for blk in model.blocks]
    amg = linalg.DeviceAMG(model.blocks, Kes, keep_level0=True)
    stored = _ops_block(list(zip(model.blocks, Kes)), free) if operator == "stored" else None
    del Kes
    M = lumped_mass(model) * free

    def K(v):
        out = None
        for blk in model.blocks:
            y = blk.tangent_matvec(v)
            out = y if out is None else out + y
        return out

    def A(V):
        if stored is not None:
            return stored(V)
        return torch.stack([K(V[:, j].contiguous()) for j in range(V.shape[1])], 1) * free[:, None]

    def B(V):
        return M[:, None] * V

    def T(R):
        return torch.stack([amg.vcycle(R[:, j].contiguous()) for j in range(R.shape[1])], 1) * free[:, None]

    m = nmodes + max(4, nmodes // 2)
    g = torch.Generator(device="cuda").manual_seed(0)
    X0 = torch.randn(nd, m, dtype=torch.float64, device="cuda", generator=g) * free[:, None]
    lam, V, it = lobpcg(A, B, T, X0, nmodes, tol=tol, maxiter=maxiter, log=log)
    return np.maximum(lam, 0.0), V.T.contiguous()


def _ops_block(ops, free):
    """(n, m) -> (n, m): V -> free * sum_b K_b (free * V) of stored element ops
    [(dofs, Ke)] on their blocks (gfem/eigen.py:97-110), up to 16 columns per
    stored-Ke product (one read of each block's Ke serves all of them)."""
    def apply(V):
        W = (V * free[:, None]).contiguous()
        out = torch.empty_like(W)
        for j in range(0, W.shape[1], 16):
            Wj = W[:, j:j + 16].contiguous()
            y = None
            for blk, K in ops:
                t = blk.ebe_matvec_multi(K, Wj, apply_bc=False)
                y = t if y is None else y + t
            out[:, j:j + 16] = y * free[:, None]
        return out
    return apply


def buckling_lobpcg(model, K0ops, KGops, setup, nmodes, monitor=None, tol=1e-6, maxiter=500):
    """Buckling loads of K0 phi = -lambda KG phi (gfem/eigen.py:137-151): the
    smallest mu of KG phi = mu K0 phi by LOBPCG with A = KG, B = K0 and a device
    AMG V-cycle of K0 as preconditioner; lambda = -1/mu for mu < 0 (infinity
    otherwise).  K0ops, KGops: per block (Block, Ke) stored FP64 element matrices.
    Returns (lambda (nmodes,), modes (nmodes, ndof))."""
    from .solvers import Monitor
    mon = monitor or Monitor(False)
    free = setup.free
    for blk in model.blocks:
        blk.set_fixed(setup.fixed)
    A = _ops_block(KGops, free)
    B = _ops_block(K0ops, free)
    amg = linalg.DeviceAMG([b for b, _ in K0ops], [K for _, K in K0ops], keep_level0=True)
    mon.log(f"  buckling (device LOBPCG): {int(setup.free_np.sum())} free dofs, {amg.info()}")

    def T(R):
        return torch.stack([amg.vcycle(R[:, j].contiguous()) for j in range(R.shape[1])], 1) * free[:, None]

    m = nmodes + max(4, nmodes // 2)
    g = torch.Generator(device="cuda").manual_seed(1)
    X0 = torch.randn(model.ndof, m, dtype=torch.float64, device="cuda", generator=g) * free[:, None]
    mu, V, it = lobpcg(A, B, T, X0, nmodes, tol=tol, maxiter=maxiter, log=mon.log)
    lam = np.where(mu < 0, -1.0 / np.where(mu < 0, mu, -1.0), np.inf)
    order = np.argsort(lam)
    mon.log(f"  LOBPCG converged in {it} iterations")
    return lam[order], V.T[order].contiguous()


def buckling(model, step, nmodes, state=None, monitor=None, tol=1e-6, linear_solver="auto"):
    """Linear (eigenvalue) buckling (gfem/solvers.py:1074-1110): the linear response
    to the step's loads with its prescribed DOFs held at zero, the element stresses
    of that response, K0 at u = 0 and the initial-stress stiffness KG, then
    :func:`buckling_lobpcg`.  Returns (load factors (nmodes,), modes (nmodes, ndof))."""
    from .solvers import Step, StaticSolver
    base = Step("base", bcs=[(b[0], b[1], 0.0) for b in step.bcs], loads=step.loads, dloads=step.dloads)
    solver = StaticSolver(model, linear_solver=linear_solver, cg_tol=1e-10, verbose=False)
    u, states, _ = solver.solve(base, state=State(model))
    stress = model.stresses(u, states)
    zero = torch.zeros(model.ndof, dtype=torch.float64, device="cuda")
    K0ops = [(b, b.stiffness(zero, b.init_state())) for b in model.blocks]
    KGops = [(b, b.geometric_stiffness(st["S"])) for b, st in zip(model.blocks, stress)]
    setup = _Setup(model, base, state or State(model))
    return buckling_lobpcg(model, K0ops, KGops, setup, nmodes, monitor, tol)

