"""Many load cases on one linear-elastic model (drop-in for
``gfem.optimize.multi_load_cases``, gfem/optimize.py:116-143).

The reference takes the element matrices at u = 0 and runs one Jacobi-PCG per load
case (vmapped), on the free part of each load vector, with the step's boundary
conditions (prescribed DOFs held at zero: identity rows, zero right-hand side).

``method="batch"`` (default) solves every case in one batched run instead: each
case is an instance of :class:`batch.BatchSolver` (FP32 matrix-free AMG-PCG inside
FP64 refinement to ``cg_tol``, every instance with its own scalars and stopping
test).  A model of several blocks (materials or element types) solves its cases one
after another with the same FP32/FP64 mixed solver over all of its blocks and one
device hierarchy.  ``method="jacobi"`` keeps the reference's algorithm: FP64
stored-Ke Jacobi-PCG for every case, to ``cg_tol`` — on a one-block model all cases
(up to 16 per call) share each stored-Ke product (``Block.multi_pcg``: one read of
Ke per iteration for every case, each case with its own scalars and stopping test,
the loop on the device), on a model of several blocks one case after another.
"""
import numpy as np
import torch

from . import batch, linalg
from .linalg import NativeSolver
from .materials import LinearElastic
from .solvers import State, _Setup


def multi_load_cases(model, step, cases, cg_tol=1e-8, method="batch"):
    """(ncase, ndof) displacements of the load vectors ``cases`` (ncase, ndof) under
    the boundary conditions of ``step`` (FP64 tensor on the device)."""
    if not all(isinstance(b.material, LinearElastic) for b in model.blocks):
        raise TypeError("multi_load_cases is linear elastic")
    if method not in ("batch", "jacobi"):
        raise ValueError(f"unknown method {method!r}")
    F = np.asarray(cases.detach().cpu() if isinstance(cases, torch.Tensor) else cases, dtype=np.float64)
    F = F.reshape(-1, model.ndof)
    setup = _Setup(model, step, State(model))
    free = setup.free_np
    rhs = F * free[None, :]
    if method == "batch" and len(model.blocks) == 1:
        blk = model.blocks[0]
        p = batch.Problem(model.X, blk.conn, blk.etype, blk.material, setup.fixed, rhs)
        S = batch.BatchSolver([p])
        x, info = S.solve(tol=cg_tol)
        return torch.stack(S.split(x))
    zero = torch.zeros(model.ndof, dtype=torch.float64, device="cuda")
    for blk in model.blocks:
        blk.set_fixed(setup.fixed)
    Kes = [blk.stiffness(zero, blk.init_state()) for blk in model.blocks]
    if method == "batch":
        S = NativeSolver(model.blocks, "mf32", "amg", linalg.DeviceAMG(model.blocks, Kes))
        del Kes
        return torch.stack([S.mixed(torch.as_tensor(f, device="cuda"), tol=cg_tol)[0] for f in rhs])
    if len(model.blocks) == 1:
        B = torch.as_tensor(rhs.T.copy(), device="cuda")
        X, iters, rel = model.blocks[0].multi_pcg(Kes[0], B, tol=cg_tol, maxiter=20000)
        return X.T.contiguous()
    S = NativeSolver(model.blocks, "ebe64", "jacobi", None)
    S.set_ke(Kes)
    out = []
    for f in rhs:
        x, k, rr = S.pcg(torch.as_tensor(f, device="cuda"), tol=cg_tol, maxiter=20000)
        out.append(x)
    return torch.stack(out)
