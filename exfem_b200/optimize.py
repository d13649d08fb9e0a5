"""Many load cases on one linear-elastic model (drop-in for
``gfem.optimize.multi_load_cases``, gfem/optimize.py:116-143).

The reference takes the element matrices at u = 0 and runs one Jacobi-PCG per load
case (vmapped), on the free part of each load vector, with the step's boundary
conditions (prescribed DOFs held at zero: identity rows, zero right-hand side).

``method="batch"`` (default) solves every case in one batched run instead: each
case is an instance of :class:`batch.BatchSolver` (FP32 matrix-free AMG-PCG inside
FP64 refinement to ``cg_tol``, every instance with its own scalars and stopping
test).  ``method="jacobi"`` keeps the reference's algorithm: FP64 stored-Ke
Jacobi-PCG per case, to ``cg_tol``.
"""
import numpy as np
import torch

from . import batch
from .linalg import NativeSolver
from .materials import LinearElastic
from .solvers import State, _Setup


def multi_load_cases(model, step, cases, cg_tol=1e-8, method="batch"):
    """(ncase, ndof) displacements of the load vectors ``cases`` (ncase, ndof) under
    the boundary conditions of ``step`` (FP64 tensor on the device)."""
    if len(model.blocks) != 1:
        raise NotImplementedError("multi_load_cases covers single-block models")
    blk = model.blocks[0]
    if not isinstance(blk.material, LinearElastic):
        raise TypeError("multi_load_cases is linear elastic")
    F = np.asarray(cases.detach().cpu() if isinstance(cases, torch.Tensor) else cases, dtype=np.float64)
    F = F.reshape(-1, model.ndof)
    setup = _Setup(model, step, State(model))
    free = setup.free_np
    rhs = F * free[None, :]
    if method == "batch":
        p = batch.Problem(model.X, blk.conn, blk.etype, blk.material, setup.fixed, rhs)
        S = batch.BatchSolver([p])
        x, info = S.solve(tol=cg_tol)
        return torch.stack(S.split(x))
    if method != "jacobi":
        raise ValueError(f"unknown method {method!r}")
    Ke = blk.stiffness(torch.zeros(model.ndof, dtype=torch.float64, device="cuda"), blk.init_state())
    blk.set_fixed(setup.fixed)
    S = NativeSolver(blk, "ebe64", "jacobi", None)
    S.set_ke(Ke)
    out = []
    for f in rhs:
        x, k, rr = S.pcg(torch.as_tensor(f, device="cuda"), tol=cg_tol, maxiter=20000)
        out.append(x)
    return torch.stack(out)
