"""Smoothed-aggregation set-up on the device (linalg.DeviceAMG) against the host
set-up (linalg.amg_setup) and the oracle's direct solve.

Bars: the device hierarchy has the host hierarchy's level sizes (the same
aggregation of the same strength graph), and with the spectral bounds made equal
its V-cycle equals the host hierarchy's to 1e-10 (FP64; the products are summed
in another order, nothing else differs); solves preconditioned by it reach the
oracle's direct solution to 1e-8 relative displacement (plain FP64 path and mixed
FP32/FP64 path).
"""
import ctypes as C

import numpy as np
import pytest
import torch

from helpers import cantilever_bcs, rel_err, tet10_box
from oracle import fem as ofem
from oracle import solvers as osol

pytestmark = pytest.mark.gpu

E, NU = 210000.0, 0.3


def _hex_case():
    import exfem_b200 as xf
    from exfem_b200 import mesh
    X, c = mesh.box_hex(100.0, 20.0, 20.0, 40, 8, 8)
    X = mesh.jitter_interior(X, [2.5, 2.5, 2.5], 0.1, 4)
    fix, tip, bcs, loads = cantilever_bcs(X, 100.0)
    return X, c, xf.HEX8, ofem.HEX8, bcs, loads, None


def _tet_case(n=8):
    import exfem_b200 as xf
    from exfem_b200 import mesh
    X, c = tet10_box(1.0, 1.0, 1.0, n, n, n, frac=0.1, seed=2)
    sc = np.exp(np.random.default_rng(3).uniform(0, np.log(10), size=len(c)))
    fix = mesh.nodes_where(X, lambda x, y, z: z < 1e-9)
    top = mesh.nodes_where(X, lambda x, y, z: z > 1 - 1e-9)
    bcs = [(fix, d, 0.0) for d in range(3)]
    loads = [(top, 2, 1.0 / len(top))]
    return X, c, xf.TET10, ofem.TET10, bcs, loads, sc


@pytest.mark.parametrize("case", ["hex", "tet"])
def test_device_setup_matches_host_setup(cuda, case):
    import exfem_b200 as xf
    from exfem_b200 import _lib, linalg
    from exfem_b200._lib import lib
    # both meshes coarsen twice: 3x3 node blocks, then 6x6 aggregate blocks
    X, c, pet, oet, bcs, loads, sc = _hex_case() if case == "hex" else _tet_case()
    om = ofem.Model(X)
    om.add_block(c, oet, ofem.LinearElastic(E, NU))
    setup = osol.Setup(om, osol.Step(bcs=bcs, loads=loads))
    pm = xf.Model(X)
    blk = pm.add_block(c, pet, xf.LinearElastic(E, NU))
    fields = dict(scale=[sc]) if sc is not None else None
    Ke = pm.element_stiffness(torch.zeros(pm.ndof, device="cuda", dtype=torch.float64), pm.init_state(), fields)[0]
    blk.set_fixed(setup.fixed)
    A = linalg.bc_matrix(linalg.ops_assemble([(blk.dofs(), Ke)], pm.ndof), setup.free)
    host = xf.AMG(A, X)
    dev = linalg.DeviceAMG(blk, Ke, keep_level0=True)
    assert host.nlevels >= 3
    assert dev.sizes == host.sizes
    # same spectral bounds on both (per-row form of each level's uniform bound)
    for l, lv in enumerate(host.levels):
        rows = np.full(lv["n"], lv["rho"])
        for h in (host.handle, dev.handle):
            _lib.check(lib.exfem_amg_set_level_rows(h, l, rows.ctypes.data))
    b = np.random.default_rng(0).standard_normal(pm.ndof) * setup.free
    bt = torch.as_tensor(b, device="cuda")
    assert rel_err(dev.vcycle(bt), host.vcycle(bt)) < 1e-10
    blk.set_fixed(None)


def test_device_setup_plain_fp64_solve(cuda):
    import exfem_b200 as xf
    X, c, pet, oet, bcs, loads, _ = _hex_case()
    om = ofem.Model(X)
    om.add_block(c, oet, ofem.LinearElastic(E, NU))
    uo, _, _ = osol.StaticSolver(om, rtol=1e-6).solve(osol.Step(bcs=bcs, loads=loads))
    pm = xf.Model(X)
    pm.add_block(c, pet, xf.LinearElastic(E, NU))
    s = xf.StaticSolver(pm, rtol=1e-6, linear_solver="amg", cg_tol=1e-10, verbose=False, amg_setup="device")
    up, _, _ = s.solve(xf.Step(bcs=bcs, loads=loads))
    assert isinstance(s.lin.amg, xf.linalg.DeviceAMG)
    assert rel_err(up, uo) < 1e-8


def test_device_setup_mixed_solve(cuda):
    import exfem_b200 as xf
    X, c, pet, oet, bcs, loads, sc = _tet_case(6)
    om = ofem.Model(X)
    om.add_block(c, oet, ofem.LinearElastic(1000.0, 0.3))
    uo, _, _ = osol.StaticSolver(om, rtol=1e-6, scale=[sc]).solve(osol.Step(bcs=bcs, loads=loads))
    res = {}
    for where in ("host", "device"):
        pm = xf.Model(X)
        pm.add_block(c, pet, xf.LinearElastic(1000.0, 0.3))
        s = xf.StaticSolver(pm, rtol=1e-6, linear_solver="mixed", cg_tol=1e-10, verbose=False, amg_setup=where)
        res[where], _, _ = s.solve(xf.Step(bcs=bcs, loads=loads), scale=[sc])
        assert rel_err(res[where], uo) < 1e-8
    assert rel_err(res["device"], res["host"]) < 1e-8
