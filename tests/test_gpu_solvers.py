"""Device AMG V-cycle, PCG, mixed refinement and the Newton loop against the oracle.

Bars: the device V-cycle equals the oracle's restatement of gfem/linalg.py:156-195
on the same hierarchy to 1e-12 (FP64); converged displacements agree with the
oracle's direct solve to 1e-8 relative (the plain FP64 path at cg_tol 1e-10, and
the mixed FP32/FP64 path at tol 1e-9); the J2 Newton loop reproduces the
oracle's per-increment Newton iteration counts; the reference's analytic checks
(tests/test_verification.py:27-36, 39-52, 66-83) hold on the device path.
"""
import numpy as np
import pytest
import torch

from helpers import cantilever_bcs, jittered_box, rel_err, tet10_box
from oracle import fem as ofem
from oracle import linalg as olin
from oracle import solvers as osol

pytestmark = pytest.mark.gpu

E, NU = 210000.0, 0.3


def _config1():
    import exfem_b200 as xf
    from exfem_b200 import mesh
    X, c = mesh.box_hex(100.0, 20.0, 20.0, 20, 4, 4)
    fix, tip, bcs, loads = cantilever_bcs(X, 100.0)
    pm = xf.Model(X)
    pm.add_block(c, xf.HEX8, xf.LinearElastic(E, NU))
    om = ofem.Model(X)
    om.add_block(c, ofem.HEX8, ofem.LinearElastic(E, NU))
    return X, c, bcs, loads, pm, om


def _oracle_direct(om, bcs, loads):
    st = osol.Step(bcs=bcs, loads=loads)
    u, s, info = osol.StaticSolver(om, rtol=1e-6).solve(st)
    return u


def test_vcycle_matches_oracle(cuda):
    import exfem_b200 as xf
    X, c, bcs, loads, pm, om = _config1()
    setup = osol.Setup(om, osol.Step(bcs=bcs, loads=loads))
    ops = [(d, K.numpy()) for d, K in om.stiffness_ops(torch.zeros(om.ndof, dtype=torch.float64), om.init_state())]
    A = olin.bc_matrix(ofem.ops_assemble(ops, om.ndof), setup.free)
    amg = xf.AMG(A, X)
    assert amg.nlevels >= 2
    levels = [dict(A=lv["A"], dinv=lv["dinv"], rho=lv["rho"], P=lv["P"], R=lv["R"]) for lv in amg.levels]
    b = np.random.default_rng(0).standard_normal(om.ndof) * setup.free
    zo = olin.vcycle(levels, amg.coarse, b)
    zp = amg.vcycle(torch.as_tensor(b, device="cuda"))
    assert rel_err(zp, zo) < 1e-12
    z32 = amg.vcycle(torch.as_tensor(b, device="cuda", dtype=torch.float32))
    assert rel_err(z32.double(), zo) < 1e-4
    # level 0 smoothed with the matrix-free tangent (gfem/solvers.py:311-314)
    blk = pm.blocks[0]
    blk.set_fixed(setup.fixed)
    blk.tangent_update(torch.zeros(pm.ndof, device="cuda"), pm.init_state()[0])
    d = blk.tangent_diagonal().cpu().numpy()
    dinv0 = np.where(setup.free > 0, 1.0 / np.where(np.abs(d) > 0, d, 1.0), 1.0)
    A0 = lambda v: A @ v                                        # the same operator, assembled
    zo0 = olin.vcycle(levels, amg.coarse, b, A0=A0, dinv0=dinv0)
    zp0 = amg.vcycle(torch.as_tensor(b, device="cuda"), blk, torch.as_tensor(dinv0, device="cuda"))
    assert rel_err(zp0, zo0) < 1e-11
    blk.set_fixed(None)


@pytest.mark.parametrize("method,tangent,operator", [("amg", "ebe", "gather"), ("amg", "ebe", "csr"),
                                                     ("amg", "mf", "gather"), ("mixed", "mf", "gather"),
                                                     ("jacobi", "ebe", "gather"), ("jacobi", "ebe", "csr")])
def test_config1_linear_solve(cuda, method, tangent, operator):
    import exfem_b200 as xf
    X, c, bcs, loads, pm, om = _config1()
    uo = _oracle_direct(om, bcs, loads)
    st = xf.Step(bcs=bcs, loads=loads)
    tol = 1e-10 if method != "mixed" else 1e-9
    up, s, info = xf.StaticSolver(pm, rtol=1e-6, linear_solver=method, tangent=tangent, cg_tol=tol,
                                  verbose=False, operator=operator).solve(st)
    err = rel_err(up, uo)
    assert err < (1e-8 if method != "jacobi" else 1e-7), err


def test_graph_and_eager_pcg_agree(cuda):
    import exfem_b200 as xf
    X, c, bcs, loads, pm, om = _config1()
    res = []
    for graph in (True, False):
        st = xf.Step(bcs=bcs, loads=loads)
        s = xf.StaticSolver(pm, rtol=1e-6, linear_solver="amg", cg_tol=1e-10, verbose=False, graph=graph)
        u, _, _ = s.solve(st)
        res.append((u.cpu().numpy(), s.lin.last_iters))
    assert res[0][1] == res[1][1]
    np.testing.assert_array_equal(res[0][0], res[1][0])       # deterministic reductions


def test_device_loop_matches_host_driven_loop(cuda):
    """The PCG loop run to its stopping test inside one graph launch (conditional
    while node) gives the same iterates, bit for bit, as graphs of 8 iterations
    launched from the host and as eager launches; an iteration limit ends it."""
    from exfem_b200 import linalg
    X, c, bcs, loads, pm, om = _config1()
    blk = pm.blocks[0]
    setup = osol.Setup(om, osol.Step(bcs=bcs, loads=loads))
    blk.set_fixed(setup.fixed)
    blk.tangent_update(torch.zeros(pm.ndof, device="cuda"), pm.init_state()[0])
    ops = [(d, K.numpy()) for d, K in om.stiffness_ops(torch.zeros(om.ndof, dtype=torch.float64), om.init_state())]
    import exfem_b200 as xf
    amg = xf.AMG(olin.bc_matrix(ofem.ops_assemble(ops, om.ndof), setup.free), X)
    b = torch.as_tensor(np.random.default_rng(3).standard_normal(pm.ndof) * setup.free, device="cuda")
    modes = [dict(graph=True, device_loop=True), dict(graph=True, device_loop=False), dict(graph=False)]
    for op in ("mf64", "mf32"):
        res = []
        for kw in modes:
            S = linalg.NativeSolver(blk, op, "amg", amg, **kw)
            if op == "mf64":
                x, k, rr = S.pcg(b, tol=1e-10)
                res.append((x.cpu().numpy(), k))
                xl, kl, _ = S.pcg(b, tol=1e-14, maxiter=3)
                assert kl == 3
            else:
                x, k, p, rel = S.mixed(b, tol=1e-9)
                res.append((x.cpu().numpy(), (k, p)))
                assert rel < 1e-9
        for x, k in res[1:]:
            assert k == res[0][1]
            np.testing.assert_array_equal(x, res[0][0])
    blk.set_fixed(None)


def _j2_case(dt):
    import exfem_b200 as xf
    from exfem_b200 import mesh
    X, c = jittered_box(100.0, 20.0, 20.0, 10, 2, 2, frac=0.1, seed=1)
    fix = mesh.nodes_where(X, lambda x, y, z: x < 1e-9)
    tip = mesh.nodes_where(X, lambda x, y, z: x > 100.0 - 1e-9)
    bcs = [(fix, d, 0.0) for d in range(3)] + [(tip, 2, -2.0)]
    table = [[250.0, 0.0], [1250.0, 1.0]]
    om = ofem.Model(X)
    om.add_block(c, ofem.HEX8, ofem.J2Plasticity(E, NU, table))
    uo, so, io = osol.StaticSolver(om, rtol=1e-6).solve(osol.Step(bcs=bcs, dt_init=dt, dt_max=dt))
    pm = xf.Model(X)
    pm.add_block(c, xf.HEX8, xf.J2Plasticity(E, NU, table))
    return X, bcs, om, uo, so, io, pm


@pytest.mark.parametrize("dt", [1.0, 0.2])
def test_device_newton_increment_matches_host_loop(cuda, dt):
    """The increment as one graph launch (exfem_newton_increment: predictor, Newton
    corrections, line search and mixed solves on the device) against the host
    driver's loop on the same solver configuration: the same Newton corrections
    in every increment, displacements and von Mises stresses equal to the linear
    solves' tolerance, and both within the reference's bars of the oracle."""
    import exfem_b200 as xf
    X, bcs, om, uo, so, io, pm = _j2_case(dt)
    res = []
    for device in (True, False):
        m = xf.Model(X)
        m.add_block(pm.blocks[0].conn, xf.HEX8, xf.J2Plasticity(E, NU, [[250.0, 0.0], [1250.0, 1.0]]))
        s = xf.StaticSolver(m, rtol=1e-6, linear_solver="mixed", tangent="mf", cg_tol=1e-10, verbose=False,
                            device_newton=device)
        assert s._device_increment_ok() == device
        u, st, info = s.solve(xf.Step(bcs=bcs, dt_init=dt, dt_max=dt))
        res.append((u, m.stresses(u, st)[0]["MISES"], [h[1] for h in info["history"]]))
    (ud, md, cd), (uh, mh, ch) = res
    assert cd == ch, (cd, ch)
    assert rel_err(ud, uh) < 1e-9 and rel_err(md, mh) < 1e-8
    co = [h[1] for h in io["history"]]
    assert len(cd) == len(co) and all(abs(a - b) <= 1 for a, b in zip(cd, co)), (cd, co)
    assert rel_err(ud, uo) < 1e-5


def test_device_newton_failed_increment_cuts_back(cuda):
    """An increment that the device graph cannot converge (max_iter = 2 where the
    oracle needs more Newton corrections) comes back as failed and the host cuts the
    increment back, as for the host loop: both paths take the same increments; without
    line search both also take the same corrections."""
    import exfem_b200 as xf
    X, bcs, om, uo, so, io, pm = _j2_case(1.0)
    assert max(h[1] for h in io["history"]) >= 2
    res = []
    for device in (True, False):
        m = xf.Model(X)
        m.add_block(pm.blocks[0].conn, xf.HEX8, xf.J2Plasticity(E, NU, [[250.0, 0.0], [1250.0, 1.0]]))
        s = xf.StaticSolver(m, rtol=1e-6, max_iter=2, linear_solver="mixed", tangent="mf", cg_tol=1e-10,
                            verbose=False, device_newton=device, line_search=False)
        try:
            u, st, info = s.solve(xf.Step(bcs=bcs, dt_init=1.0, dt_max=1.0, dt_min=1e-3, max_inc=50))
            out = ("done", [round(h[0], 12) for h in info["history"]], info["increments"])
        except RuntimeError as e:
            out = ("failed", str(e).split(":")[0], None)
        res.append(out)
        m2 = xf.Model(X)
        m2.add_block(pm.blocks[0].conn, xf.HEX8, xf.J2Plasticity(E, NU, [[250.0, 0.0], [1250.0, 1.0]]))
        s2 = xf.StaticSolver(m2, rtol=1e-6, linear_solver="mixed", tangent="mf", cg_tol=1e-10, verbose=False,
                             device_newton=device, line_search=False)
        u, st, info = s2.solve(xf.Step(bcs=bcs, dt_init=1.0, dt_max=1.0))
        res.append((u, [h[1] for h in info["history"]]))
    (cut_d, full_d), (cut_h, full_h) = res[0:2], res[2:4]
    assert cut_d == cut_h, (cut_d, cut_h)
    assert cut_d[0] == "failed" or cut_d[2] > len(cut_d[1])      # at least one increment was cut back
    assert full_d[1] == full_h[1]
    assert rel_err(full_d[0], full_h[0]) < 1e-9


def test_device_newton_nonfinite_load_fails(cuda):
    """A non-finite external force makes every device increment report failure (the
    residual test sees a non-finite norm) and the step ends with the dt_min error,
    with no fault on the GPU."""
    import exfem_b200 as xf
    X, bcs, om, uo, so, io, pm = _j2_case(1.0)
    m = xf.Model(X)
    m.add_block(pm.blocks[0].conn, xf.HEX8, xf.J2Plasticity(E, NU, [[250.0, 0.0], [1250.0, 1.0]]))
    s = xf.StaticSolver(m, rtol=1e-6, linear_solver="mixed", tangent="mf", cg_tol=1e-10, verbose=False)
    assert s._device_increment_ok()
    tip = np.nonzero(X[:, 0] > 100.0 - 1e-9)[0]
    with pytest.raises(RuntimeError):
        s.solve(xf.Step(bcs=bcs[:3], loads=[(tip, 2, float("nan"))], dt_init=1.0, dt_max=1.0, dt_min=0.1))


@pytest.mark.parametrize("method,tangent", [("amg", "ebe"), ("mixed", "mf")])
def test_j2_newton_counts_single_increment(cuda, method, tangent):
    """One increment from the virgin state: no Gauss point starts on the yield
    surface, so every Newton iterate is decided by the arithmetic, not by the sign
    of a rounding-level yield function, and the iteration counts must be equal."""
    import exfem_b200 as xf
    X, bcs, om, uo, so, io, pm = _j2_case(1.0)
    up, sp, ip = xf.StaticSolver(pm, rtol=1e-6, linear_solver=method, tangent=tangent, cg_tol=1e-10,
                                 verbose=False).solve(xf.Step(bcs=bcs, dt_init=1.0, dt_max=1.0))
    assert [h[1] for h in ip["history"]] == [h[1] for h in io["history"]], (ip["history"], io["history"])
    assert float(so[0][..., 9].max()) > 0
    assert rel_err(up, uo) < 1e-6
    mo = om.stresses(torch.as_tensor(uo), so)[0]["MISES"]
    assert rel_err(pm.stresses(up, sp)[0]["MISES"], mo) < 1e-5


@pytest.mark.parametrize("method,tangent", [("amg", "ebe"), ("mixed", "mf")])
def test_j2_newton_multi_increment(cuda, method, tangent):
    """Five increments.  After the first, every plastic Gauss point starts the
    increment exactly on the yield surface, where the predictor's choice between
    the elastic and the consistent tangent follows the sign of a rounding-level
    yield function (in the reference as well); counts may then differ by one per
    increment while the converged states agree to the Newton tolerance."""
    import exfem_b200 as xf
    X, bcs, om, uo, so, io, pm = _j2_case(0.2)
    up, sp, ip = xf.StaticSolver(pm, rtol=1e-6, linear_solver=method, tangent=tangent, cg_tol=1e-10,
                                 verbose=False).solve(xf.Step(bcs=bcs, dt_init=0.2, dt_max=0.2))
    co, cp = [h[1] for h in io["history"]], [h[1] for h in ip["history"]]
    assert len(co) == len(cp) and co[:2] == cp[:2], (cp, co)
    assert all(abs(a - b) <= 1 for a, b in zip(co, cp)), (cp, co)
    assert rel_err(up, uo) < 1e-5
    mo = om.stresses(torch.as_tensor(uo), so)[0]["MISES"]
    assert rel_err(pm.stresses(up, sp)[0]["MISES"], mo) < 1e-4


@pytest.mark.parametrize("etype", ["C3D8", "C3D10"])
def test_patch_linear(cuda, etype):
    """tests/test_verification.py:27-36 on the device path."""
    import exfem_b200 as xf
    from exfem_b200 import mesh
    Ev = 200e3
    X, c = mesh.box_hex(1, 1, 1, 2, 2, 2)
    if etype == "C3D10":
        X, c = mesh.tet4_to_tet10(*mesh.hex_to_tet4(X, c))
    m = xf.Model(X)
    m.add_block(c, xf.ELEMENTS[etype], xf.LinearElastic(Ev, NU))
    w = lambda f: mesh.nodes_where(X, f)
    bcs = [(w(lambda x, y, z: x < 1e-9), 0, 0.0), (w(lambda x, y, z: y < 1e-9), 1, 0.0),
           (w(lambda x, y, z: z < 1e-9), 2, 0.0), (w(lambda x, y, z: x > 1 - 1e-9), 0, 1e-3)]
    u, s, info = xf.StaticSolver(m, linear_solver="amg", cg_tol=1e-12, verbose=False).solve(xf.Step(bcs=bcs))
    S = m.stresses(u, s)[0]["S"].cpu().numpy()
    assert np.allclose(S[:, 0, 0], Ev * 1e-3, rtol=1e-6)
    assert np.allclose(S[:, 1, 1], 0, atol=1e-6 * Ev)
    U = u.cpu().numpy().reshape(-1, 3)
    assert np.allclose(U[:, 1].min(), -NU * 1e-3, rtol=1e-6)


def test_j2_uniaxial_hardening(cuda):
    """tests/test_verification.py:39-52 on the device path."""
    import exfem_b200 as xf
    from exfem_b200 import mesh
    Ev, sy, H = 200e3, 250.0, 2000.0
    X, c = mesh.box_hex(1, 1, 1, 1, 1, 1)
    m = xf.Model(X)
    m.add_block(c, xf.HEX8, xf.J2Plasticity(Ev, NU, [[sy, 0.0], [sy + H * 0.1, 0.1]]))
    w = lambda f: mesh.nodes_where(X, f)
    bcs = [(w(lambda x, y, z: x < 1e-9), 0, 0.0), (w(lambda x, y, z: y < 1e-9), 1, 0.0),
           (w(lambda x, y, z: z < 1e-9), 2, 0.0), (w(lambda x, y, z: x > 1 - 1e-9), 0, 0.01)]
    u, s, info = xf.StaticSolver(m, linear_solver="amg", cg_tol=1e-12, verbose=False).solve(
        xf.Step(bcs=bcs, dt_init=0.1, dt_max=0.1))
    r = m.stresses(u, s)[0]
    sxx = float(r["S"][0, 0, 0])
    eps, ey = 0.01, sy / Ev
    expected = sy + Ev * H / (Ev + H) * (eps - ey)
    assert abs(sxx - expected) / expected < 1e-4
    assert abs(float(r["PEEQ"][0]) - (eps - sxx / Ev)) < 1e-6


def test_tet10_cantilever_vs_beam_theory(cuda):
    """tests/test_verification.py:66-83 on the device path."""
    import exfem_b200 as xf
    from exfem_b200 import mesh
    Ev, L, h = 200e3, 10.0, 1.0
    X, c = mesh.box_hex(L, h, h, 20, 2, 2)
    X, c = mesh.tet4_to_tet10(*mesh.hex_to_tet4(X, c))
    m = xf.Model(X)
    m.add_block(c, xf.TET10, xf.LinearElastic(Ev, NU))
    fix = mesh.nodes_where(X, lambda x, y, z: x < 1e-9)
    tip = mesh.nodes_where(X, lambda x, y, z: x > L - 1e-9)
    st = xf.Step(bcs=[(fix, d, 0.0) for d in range(3)], loads=[(tip, 1, -1.0 / len(tip))])
    u, s, info = xf.StaticSolver(m, linear_solver="mixed", cg_tol=1e-10, verbose=False).solve(st)
    I = h ** 4 / 12
    d_beam = L ** 3 / (3 * Ev * I) + L / (5 / 6 * Ev / (2 * (1 + NU)) * h * h)
    d = -float(u.cpu().numpy().reshape(-1, 3)[tip, 1].mean())
    assert abs(d - d_beam) / d_beam < 0.03
    R = info["reactions"].cpu().numpy().reshape(-1, 3)[:, 1].sum()
    assert abs(R - 1.0) < 1e-6


def test_tet10_mixed_vs_direct(cuda):
    import exfem_b200 as xf
    from exfem_b200 import mesh
    X, c = tet10_box(1.0, 1.0, 1.0, 4, 4, 4, frac=0.1, seed=2)
    rng = np.random.default_rng(3)
    sc = np.exp(rng.uniform(0, np.log(10), size=len(c)))
    fix = mesh.nodes_where(X, lambda x, y, z: z < 1e-9)
    top = mesh.nodes_where(X, lambda x, y, z: z > 1 - 1e-9)
    bcs = [(fix, d, 0.0) for d in range(3)]
    loads = [(top, 2, 1.0 / len(top))]
    om = ofem.Model(X)
    om.add_block(c, ofem.TET10, ofem.LinearElastic(1000.0, 0.3))
    uo, _, _ = osol.StaticSolver(om, rtol=1e-6, scale=[sc]).solve(osol.Step(bcs=bcs, loads=loads))
    pm = xf.Model(X)
    pm.add_block(c, xf.TET10, xf.LinearElastic(1000.0, 0.3))
    up, _, _ = xf.StaticSolver(pm, rtol=1e-6, linear_solver="mixed", cg_tol=1e-10, verbose=False).solve(
        xf.Step(bcs=bcs, loads=loads), scale=[sc])
    assert rel_err(up, uo) < 1e-8


@pytest.mark.parametrize("method", ["mixed", "amg"])
def test_config3_construction_matches_oracle(cuda, method):
    """The mixed-precision scale case built exactly as at full size, on a sub-cube
    the oracle's direct solve handles (8^3 hexahedra x 6 Kuhn C3D10, 14,739 DOF):
    interior jitter +-10% h, per-element E log-uniform in [1, 10] GPa through the
    stiffness scale, z = 0 clamped, 1 MPa outward traction on z = 1 as the pressure
    vector of the top sub-surface of the skin.  The mixed FP32/FP64 path and the
    plain FP64 path (device set-up of the hierarchy) against the oracle's load
    vector and sparse direct solution: 1e-8 relative displacement."""
    import exfem_b200 as xf
    from exfem_b200 import loads, mesh, surfaces
    from oracle import loads as oloads
    n = 8
    X, c = mesh.box_hex(1.0, 1.0, 1.0, n, n, n)
    X = mesh.jitter_interior(X, 1.0 / n, 0.1, 0)
    X, c = mesh.tet4_to_tet10(*mesh.hex_to_tet4(X, c))
    sc = np.exp(np.random.default_rng(1).uniform(0.0, np.log(10.0), size=len(c)))
    fix = np.nonzero(X[:, 2] < 1e-9)[0]
    top = np.nonzero(X[:, 2] > 1 - 1e-9)[0]
    bcs = [(fix, d, 0.0) for d in range(3)]
    fo = oloads.pressure_vector(X, oloads.sub_surface(oloads.skin_tet10(X, c), top, len(X)), -1.0)
    om = ofem.Model(X)
    om.add_block(c, ofem.TET10, ofem.LinearElastic(1000.0, 0.3))
    uo, _, _ = osol.StaticSolver(om, rtol=1e-6, scale=[sc]).solve(osol.Step(bcs=bcs, dloads=[fo]))
    pm = xf.Model(X)
    pm.add_block(c, xf.TET10, xf.LinearElastic(1000.0, 0.3))
    f = loads.pressure_vector(X, surfaces.sub_surface(surfaces.skin(X, pm.blocks), top), -1.0)
    assert np.abs(f - fo).max() <= 1e-14 * np.abs(fo).max()
    up, _, _ = xf.StaticSolver(pm, rtol=1e-6, linear_solver=method, tangent="mf", cg_tol=1e-11, verbose=False,
                               amg_setup="device").solve(xf.Step(bcs=bcs, dloads=[f]), scale=[sc])
    assert rel_err(up, uo) < 1e-8, rel_err(up, uo)


def test_bounded_wait_gives_up_and_context_stays_usable(cuda):
    """Failure detection without a GPU fault: a kernel whose barrier nothing arrives
    on must give up after its poll limit and report EXFEM_ERR_TIMEOUT; the next
    product still works and the block reports no failed wait."""
    from exfem_b200 import _lib
    from exfem_b200._lib import lib, stream_ptr
    st = lib.exfem_selftest_bounded_wait(1 << 10, stream_ptr())
    assert st == _lib.ERR_TIMEOUT
    assert "gave up" in _lib.last_error()
    X, c = tet10_box(1, 1, 1, 3, 2, 2)
    import exfem_b200 as xf
    m = xf.Model(X)
    blk = m.add_block(c, xf.TET10, xf.LinearElastic(1000.0, 0.3))
    v = torch.randn(m.ndof, dtype=torch.float32, device="cuda")
    y = blk.tangent_matvec(v)
    torch.cuda.synchronize()
    assert torch.isfinite(y).all()
    assert lib.exfem_block_status(blk.handle, stream_ptr()) == _lib.OK


def test_deck_solve_matches_oracle(cuda):
    """An input deck read by the deck reader (tests/golden/cantilever_c3d10.inp:
    encastre, surface pressure, tip load) solved on the device (mixed path) against
    the oracle's direct solve of the same problem built from the generator's arrays
    and the oracle's own pressure restatement: 1e-8 relative."""
    import importlib.util
    import os

    from exfem_b200 import deck
    from oracle import loads as oloads
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    spec = importlib.util.spec_from_file_location("make_deck", os.path.join(here, "make_deck.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    ref = mk.case()
    m, steps = deck.read_inp(os.path.join(here, "cantilever_c3d10.inp"))
    import exfem_b200 as xf
    up, _, _ = xf.StaticSolver(m, rtol=1e-6, linear_solver="mixed", cg_tol=1e-10, verbose=False).solve(steps[0])
    X, c = ref["X"], ref["conn"]
    top = np.nonzero(X[:, 2] > 1 - 1e-9)[0]
    f = oloads.pressure_vector(X, oloads.sub_surface(oloads.skin_tet10(X, c), top, len(X)), mk.PRESSURE)
    om = ofem.Model(X)
    om.add_block(c, ofem.TET10, ofem.LinearElastic(mk.E, mk.NU))
    st = osol.Step(bcs=[(ref["fix"], d, 0.0) for d in range(3)], loads=[([ref["tip"]], 2, mk.TIP_LOAD)], dloads=[f])
    uo, _, _ = osol.StaticSolver(om, rtol=1e-6).solve(st)
    assert rel_err(up, uo) < 1e-8


def test_csr_operator_matches_gather_product(cuda):
    """The device-assembled CSR operator (operator="csr") applies the same matrix as
    the element-by-element product of the same element matrices, prescribed DOFs as
    identity rows (gfem/model.py:195-238 against 162-166): one PCG iteration on each
    gives the same iterate to rounding, and J2 Newton counts stay those of the
    oracle on one increment."""
    import exfem_b200 as xf
    from exfem_b200 import linalg
    X, c, bcs, loads, pm, om = _config1()
    blk = pm.blocks[0]
    setup = osol.Setup(om, osol.Step(bcs=bcs, loads=loads))
    blk.set_fixed(setup.fixed)
    Ke = blk.stiffness(torch.zeros(pm.ndof, dtype=torch.float64, device="cuda"), blk.init_state())
    b = torch.as_tensor(np.random.default_rng(1).standard_normal(pm.ndof) * setup.free, device="cuda")
    res = {}
    for op in ("ebe64", "csr64"):
        S = linalg.NativeSolver(blk, op, "jacobi", None, graph=False)
        S.set_ke(Ke)
        res[op] = S.pcg(b, tol=1e-12, maxiter=1)[0]
    assert rel_err(res["csr64"], res["ebe64"]) < 1e-13
    X2, bcs2, om2, uo, so, io, pm2 = _j2_case(1.0)
    up, sp, ip = xf.StaticSolver(pm2, rtol=1e-6, linear_solver="amg", tangent="ebe", cg_tol=1e-10, verbose=False,
                                 operator="csr").solve(xf.Step(bcs=bcs2, dt_init=1.0, dt_max=1.0))
    assert [h[1] for h in ip["history"]] == [h[1] for h in io["history"]]
    assert rel_err(up, uo) < 1e-6


def test_newton_cuts_back_on_nonfinite_residual(cuda):
    """Failure detection on the host (gfem/solvers.py:562-563, 588-594, 663-664): a
    non-finite internal force injected into the first increment's Newton loop makes
    the increment fail and cut back (dt x 0.25), and the step completes with the
    solution of an unfaulted run over the same increments."""
    import exfem_b200 as xf

    class Faulty(xf.StaticSolver):
        calls = 0

        def _fint(self, u, s, fields):
            f, st = super()._fint(u, s, fields)
            Faulty.calls += 1
            if Faulty.calls == 1:
                f = f.clone()
                f[0] = float("nan")
            return f, st

    X, bcs, om, uo, so, io, pm = _j2_case(1.0)
    uf, sf, inf_ = Faulty(pm, rtol=1e-6, linear_solver="mixed", tangent="mf", cg_tol=1e-10,
                          verbose=False).solve(xf.Step(bcs=bcs, dt_init=1.0, dt_max=1.0))
    assert Faulty.calls > 1
    assert inf_["increments"] == len(inf_["history"]) + 1          # one failed increment
    assert inf_["history"][0][0] == 0.25                           # the cutback increment
    X2, bcs2, om2, uo2, so2, io2, pm2 = _j2_case(1.0)
    ur, sr, inr = xf.StaticSolver(pm2, rtol=1e-6, linear_solver="mixed", tangent="mf", cg_tol=1e-10,
                                  verbose=False).solve(xf.Step(bcs=bcs2, dt_init=0.25, dt_max=1.0))
    assert [h[0] for h in inr["history"]] == [h[0] for h in inf_["history"]]
    assert rel_err(uf, ur) < 1e-9


def test_pcg_iteration_limit_reports_not_converged(cuda):
    """PCG that runs out of iterations returns its iterate with the not-converged
    status (a warning in the reference, gfem/solvers.py:472-473), not an error."""
    from exfem_b200 import _lib, linalg
    from exfem_b200._lib import lib
    X, c, bcs, loads, pm, om = _config1()
    blk = pm.blocks[0]
    setup = osol.Setup(om, osol.Step(bcs=bcs, loads=loads))
    blk.set_fixed(setup.fixed)
    S = linalg.NativeSolver(blk, "mf64", "jacobi", None)
    b = torch.as_tensor(np.random.default_rng(2).standard_normal(pm.ndof) * setup.free, device="cuda")
    x, k, rr = S.pcg(b, tol=1e-14, maxiter=3)
    assert k == 3 and rr > 1e-14 and torch.isfinite(x).all()
    import ctypes as C
    xo = torch.empty_like(b)
    kk, r2 = C.c_int(), C.c_double()
    st = lib.exfem_solver_pcg(S._h, _lib.ptr(b), _lib.ptr(xo), 1e-14, 3, C.byref(kk), C.byref(r2), _lib.stream_ptr())
    assert st == _lib.NOT_CONVERGED and kk.value == 3


@pytest.mark.parametrize("operator", ["mf", "stored"])
def test_modal_lobpcg_matches_sparse_eigensolver(cuda, operator):
    """Modal analysis (gfem/eigen.py:32-124) of the clamped config-1 steel cantilever:
    the four lowest w^2 by LOBPCG on the device operators (matrix-free stiffness
    column by column, or the stored element matrices on 16 columns per product;
    HRZ-lumped mass, device AMG preconditioner) against SciPy's shift-invert Lanczos
    on the oracle's assembled stiffness and lumped mass (free DOFs): 1e-7 relative;
    each mode's residual ||K phi - w^2 M phi|| small and the modes M-orthonormal."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    import exfem_b200 as xf
    from exfem_b200 import eigen, mesh
    X, c = mesh.box_hex(100.0, 20.0, 20.0, 20, 4, 4)
    fix = mesh.nodes_where(X, lambda x, y, z: x < 1e-9)
    bcs = [(fix, d, 0.0) for d in range(3)]
    rho = 7.85e-9
    pm = xf.Model(X)
    pm.add_block(c, xf.HEX8, xf.LinearElastic(E, NU, density=rho))
    w2, modes = eigen.modal_lobpcg(pm, xf.Step(bcs=bcs), 4, tol=1e-8, operator=operator)
    om = ofem.Model(X)
    om.add_block(c, ofem.HEX8, ofem.LinearElastic(E, NU, density=rho))
    ops = [(d, K.numpy()) for d, K in om.stiffness_ops(torch.zeros(om.ndof, dtype=torch.float64), om.init_state())]
    Kf = ofem.ops_assemble(ops, om.ndof).tocsr()
    Mf = ofem.lumped_mass(om)
    setup = osol.Setup(om, osol.Step(bcs=bcs))
    free = np.nonzero(setup.free > 0)[0]
    lam, _ = spla.eigsh(Kf[free][:, free], k=4, M=sp.diags(Mf[free]), sigma=0.0, which="LM")
    lam = np.sort(lam)
    np.testing.assert_allclose(w2, lam, rtol=1e-7)
    Phi = modes.cpu().numpy()
    for j in range(4):
        r = Kf @ Phi[j] - w2[j] * Mf * Phi[j]
        assert np.linalg.norm(r[free]) <= 1e-6 * w2[j] * np.linalg.norm(Mf * Phi[j])
    G = (Phi * Mf[None, :]) @ Phi.T
    np.testing.assert_allclose(G, np.eye(4), atol=1e-8)


def test_result_frame_written_for_a_solution(cuda, tmp_path):
    """Output of a device solution (deck output of served requests): displacement,
    von Mises and PEEQ of the config-1 cantilever written to .vtu hold the solver's
    values and the element stresses the oracle computes for the same displacement."""
    import base64
    import xml.etree.ElementTree as ET

    import exfem_b200 as xf
    from exfem_b200 import results
    X, c, bcs, loads, pm, om = _config1()
    u, states, _ = xf.StaticSolver(pm, rtol=1e-6, linear_solver="amg", cg_tol=1e-10, verbose=False).solve(
        xf.Step(bcs=bcs, loads=loads))
    results.write_frame(tmp_path / "r.vtu", pm, u, states)
    arrays = {}
    for da in ET.parse(tmp_path / "r.vtu").getroot().iter("DataArray"):
        raw = base64.b64decode(da.text)
        n = int(np.frombuffer(raw[:8], np.uint64)[0])
        if da.get("type") == "Float64":
            arrays[da.get("Name")] = np.frombuffer(raw[8:8 + n], np.float64)
    np.testing.assert_array_equal(arrays["U"], u.cpu().numpy())
    mo = om.stresses(torch.as_tensor(u.cpu()), om.init_state())[0]["MISES"]
    assert rel_err(arrays["MISES"], mo) < 1e-10
    assert np.all(arrays["PEEQ"] == 0.0)


@pytest.mark.parametrize("tangent", ["ebe", "mf"])
def test_cheby_solver_matches_oracle(cuda, tangent):
    """linear_solver="cheby" (gfem/solvers.py:289-306, 328-342): the config-1
    cantilever against the oracle's direct solution (1e-8), the device power-iteration
    bound against the oracle's on the same assembled operator (1e-10), and one
    preconditioner application against the oracle's polynomial (1e-12)."""
    import exfem_b200 as xf
    from exfem_b200 import linalg, mesh
    X, c = mesh.box_hex(100.0, 20.0, 20.0, 20, 4, 4)
    _, tip, bcs, loads = cantilever_bcs(X, 100.0)
    om = ofem.Model(X)
    om.add_block(c, ofem.HEX8, ofem.LinearElastic(E, NU))
    uo, _, _ = osol.StaticSolver(om, rtol=1e-6).solve(osol.Step(bcs=bcs, loads=loads))
    pm = xf.Model(X)
    pm.add_block(c, xf.HEX8, xf.LinearElastic(E, NU))
    s = xf.StaticSolver(pm, rtol=1e-6, linear_solver="cheby", tangent=tangent, cg_tol=1e-11, verbose=False)
    up, _, _ = s.solve(xf.Step(bcs=bcs, loads=loads))
    assert rel_err(up, uo) < 1e-8, rel_err(up, uo)
    # the bound and the polynomial on the assembled operator
    setup = osol.Setup(om, osol.Step(bcs=bcs, loads=loads))
    ops = [(d, K.numpy()) for d, K in om.stiffness_ops(torch.zeros(om.ndof, dtype=torch.float64), om.init_state())]
    A = olin.bc_matrix(ofem.ops_assemble(ops, om.ndof), setup.free).tocsr()
    dg = A.diagonal()
    dinv = np.where(setup.free > 0, 1.0 / np.where(np.abs(dg) > 0, dg, 1.0), 1.0)
    lo = olin.cheby_lmax(lambda v: A @ v, dinv, setup.free)
    blk = pm.blocks[0]
    blk.set_fixed(setup.fixed)
    S = linalg.NativeSolver(blk, "mf64", "cheby", None, graph=False)
    r = np.random.default_rng(5).standard_normal(pm.ndof) * setup.free
    _, k, _ = S.pcg(torch.as_tensor(r, device="cuda"), tol=1e-30, maxiter=1)
    assert abs(S.cheby_bound() - lo) <= 1e-10 * lo, (S.cheby_bound(), lo)
    assert k == 1


def test_background_hierarchy_set_up(cuda):
    """The "amg" solver with the background set-up forced on (threshold below the
    model size): the first linear solves run Chebyshev-Jacobi PCG while the
    hierarchy is set up on another stream, later ones use it; the Newton solution
    matches the oracle (1e-8) and equals the foreground set-up's to the solver
    tolerance."""
    import time as _time

    import exfem_b200 as xf
    from exfem_b200 import mesh
    X, c = jittered_box(100.0, 20.0, 20.0, 20, 4, 4, frac=0.1, seed=8)
    _, _, bcs, loads = cantilever_bcs(X, 100.0)
    om = ofem.Model(X)
    om.add_block(c, ofem.HEX8, ofem.LinearElastic(E, NU))
    uo, _, _ = osol.StaticSolver(om, rtol=1e-6).solve(osol.Step(bcs=bcs, loads=loads))
    pm = xf.Model(X)
    pm.add_block(c, xf.HEX8, xf.LinearElastic(E, NU))
    s = xf.StaticSolver(pm, rtol=1e-6, linear_solver="amg", cg_tol=1e-11, verbose=False, async_amg=1000)
    up, _, _ = s.solve(xf.Step(bcs=bcs, loads=loads))
    assert rel_err(up, uo) < 1e-8
    t0 = _time.time()
    while s.lin._amg_future is not None and not s.lin._amg_future.done() and _time.time() - t0 < 60:
        _time.sleep(0.05)
    s.lin._collect_background_build()
    assert s.lin.amg is not None and s.lin.amg.nlevels >= 2
    x = s.lin.solve(s.m.stiffness_ops(torch.zeros(pm.ndof, dtype=torch.float64, device="cuda"), pm.init_state()),
                    torch.as_tensor(s.setup.group, device="cuda") * s.setup.free, s.setup)
    assert rel_err(x, uo) < 1e-8


@pytest.mark.parametrize("kind", ["hex", "tet"])
def test_geometric_stiffness_matches_oracle(cuda, kind):
    """Initial-stress stiffness of every element under a random symmetric Cauchy
    stress (gfem/model.py:113-117) against the oracle's: 1e-12 relative."""
    import exfem_b200 as xf
    X, c = jittered_box(2.0, 1.0, 1.0, 3, 2, 2, frac=0.1, seed=9)
    et, oet = xf.HEX8, ofem.HEX8
    if kind == "tet":
        X, c = tet10_box(2.0, 1.0, 1.0, 3, 2, 2, frac=0.1, seed=9)
        et, oet = xf.TET10, ofem.TET10
    S = np.random.default_rng(3).standard_normal((len(c), 3, 3))
    S = S + S.transpose(0, 2, 1)
    pm = xf.Model(X)
    pm.add_block(c, et, xf.LinearElastic(E, NU))
    om = ofem.Model(X)
    om.add_block(c, oet, ofem.LinearElastic(E, NU))
    kp = pm.geometric_ops([dict(S=torch.as_tensor(S, device="cuda"))])[0][1]
    ko = om.geometric_ops([dict(S=torch.as_tensor(S))])[0][1]
    assert rel_err(kp, ko) < 1e-12, rel_err(kp, ko)


def test_buckling_matches_oracle(cuda):
    """Linear buckling of a clamped slender column under a unit compressive tip load
    (gfem/solvers.py:1074-1110 with the device LOBPCG of gfem/eigen.py:137-151):
    the two lowest load factors (the square section buckles alike in y and z)
    against the oracle's: base response by a direct solve, element stresses,
    K0 and KG from the oracle's element matrices, and SciPy's Lanczos on
    -KG phi = mu K0 phi (the reference's small-model path): 1e-6 relative."""
    import scipy.sparse.linalg as spla

    import exfem_b200 as xf
    from exfem_b200 import eigen, mesh
    L = 20.0
    X, c = mesh.box_hex(L, 1.0, 1.0, 20, 2, 2)
    fix = mesh.nodes_where(X, lambda x, y, z: x < 1e-9)
    tip = mesh.nodes_where(X, lambda x, y, z: x > L - 1e-9)
    bcs = [(fix, d, 0.0) for d in range(3)]
    loads = [(tip, 0, -1.0 / len(tip))]
    pm = xf.Model(X)
    pm.add_block(c, xf.HEX8, xf.LinearElastic(E, NU))
    lam, modes = eigen.buckling(pm, xf.Step(bcs=bcs, loads=loads), 2, tol=1e-9)
    om = ofem.Model(X)
    om.add_block(c, ofem.HEX8, ofem.LinearElastic(E, NU))
    uo, so, _ = osol.StaticSolver(om, rtol=1e-9).solve(osol.Step(bcs=bcs, loads=loads))
    stress = om.stresses(torch.as_tensor(uo), so)
    zero = torch.zeros(om.ndof, dtype=torch.float64)
    K0 = ofem.ops_assemble([(d, K.numpy()) for d, K in om.stiffness_ops(zero, om.init_state())], om.ndof).tocsr()
    KG = ofem.ops_assemble([(d, K.numpy()) for d, K in om.geometric_ops(stress)], om.ndof).tocsr()
    setup = osol.Setup(om, osol.Step(bcs=bcs))
    free = np.nonzero(setup.free > 0)[0]
    K0f, KGf = K0[free][:, free].tocsc(), KG[free][:, free].tocsc()
    lu = spla.splu(K0f)
    mu = spla.eigsh(-KGf, k=4, M=K0f, Minv=spla.LinearOperator(K0f.shape, matvec=lu.solve), which="LA",
                    return_eigenvectors=False)
    ref = np.sort(1.0 / mu[mu > 0])[:2]
    np.testing.assert_allclose(lam[:2], ref, rtol=1e-6)
    # Euler's clamped-free column, P_cr = pi^2 E I / (4 L^2): the coarse trilinear
    # mesh (two elements through the section) is stiffer in bending, not wrong by more
    euler = np.pi ** 2 * E * (1.0 / 12) / (4 * L * L)
    assert euler < lam[0] < 1.5 * euler, (lam[0], euler)
