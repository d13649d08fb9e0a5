"""CPU: the oracle pinned to the reference's known-answer tests and to AD checks.

The reference holds no golden vectors; its tests pin the hot path through
analytic solutions (tests/test_verification.py:27-36, 39-52, 66-83) and
cross-solver agreement (tests/test_gpu_paths.py:47-55).  The same checks are run
on the oracle here, plus finite-difference checks of its AD tangents.
"""
import numpy as np
import pytest
import torch

from exfem_b200 import mesh
from helpers import jittered_box, rel_err, smooth_field, tet10_box
from oracle import fem, linalg, solvers

E, NU = 200e3, 0.3


def _uniaxial(mat, et, n=2, tet=False):
    X, c = mesh.box_hex(1, 1, 1, n, n, n)
    if tet:
        X, c = mesh.tet4_to_tet10(*mesh.hex_to_tet4(X, c))
    m = fem.Model(X)
    m.add_block(c, et, mat)
    w = lambda f: mesh.nodes_where(X, f)
    bcs = [(w(lambda x, y, z: x < 1e-9), 0, 0.0), (w(lambda x, y, z: y < 1e-9), 1, 0.0),
           (w(lambda x, y, z: z < 1e-9), 2, 0.0)]
    return m, bcs, w(lambda x, y, z: x > 1 - 1e-9)


@pytest.mark.parametrize("et,tet", [(fem.HEX8, False), (fem.TET10, True)])
def test_patch_linear(et, tet):
    """tests/test_verification.py:27-36."""
    m, bcs, right = _uniaxial(fem.LinearElastic(E, NU), et, tet=tet)
    u, s, info = solvers.StaticSolver(m).solve(solvers.Step(bcs=bcs + [(right, 0, 1e-3)]))
    S = m.stresses(torch.as_tensor(u), s)[0]["S"].numpy()
    assert np.allclose(S[:, 0, 0], E * 1e-3, rtol=1e-6)
    assert np.allclose(S[:, 1, 1], 0, atol=1e-6 * E)
    assert np.allclose(u.reshape(-1, 3)[:, 1].min(), -NU * 1e-3, rtol=1e-6)


def test_j2_uniaxial_hardening():
    """tests/test_verification.py:39-52."""
    sy, H = 250.0, 2000.0
    m, bcs, right = _uniaxial(fem.J2Plasticity(E, NU, [[sy, 0.0], [sy + H * 0.1, 0.1]]), fem.HEX8, n=1)
    u, s, info = solvers.StaticSolver(m).solve(solvers.Step(bcs=bcs + [(right, 0, 0.01)], dt_init=0.1, dt_max=0.1))
    r = m.stresses(torch.as_tensor(u), s)[0]
    sxx = float(r["S"][0, 0, 0])
    eps, ey = 0.01, sy / E
    expected = sy + E * H / (E + H) * (eps - ey)
    assert abs(sxx - expected) / expected < 1e-4
    assert abs(float(r["PEEQ"][0]) - (eps - sxx / E)) < 1e-6


def test_tet10_cantilever_vs_beam_theory():
    """tests/test_verification.py:66-83."""
    L, h = 10.0, 1.0
    X, c = mesh.tet4_to_tet10(*mesh.hex_to_tet4(*mesh.box_hex(L, h, h, 20, 2, 2)))
    m = fem.Model(X)
    m.add_block(c, fem.TET10, fem.LinearElastic(E, NU))
    fix = mesh.nodes_where(X, lambda x, y, z: x < 1e-9)
    tip = mesh.nodes_where(X, lambda x, y, z: x > L - 1e-9)
    st = solvers.Step(bcs=[(fix, d, 0.0) for d in range(3)], loads=[(tip, 1, -1.0 / len(tip))])
    u, s, info = solvers.StaticSolver(m).solve(st)
    I = h ** 4 / 12
    d_beam = L ** 3 / (3 * E * I) + L / (5 / 6 * E / (2 * (1 + NU)) * h * h)
    d = -float(u.reshape(-1, 3)[tip, 1].mean())
    assert abs(d - d_beam) / d_beam < 0.03
    assert abs(info["reactions"].reshape(-1, 3)[:, 1].sum() - 1.0) < 1e-6


@pytest.mark.parametrize("kind", ["hex", "tet"])
@pytest.mark.parametrize("mat_kind", ["el", "j2"])
def test_ad_tangent_vs_finite_differences(kind, mat_kind):
    X, c = jittered_box(4.0, 3.0, 3.0, 2, 2, 2, frac=0.15) if kind == "hex" else tet10_box(2, 2, 2, 1, 1, 1, frac=0.15)
    et = fem.HEX8 if kind == "hex" else fem.TET10
    mat = fem.LinearElastic(210e3, 0.3) if mat_kind == "el" else fem.J2Plasticity(210e3, 0.3, [[250, 0], [1250, 1]], Hk=500.0)
    m = fem.Model(X)
    m.add_block(c, et, mat)
    s0 = m.init_state()
    if mat_kind == "j2":
        _, s0 = m.internal_force(torch.as_tensor(smooth_field(X, 4e-3, seed=3)), s0)
    u = torch.as_tensor(smooth_field(X, 6e-3, seed=2))
    v = torch.as_tensor(np.random.default_rng(1).standard_normal(m.ndof))
    h = 1e-7
    fd = (m.internal_force(u + h * v, s0)[0] - m.internal_force(u - h * v, s0)[0]) / (2 * h)
    jv = m.tangent_jvp(u, s0, v)
    assert rel_err(jv, fd) < 1e-7
    Kv = fem.ops_matvec(m.stiffness_ops(u, s0), v, m.ndof)
    assert rel_err(Kv, jv) < 1e-13


def test_pcg_jacobi_agrees_with_direct():
    """tests/test_gpu_paths.py:47-55 pattern: iterative vs direct on the oracle."""
    X, c = mesh.box_hex(10.0, 1.0, 1.0, 10, 2, 2)
    m = fem.Model(X)
    m.add_block(c, fem.HEX8, fem.LinearElastic(200e3, 0.3))
    fix = mesh.nodes_where(X, lambda x, y, z: x < 1e-9)
    tip = mesh.nodes_where(X, lambda x, y, z: x > 10 - 1e-9)
    free = np.ones(m.ndof)
    for d in range(3):
        free[fix * 3 + d] = 0
    ops = [(d, K.numpy()) for d, K in m.stiffness_ops(torch.zeros(m.ndof, dtype=torch.float64), m.init_state())]
    A = linalg.bc_matrix(fem.ops_assemble(ops, m.ndof), free)
    b = np.zeros(m.ndof)
    b[tip * 3 + 1] = -1.0 / len(tip)
    x0 = linalg.Direct(A).solve(b)
    dinv = 1.0 / A.diagonal()
    x1, k, rr = linalg.pcg(lambda v: A @ v, b, lambda r: dinv * r, tol=1e-12, maxiter=20000)
    assert np.abs(x1 - x0).max() < 1e-7 * np.abs(x0).max()


def test_oracle_gather_plan_matches_brute_force():
    X, c = mesh.box_hex(1, 1, 1, 3, 2, 2)
    plan = fem.gather_plan([c], len(X))
    off = c.size
    for n in range(len(X)):
        slots = sorted(np.nonzero(c.ravel() == n)[0].tolist())
        row = plan[n]
        assert row[:len(slots)].tolist() == slots and np.all(row[len(slots):] == off)


def test_oracle_colouring_is_proper():
    X, c = tet10_box(1, 1, 1, 3, 3, 3)
    col = fem.greedy_colouring(c, len(X))
    for k in range(col.max() + 1):
        nodes = c[col == k].ravel()
        assert len(nodes) == len(np.unique(nodes))


def test_oracle_mesh_matches_reference_fixtures():
    """The oracle's restatement of gfem/mesh.py (the CPU reference arm's mesh source)
    against the reference's own output, bit for bit, and its node jitter against the
    product's (both build the benchmark meshes)."""
    import os

    import numpy as np

    from exfem_b200 import mesh as pmesh
    from oracle import mesh as omesh
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mesh_fixtures.npz"))
    for name, args in {"c1": (100.0, 20.0, 20.0, 20, 4, 4), "small": (1.0, 1.0, 1.0, 2, 3, 4),
                       "cant": (10.0, 1.0, 1.0, 20, 2, 2)}.items():
        X, c = omesh.box_hex(*args)
        np.testing.assert_array_equal(X, z[f"{name}_hex_X"])
        np.testing.assert_array_equal(c, z[f"{name}_hex_conn"])
    _, c = omesh.box_hex(1.0, 1.0, 1.0, 3, 3, 3)
    for name in ("t", "tj"):
        Xt, t4 = omesh.hex_to_tet4(z[f"{name}_hexX"], c)
        np.testing.assert_array_equal(t4, z[f"{name}_tet4"])
        X10, c10 = omesh.tet4_to_tet10(Xt, t4)
        np.testing.assert_array_equal(X10, z[f"{name}_X10"])
        np.testing.assert_array_equal(c10, z[f"{name}_tet10"])
    X, c = omesh.box_hex(1.0, 1.0, 1.0, 6, 5, 4)
    np.testing.assert_array_equal(omesh.jitter_interior(X, [1 / 6, 1 / 5, 1 / 4], 0.1, 9),
                                  pmesh.jitter_interior(X, [1 / 6, 1 / 5, 1 / 4], 0.1, 9))


def test_config2_fixture_describes_this_mesh():
    """The full-size J2 fixture was made on the mesh the GPU test rebuilds (digest of
    the jittered 100 x 20 x 20 C3D8 cantilever), and holds a Newton history that
    converged: ten increments, each residual-ratio history ending below rtol 1e-6."""
    import hashlib
    import os
    ref = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "config2_j2_oracle.npz"))
    L = 1000.0
    X, c = mesh.box_hex(L, 200.0, 200.0, 100, 20, 20)
    X = mesh.jitter_interior(X, [L / 100, 200.0 / 20, 200.0 / 20], 0.1, 0)
    digest = hashlib.sha256(np.ascontiguousarray(X).tobytes() +
                            np.ascontiguousarray(c, dtype=np.int64).tobytes()).hexdigest()
    assert digest == str(ref["mesh_digest"])
    assert ref["newton"].shape == (10,) and ref["u"].shape == (3 * len(X),)
    assert ref["mises"].shape == (len(c),) and np.all(np.isfinite(ref["u"]))
    tip = X[:, 0] > L - 1e-9
    assert np.allclose(ref["u"].reshape(-1, 3)[tip, 2], -5.0)
    for row in ref["ratios"]:
        assert row[np.isfinite(row)][-1] < 1e-6
