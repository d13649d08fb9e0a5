"""Models of several element blocks on the device solver path (gfem/model.py:466-486:
the reference's Model is a list of blocks; its gather plan, gfem/model.py:241-261,
and its assembled tangent cover all of them): two materials on one C3D8 mesh, a
mixed C3D8 + C3D10 mesh, an elastic block beside a J2 block through Newton, a
multi-section input deck, several load cases and modal analysis — each against the
oracle (sparse direct FP64 solves of the oracle's own element matrices)."""
import numpy as np
import pytest
import torch

from helpers import rel_err
from oracle import fem as ofem
from oracle import solvers as osol

pytestmark = pytest.mark.gpu

STEEL, ALU = (210000.0, 0.3), (70000.0, 0.33)


def _two_material_mesh():
    from exfem_b200 import mesh
    X, c = mesh.box_hex(100.0, 20.0, 20.0, 20, 4, 4)
    X = mesh.jitter_interior(X, [5.0, 5.0, 5.0], 0.1, 4)
    left = X[c].mean(1)[:, 0] < 50.0
    return X, [c[left], c[~left]]


def _mixed_mesh():
    """C3D8 for x < 50, Kuhn-split C3D10 for x > 50, sharing the corner nodes at x = 50."""
    from exfem_b200 import mesh
    X, c = mesh.box_hex(100.0, 20.0, 20.0, 10, 2, 2)
    X = mesh.jitter_interior(X, [10.0, 10.0, 10.0], 0.1, 5)
    left = X[c].mean(1)[:, 0] < 50.0
    X10, c10 = mesh.tet4_to_tet10(*mesh.hex_to_tet4(X, c[~left]))
    return X10, c[left], c10


def _cantilever_step(X, L=100.0, load=-1000.0):
    from exfem_b200 import mesh
    fix = mesh.nodes_where(X, lambda x, y, z: x < 1e-9)
    tip = mesh.nodes_where(X, lambda x, y, z: x > L - 1e-9)
    return [(fix, d, 0.0) for d in range(3)], [(tip, 2, load / len(tip))]


@pytest.mark.parametrize("method,tangent,operator", [("amg", "ebe", "gather"), ("amg", "mf", "gather"),
                                                     ("mixed", "mf", "gather"), ("amg", "ebe", "csr"),
                                                     ("jacobi", "ebe", "gather")])
def test_two_material_model_matches_oracle(cuda, method, tangent, operator):
    import exfem_b200 as xf
    X, (ca, cb) = _two_material_mesh()
    bcs, loads = _cantilever_step(X)
    om = ofem.Model(X)
    om.add_block(ca, ofem.HEX8, ofem.LinearElastic(*STEEL))
    om.add_block(cb, ofem.HEX8, ofem.LinearElastic(*ALU))
    uo, _, _ = osol.StaticSolver(om, rtol=1e-6).solve(osol.Step(bcs=bcs, loads=loads))
    pm = xf.Model(X)
    pm.add_block(ca, xf.HEX8, xf.LinearElastic(*STEEL))
    pm.add_block(cb, xf.HEX8, xf.LinearElastic(*ALU))
    np.testing.assert_array_equal(pm.gather(), ofem.gather_plan([ca, cb], len(X)))
    up, _, _ = xf.StaticSolver(pm, rtol=1e-6, linear_solver=method, tangent=tangent, operator=operator,
                               cg_tol=1e-11, verbose=False).solve(xf.Step(bcs=bcs, loads=loads))
    assert rel_err(up, uo) < 1e-8, rel_err(up, uo)


@pytest.mark.parametrize("method,tangent,setup", [("amg", "ebe", "device"), ("mixed", "mf", "device"),
                                                  ("amg", "ebe", "host")])
def test_mixed_element_model_matches_oracle(cuda, method, tangent, setup):
    import exfem_b200 as xf
    X, ch, ct = _mixed_mesh()
    bcs, loads = _cantilever_step(X)
    om = ofem.Model(X)
    om.add_block(ch, ofem.HEX8, ofem.LinearElastic(*STEEL))
    om.add_block(ct, ofem.TET10, ofem.LinearElastic(*STEEL))
    uo, _, _ = osol.StaticSolver(om, rtol=1e-6).solve(osol.Step(bcs=bcs, loads=loads))
    pm = xf.Model(X)
    pm.add_block(ch, xf.HEX8, xf.LinearElastic(*STEEL))
    pm.add_block(ct, xf.TET10, xf.LinearElastic(*STEEL))
    up, _, _ = xf.StaticSolver(pm, rtol=1e-6, linear_solver=method, tangent=tangent, cg_tol=1e-11, verbose=False,
                               amg_setup=setup).solve(xf.Step(bcs=bcs, loads=loads))
    assert rel_err(up, uo) < 1e-8, rel_err(up, uo)
    # element quantities of both blocks against the oracle's
    so = om.stresses(torch.as_tensor(uo), om.init_state())
    sp = pm.stresses(up, pm.init_state())
    for a, b in zip(sp, so):
        assert rel_err(a["MISES"], b["MISES"]) < 1e-7


def test_elastic_and_j2_blocks_newton_matches_oracle(cuda):
    """A J2 block at the clamped end and an elastic block beyond it, one increment
    from the virgin state (so every Newton iterate is decided by the arithmetic):
    Newton counts equal, displacements and von Mises to the Newton tolerance."""
    import exfem_b200 as xf
    from exfem_b200 import mesh
    X, c = mesh.box_hex(100.0, 20.0, 20.0, 10, 2, 2)
    X = mesh.jitter_interior(X, [10.0, 10.0, 10.0], 0.1, 6)
    near = X[c].mean(1)[:, 0] < 30.0
    fix = mesh.nodes_where(X, lambda x, y, z: x < 1e-9)
    tip = mesh.nodes_where(X, lambda x, y, z: x > 100.0 - 1e-9)
    bcs = [(fix, d, 0.0) for d in range(3)] + [(tip, 2, -1.5)]
    table = [[250.0, 0.0], [1250.0, 1.0]]
    om = ofem.Model(X)
    om.add_block(c[near], ofem.HEX8, ofem.J2Plasticity(*STEEL, table))
    om.add_block(c[~near], ofem.HEX8, ofem.LinearElastic(*STEEL))
    uo, so, io = osol.StaticSolver(om, rtol=1e-6).solve(osol.Step(bcs=bcs))
    assert float(so[0][..., 9].max()) > 0                     # the J2 block yielded
    for method, tangent in (("amg", "ebe"), ("mixed", "mf")):
        pm = xf.Model(X)
        pm.add_block(c[near], xf.HEX8, xf.J2Plasticity(*STEEL, table))
        pm.add_block(c[~near], xf.HEX8, xf.LinearElastic(*STEEL))
        up, sp, ip = xf.StaticSolver(pm, rtol=1e-6, linear_solver=method, tangent=tangent, cg_tol=1e-11,
                                     verbose=False).solve(xf.Step(bcs=bcs))
        assert [h[1] for h in ip["history"]] == [h[1] for h in io["history"]], (method, ip["history"], io["history"])
        assert rel_err(up, uo) < 1e-6
        mo = om.stresses(torch.as_tensor(uo), so)
        mp = pm.stresses(up, sp)
        for a, b in zip(mp, mo):
            assert rel_err(a["MISES"], b["MISES"]) < 1e-5


def test_multi_block_device_newton_matches_host_loop(cuda):
    """The device Newton increment over a J2 block and an elastic block (forces,
    tangent products and states summed block by block) against the host loop, over
    four increments so that the J2 block carries plastic history: the same Newton
    counts, displacements and states to the Newton tolerance."""
    import exfem_b200 as xf
    from exfem_b200 import mesh
    X, c = mesh.box_hex(100.0, 20.0, 20.0, 10, 2, 2)
    X = mesh.jitter_interior(X, [10.0, 10.0, 10.0], 0.1, 6)
    near = X[c].mean(1)[:, 0] < 30.0
    fix = mesh.nodes_where(X, lambda x, y, z: x < 1e-9)
    tip = mesh.nodes_where(X, lambda x, y, z: x > 100.0 - 1e-9)
    bcs = [(fix, d, 0.0) for d in range(3)] + [(tip, 2, -1.5)]
    table = [[250.0, 0.0], [1250.0, 1.0]]
    out = {}
    for device in (False, True):
        pm = xf.Model(X)
        pm.add_block(c[near], xf.HEX8, xf.J2Plasticity(*STEEL, table))
        pm.add_block(c[~near], xf.HEX8, xf.LinearElastic(*STEEL))
        sv = xf.StaticSolver(pm, rtol=1e-6, linear_solver="mixed", tangent="mf", cg_tol=1e-11, verbose=False,
                             device_newton=device)
        assert sv._device_increment_ok() == device
        out[device] = sv.solve(xf.Step(bcs=bcs, dt_init=0.25))
    (uh, sh, ih), (ud, sd, idv) = out[False], out[True]
    assert float(sh[0][..., 9].max()) > 0
    assert [h[1] for h in idv["history"]] == [h[1] for h in ih["history"]], (idv["history"], ih["history"])
    assert rel_err(ud, uh) < 1e-6
    for a, b in zip(sd, sh):
        assert rel_err(a, b) < 1e-5


def _write_two_section_deck(path, X, ca, cb):
    out = ["*HEADING", "two sections, two materials", "*NODE"]
    out += [f"{i + 1}, {X[i, 0]:.17g}, {X[i, 1]:.17g}, {X[i, 2]:.17g}" for i in range(len(X))]
    e = 1
    for name, conn in (("LEFT", ca), ("RIGHT", cb)):
        out.append(f"*ELEMENT, TYPE=C3D8, ELSET={name}")
        for row in conn:
            out.append(f"{e}, " + ", ".join(str(int(n) + 1) for n in row))
            e += 1
    fix = np.nonzero(X[:, 0] < 1e-9)[0] + 1
    tip = np.nonzero(X[:, 0] > 100.0 - 1e-9)[0] + 1
    out.append("*NSET, NSET=FIX")
    out += [", ".join(str(n) for n in fix[i:i + 8]) for i in range(0, len(fix), 8)]
    out.append("*NSET, NSET=TIP")
    out += [", ".join(str(n) for n in tip[i:i + 8]) for i in range(0, len(tip), 8)]
    out += ["*SOLID SECTION, ELSET=LEFT, MATERIAL=STEEL", ",", "*SOLID SECTION, ELSET=RIGHT, MATERIAL=ALU", ",",
            "*MATERIAL, NAME=STEEL", "*ELASTIC", f"{STEEL[0]:g}, {STEEL[1]:g}",
            "*MATERIAL, NAME=ALU", "*ELASTIC", f"{ALU[0]:g}, {ALU[1]:g}",
            "*STEP, NAME=Load", "*STATIC", "1, 1", "*BOUNDARY", "FIX, ENCASTRE", "*CLOAD",
            f"TIP, 3, {-1000.0 / len(tip):.17g}", "*END STEP"]
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")
    return fix - 1, tip - 1


def test_multi_section_deck_solves(cuda, tmp_path):
    """An input deck with two element sets, each with its own section and material,
    becomes a two-block model that the device solvers solve (against the oracle)."""
    import exfem_b200 as xf
    from exfem_b200 import deck
    X, (ca, cb) = _two_material_mesh()
    path = str(tmp_path / "two_sections.inp")
    fix, tip = _write_two_section_deck(path, X, ca, cb)
    m, steps = deck.read_inp(path)
    assert len(m.blocks) == 2
    up, _, _ = xf.StaticSolver(m, rtol=1e-6, linear_solver="mixed", cg_tol=1e-11, verbose=False).solve(steps[0])
    om = ofem.Model(X)
    om.add_block(ca, ofem.HEX8, ofem.LinearElastic(*STEEL))
    om.add_block(cb, ofem.HEX8, ofem.LinearElastic(*ALU))
    st = osol.Step(bcs=[(fix, d, 0.0) for d in range(3)], loads=[(tip, 2, -1000.0 / len(tip))])
    uo, _, _ = osol.StaticSolver(om, rtol=1e-6).solve(st)
    assert rel_err(up, uo) < 1e-8, rel_err(up, uo)


def test_multi_block_load_cases_and_modes(cuda):
    """optimize.multi_load_cases on a two-material model (both methods) against the
    oracle's direct solves, and the lowest eigenvalue of the model's modal analysis
    against a sparse shift-invert solve of the oracle's stiffness and the lumped mass."""
    import scipy.sparse.linalg as spla

    import exfem_b200 as xf
    from exfem_b200 import eigen, optimize
    from oracle import linalg as olin
    X, (ca, cb) = _two_material_mesh()
    bcs, _ = _cantilever_step(X)
    pm = xf.Model(X)
    pm.add_block(ca, xf.HEX8, xf.LinearElastic(*STEEL))
    pm.add_block(cb, xf.HEX8, xf.LinearElastic(*ALU))
    om = ofem.Model(X)
    om.add_block(ca, ofem.HEX8, ofem.LinearElastic(*STEEL))
    om.add_block(cb, ofem.HEX8, ofem.LinearElastic(*ALU))
    setup = osol.Setup(om, osol.Step(bcs=bcs))
    ops = [(d, K.numpy()) for d, K in om.stiffness_ops(torch.zeros(om.ndof, dtype=torch.float64), om.init_state())]
    A = olin.bc_matrix(ofem.ops_assemble(ops, om.ndof), setup.free).tocsc()
    tip = np.nonzero(X[:, 0] > 100.0 - 1e-9)[0]
    F = np.zeros((3, pm.ndof))
    for k in range(3):
        F[k, 3 * tip + k] = 100.0 / len(tip)
    ref = [spla.spsolve(A, F[k] * setup.free) for k in range(3)]
    for method in ("batch", "jacobi"):
        U = optimize.multi_load_cases(pm, xf.Step(bcs=bcs), F, cg_tol=1e-11, method=method)
        for k in range(3):
            assert rel_err(U[k], ref[k]) < 1e-8, (method, k, rel_err(U[k], ref[k]))
    import scipy.sparse as sp
    w2, _ = eigen.modal_lobpcg(pm, xf.Step(bcs=bcs), 2, tol=1e-9)
    M = ofem.lumped_mass(om)
    free = np.nonzero(setup.free > 0)[0]
    Kf = ofem.ops_assemble(ops, om.ndof).tocsr()[free][:, free]
    lam = np.sort(spla.eigsh(Kf, k=2, M=sp.diags(M[free]), sigma=0.0, which="LM", return_eigenvectors=False))
    np.testing.assert_allclose(w2, lam, rtol=1e-7)
