"""The J2 Newton case at full size against the oracle (tests/golden/config2_j2_oracle.npz,
made by tests/golden/make_config2.py with the CPU oracle's Newton procedure and exact
sparse-direct linear solves): C3D8 cantilever of 100 x 20 x 20 elements (133,623 DOF),
interior nodes jittered, J2 with linear hardening, tip -5 mm in 10 increments, Newton
rtol 1e-6.  The device solves its linear systems to 1e-12 so that its Newton iterates
follow the oracle's exact ones: the Newton corrections of every increment must be the
same, the displacements agree to 1e-8 and the von Mises stresses to 1e-7 (relative to
the largest)."""
import hashlib
import os

import numpy as np
import pytest
import torch

from helpers import rel_err

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "config2_j2_oracle.npz")


def _mesh():
    from exfem_b200 import mesh
    nx, ny, nz, L = 100, 20, 20, 1000.0
    X, c = mesh.box_hex(L, 200.0, 200.0, nx, ny, nz)
    X = mesh.jitter_interior(X, [L / nx, 200.0 / ny, 200.0 / nz], 0.1, 0)
    fix = mesh.nodes_where(X, lambda x, y, z: x < 1e-9)
    tip = mesh.nodes_where(X, lambda x, y, z: x > L - 1e-9)
    return X, c, [(fix, d, 0.0) for d in range(3)] + [(tip, 2, -5.0)]


@pytest.mark.parametrize("method,tangent", [("amg", "ebe"), ("mixed", "mf")])
def test_config2_newton_matches_oracle(cuda, method, tangent):
    import exfem_b200 as xf
    ref = np.load(FIXTURE)
    X, c, bcs = _mesh()
    digest = hashlib.sha256(np.ascontiguousarray(X).tobytes() +
                            np.ascontiguousarray(c, dtype=np.int64).tobytes()).hexdigest()
    assert digest == str(ref["mesh_digest"]), "the mesh differs from the one the fixture was made on"
    m = xf.Model(X)
    m.add_block(c, xf.HEX8, xf.J2Plasticity(210000.0, 0.3, [[250.0, 0.0], [1250.0, 1.0]]))
    s = xf.StaticSolver(m, rtol=1e-6, linear_solver=method, tangent=tangent, cg_tol=1e-12, verbose=False)
    u, st, info = s.solve(xf.Step(bcs=bcs, dt_init=0.1, dt_max=0.1))
    counts = [int(h[1]) for h in info["history"]]
    assert counts == [int(k) for k in ref["newton"]], (counts, ref["newton"])
    assert rel_err(u, ref["u"]) < 1e-8, rel_err(u, ref["u"])
    out = m.stresses(u, st)[0]
    assert rel_err(out["MISES"], ref["mises"]) < 1e-7, rel_err(out["MISES"], ref["mises"])
    assert rel_err(out["PEEQ"], ref["peeq"]) < 1e-6, rel_err(out["PEEQ"], ref["peeq"])
