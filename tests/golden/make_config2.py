"""Oracle fixture of the J2 Newton case at full size (test infrastructure).

The C3D8 cantilever of 100 x 20 x 20 elements on a 1000 x 200 x 200 mm box
(44,541 nodes, 133,623 DOF), interior nodes jittered +-10% of the element size
(seed 0), J2 plasticity E = 210 GPa, nu = 0.3, yield 250 MPa, linear hardening
H = 1 GPa, x = 0 clamped, tip -z displacement ramped to 5 mm in 10 increments,
Newton rtol 1e-6, solved by the CPU oracle's Newton procedure (oracle/solvers.py,
the reference's gfem/solvers.py:481-683 with exact sparse-direct linear solves;
SuperLU with the MMD ordering of A^T + A, which takes about 100 s per factorisation
here where COLAMD takes far longer).  About an hour on 8 cores:

    python tests/golden/make_config2.py

Writes ``tests/golden/config2_j2_oracle.npz``: the per-increment Newton counts and
residual-ratio histories, the final displacement, the element von Mises stress and
PEEQ, and a digest of the mesh so the test can confirm it rebuilt the same one.
"""
import hashlib
import os
import sys
import time

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def config2_mesh(nx=100, ny=20, nz=20, seed=0):
    from exfem_b200 import mesh
    L, h = 1000.0, 1000.0 / nx
    X, c = mesh.box_hex(L, 200.0, 200.0, nx, ny, nz)
    X = mesh.jitter_interior(X, [h, 200.0 / ny, 200.0 / nz], 0.1, seed)
    fix = mesh.nodes_where(X, lambda x, y, z: x < 1e-9)
    tip = mesh.nodes_where(X, lambda x, y, z: x > L - 1e-9)
    bcs = [(fix, d, 0.0) for d in range(3)] + [(tip, 2, -5.0)]
    return X, c, bcs


def digest(X, c):
    return hashlib.sha256(np.ascontiguousarray(X).tobytes() + np.ascontiguousarray(c, dtype=np.int64).tobytes()
                          ).hexdigest()


class _Recorder:
    def __init__(self):
        self.hist = []


def main():
    from oracle import fem as ofem
    from oracle import solvers as osol
    torch.set_num_threads(os.cpu_count())
    X, c, bcs = config2_mesh()
    om = ofem.Model(X)
    om.add_block(c, ofem.HEX8, ofem.J2Plasticity(210000.0, 0.3, [[250.0, 0.0], [1250.0, 1.0]]))
    sol = osol.StaticSolver(om, rtol=1e-6, log=lambda s: print(s, flush=True), permc_spec="MMD_AT_PLUS_A")
    ratios = []
    newton = sol._newton

    def recording_newton(*a, **k):
        out = newton(*a, **k)
        ratios.append(np.asarray(out[4], float))
        return out
    sol._newton = recording_newton
    t0 = time.time()
    u, st, info = sol.solve(osol.Step(bcs=bcs, dt_init=0.1, dt_max=0.1))
    print("solved in", time.time() - t0, "s", [h[1] for h in info["history"]], flush=True)
    stress = om.stresses(torch.as_tensor(u), st)[0]
    width = max(len(r) for r in ratios)
    hist = np.full((len(ratios), width), np.nan)
    for i, r in enumerate(ratios):
        hist[i, :len(r)] = r
    np.savez_compressed(os.path.join(HERE, "config2_j2_oracle.npz"),
                        newton=np.array([h[1] for h in info["history"]], np.int64),
                        times=np.array([h[0] for h in info["history"]]), ratios=hist,
                        u=np.asarray(u), mises=stress["MISES"].numpy(), peeq=stress["PEEQ"].numpy(),
                        mesh_digest=np.array(digest(X, c)))


if __name__ == "__main__":
    main()
