"""Generate the committed mesh fixtures from the reference's own ``gfem/mesh.py``.

The reference package cannot be imported (``gfem/__init__.py`` imports jax, which
is not installed), but ``gfem/mesh.py`` is pure NumPy, so it is loaded by file
path.  Run in a container where the reference tree exists:

    python tests/golden/make_golden.py /path/to/reference

Outputs ``tests/golden/mesh_fixtures.npz``: for each case the node coordinates and
connectivity produced by ``box_hex`` (gfem/mesh.py:5-16), ``hex_to_tet4``
(mesh.py:19-29) and ``tet4_to_tet10`` (mesh.py:32-38), including a jittered case
(the orientation fix in ``hex_to_tet4`` only fires on distorted meshes).
"""
import importlib.util
import os
import sys

import numpy as np


def load_reference_mesh(root):
    path = os.path.join(root, "gfem", "mesh.py")
    spec = importlib.util.spec_from_file_location("_ref_gfem_mesh", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def jitter(X, h, seed):
    """Interior-only jitter of +-0.3 h (large, to trigger negative Kuhn volumes)."""
    X = np.array(X, float)
    lo, hi = X.min(0), X.max(0)
    inner = np.all((X > lo + 1e-9) & (X < hi - 1e-9), axis=1)
    d = np.random.default_rng(seed).uniform(-0.3, 0.3, size=X.shape) * h
    X[inner] += d[inner]
    return X


def main(root):
    rm = load_reference_mesh(root)
    out = {}
    cases = {"c1": (100.0, 20.0, 20.0, 20, 4, 4), "small": (1.0, 1.0, 1.0, 2, 3, 4),
             "cant": (10.0, 1.0, 1.0, 20, 2, 2)}
    for name, args in cases.items():
        X, c = rm.box_hex(*args)
        out[f"{name}_hex_X"], out[f"{name}_hex_conn"] = X, c
    X, c = rm.box_hex(1.0, 1.0, 1.0, 3, 3, 3)
    for name, Xh in (("t", X), ("tj", jitter(X, 1 / 3, 7))):
        Xt, ct = rm.hex_to_tet4(Xh, c)
        X10, c10 = rm.tet4_to_tet10(Xt, ct)
        out[f"{name}_hexX"], out[f"{name}_tet4"] = Xh, ct
        out[f"{name}_X10"], out[f"{name}_tet10"] = X10, c10
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mesh_fixtures.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    # the reference checkout: argument, EXFEM_REFERENCE_DIR, or "reference" beside this repository
    repo = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    default = os.environ.get("EXFEM_REFERENCE_DIR", os.path.join(os.path.dirname(repo), "reference"))
    main(sys.argv[1] if len(sys.argv) > 1 else default)
