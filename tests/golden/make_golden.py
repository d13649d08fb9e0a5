"""Generate the committed fixtures from the reference's own source code.

The reference package cannot be imported (``gfem/__init__.py`` imports jax, which
is not installed), but the functions pinned here are NumPy code:

  * ``gfem/mesh.py`` is pure NumPy and is loaded by file path: ``box_hex``
    (mesh.py:5-16), ``hex_to_tet4`` (19-29) and ``tet4_to_tet10`` (32-38), including
    a jittered case (the orientation fix in ``hex_to_tet4`` only fires on distorted
    meshes) -> ``mesh_fixtures.npz``;
  * ``gather_plan`` (gfem/model.py:241-261) is NumPy apart from its final
    ``jnp.asarray``: its definition alone is taken from the module's syntax tree and
    run with NumPy standing in for ``jax.numpy``;
  * ``gfem/surfaces.py`` (``skin``, ``orient_outward``, ``element_face_surface``,
    ``sub_surface``, ``Surface.integrate``) and the NumPy load vectors of
    ``gfem/loads.py`` (``pressure_vector`` 39-51, ``traction_vector`` 54-57) are
    loaded by path with a stand-in ``jax`` module: ``jax.numpy`` is NumPy and
    ``jax.jacfwd`` a complex-step derivative, which ``gfem/elements.py`` uses to
    tabulate shape-function derivatives at import (exact to rounding for the
    polynomial shape functions)  -> ``ref_index_fixtures.npz``.

Run in a container where the reference tree exists:

    python tests/golden/make_golden.py /path/to/reference
"""
import ast
import importlib.util
import os
import sys
import types
from types import SimpleNamespace

import numpy as np


def load_reference_mesh(root):
    path = os.path.join(root, "gfem", "mesh.py")
    spec = importlib.util.spec_from_file_location("_ref_gfem_mesh", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def jitter(X, h, seed, frac=0.3):
    """Interior-only jitter of +-frac h (0.3: large, to trigger negative Kuhn volumes)."""
    X = np.array(X, float)
    lo, hi = X.min(0), X.max(0)
    inner = np.all((X > lo + 1e-9) & (X < hi - 1e-9), axis=1)
    d = np.random.default_rng(seed).uniform(-frac, frac, size=X.shape) * h
    X[inner] += d[inner]
    return X


# ------------------------------------------------------------------ stand-in jax
def _complex_step_jacfwd(f, h=1e-30):
    """d f / d p of a function of one vector argument by the complex step."""
    def jac(p):
        p = np.asarray(p, dtype=float)
        cols = []
        for k in range(p.size):
            q = p.astype(complex)
            q[k] += 1j * h
            cols.append(np.imag(np.asarray(f(q))) / h)
        return np.stack(cols, axis=-1)
    return jac


def _install_fake_jax():
    jax = types.ModuleType("jax")
    jax.numpy = np
    jax.jacfwd = _complex_step_jacfwd
    saved = {k: sys.modules.get(k) for k in ("jax", "jax.numpy")}
    sys.modules["jax"], sys.modules["jax.numpy"] = jax, np
    return saved


def _restore(saved):
    for k, v in saved.items():
        if v is None:
            sys.modules.pop(k, None)
        else:
            sys.modules[k] = v


def load_reference_surfaces(root):
    """gfem.elements, gfem.surfaces and gfem.loads as a stand-in package (by path)."""
    saved = _install_fake_jax()
    try:
        pkg = types.ModuleType("_refgfem")
        pkg.__path__ = [os.path.join(root, "gfem")]
        sys.modules["_refgfem"] = pkg
        mods = {}
        for name in ("elements", "surfaces", "loads"):
            spec = importlib.util.spec_from_file_location(f"_refgfem.{name}", os.path.join(root, "gfem", f"{name}.py"))
            mod = importlib.util.module_from_spec(spec)
            sys.modules[f"_refgfem.{name}"] = mod
            spec.loader.exec_module(mod)
            mods[name] = mod
        return mods
    finally:
        _restore(saved)


def load_reference_gather_plan(root):
    path = os.path.join(root, "gfem", "model.py")
    tree = ast.parse(open(path).read(), path)
    fn = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == "gather_plan"]
    assert len(fn) == 1
    ns = {"np": np, "jnp": np}
    exec(compile(ast.Module(body=fn, type_ignores=[]), path, "exec"), ns)
    return ns["gather_plan"]


# ------------------------------------------------------------------ cases
def index_cases(rm):
    """Meshes of the plan / skin fixtures: (X, [(element type name, conn), ...])."""
    cases = {}
    X, c = rm.box_hex(100.0, 20.0, 20.0, 20, 4, 4)                        # config 1
    cases["c1"] = (X, [("C3D8", c)])
    X, c = rm.box_hex(1.0, 1.0, 1.0, 3, 3, 3)
    Xj = jitter(X, 1 / 3, 11, 0.1)
    Xt, ct = rm.hex_to_tet4(Xj, c)
    X10, c10 = rm.tet4_to_tet10(Xt, ct)
    cases["tet10"] = (X10, [("C3D10", c10)])
    cases["hex"] = (jitter(X, 1 / 3, 12, 0.1), [("C3D8", c)])
    # two C3D8 blocks (two materials) splitting one jittered box
    X, c = rm.box_hex(2.0, 1.0, 1.0, 4, 3, 2)
    X = jitter(X, np.array([0.5, 1 / 3, 0.5]), 13, 0.1)
    left = X[c].mean(1)[:, 0] < 1.0
    cases["two"] = (X, [("C3D8", c[left]), ("C3D8", c[~left])])
    # mixed: C3D8 for x < 1, Kuhn C3D10 for x > 1, sharing the corner nodes at x = 1
    X, c = rm.box_hex(2.0, 1.0, 1.0, 4, 2, 2)
    X = jitter(X, np.array([0.5, 0.5, 0.5]), 14, 0.1)
    left = X[c].mean(1)[:, 0] < 1.0
    Xt, ct = rm.hex_to_tet4(X, c[~left])
    X10, c10 = rm.tet4_to_tet10(Xt, ct)
    cases["mixed"] = (X10, [("C3D8", c[left]), ("C3D10", c10)])
    return cases


def main(root):
    rm = load_reference_mesh(root)
    here = os.path.dirname(os.path.abspath(__file__))
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
    dst = os.path.join(here, "mesh_fixtures.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, {k: v.shape for k, v in out.items()})

    # gather plans, skins, sub-surfaces and load vectors from the reference's code
    plan = load_reference_gather_plan(root)
    ref = load_reference_surfaces(root)
    E = ref["elements"].ELEMENTS
    out = {}
    for name, (X, blocks) in index_cases(rm).items():
        out[f"{name}_X"] = X
        out[f"{name}_nblk"] = np.array(len(blocks))
        for i, (et, c) in enumerate(blocks):
            out[f"{name}_b{i}_etype"] = np.array(et)
            out[f"{name}_b{i}_conn"] = np.asarray(c)
        out[f"{name}_plan"] = np.asarray(plan([c for _, c in blocks], len(X)))
        blks = [SimpleNamespace(conn=np.asarray(c), etype=E[et]) for et, c in blocks]
        sk = ref["surfaces"].skin(X, blks)
        top = np.nonzero(X[:, 2] > X[:, 2].max() - 1e-9)[0]
        sub = ref["surfaces"].sub_surface(sk, top)
        for tag, s in (("skin", sk), ("sub", sub)):
            out[f"{name}_{tag}_types"] = np.array([ft.name for ft, _ in s.groups])
            for g, (ft, f) in enumerate(s.groups):
                out[f"{name}_{tag}_g{g}"] = f
        out[f"{name}_pressure"] = ref["loads"].pressure_vector(X, sub, -1.0)
        out[f"{name}_traction"] = ref["loads"].traction_vector(X, sub, [1.0, 0.5, -0.25])
        w, area, nsum = sk.integrate(X)
        out[f"{name}_skin_w"], out[f"{name}_skin_area"], out[f"{name}_skin_nsum"] = w, np.array(area), nsum
    dst = os.path.join(here, "ref_index_fixtures.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, len(out), "arrays")


if __name__ == "__main__":
    # the reference checkout: argument, EXFEM_REFERENCE_DIR, or "reference" beside this repository
    repo = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    default = os.environ.get("EXFEM_REFERENCE_DIR", os.path.join(os.path.dirname(repo), "reference"))
    main(sys.argv[1] if len(sys.argv) > 1 else default)
