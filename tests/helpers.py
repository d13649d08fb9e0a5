"""Shared builders for the tests: meshes, loads and small comparisons."""
import numpy as np

from exfem_b200 import mesh


def rel_err(a, b):
    a = np.asarray(a.detach().cpu() if hasattr(a, "detach") else a, dtype=np.float64)
    b = np.asarray(b.detach().cpu() if hasattr(b, "detach") else b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def jittered_box(L, H, W, nx, ny, nz, frac=0.1, seed=0):
    X, c = mesh.box_hex(L, H, W, nx, ny, nz)
    h = np.array([L / nx, H / ny, W / nz])
    return mesh.jitter_interior(X, h, frac, seed), c


def tet10_box(L, H, W, nx, ny, nz, frac=0.1, seed=0):
    X, c = jittered_box(L, H, W, nx, ny, nz, frac, seed)
    return mesh.tet4_to_tet10(*mesh.hex_to_tet4(X, c))


def cantilever_bcs(X, L, load=-1000.0, dof=2):
    """x=0 clamped, total ``load`` along ``dof`` split over the x=L nodes (config 1)."""
    fix = mesh.nodes_where(X, lambda x, y, z: x < 1e-9)
    tip = mesh.nodes_where(X, lambda x, y, z: x > L - 1e-9)
    bcs = [(fix, d, 0.0) for d in range(3)]
    loads = [(tip, dof, load / len(tip))]
    return fix, tip, bcs, loads


def smooth_field(X, amp, seed=0):
    """A smooth nodal displacement field with a random linear part (for kernel tests)."""
    rng = np.random.default_rng(seed)
    G = rng.uniform(-1, 1, size=(3, 3)) * amp
    Xc = X - X.mean(0)
    u = Xc @ G.T + 0.2 * amp * np.sin(3.0 * Xc / max(np.ptp(X), 1e-30)) * np.ptp(X)
    return u.reshape(-1)
