"""Checkpoint / resume of a static analysis between increments.

The reference keeps no solver checkpoint; its ``State`` carries the displacement,
the material states, the external force and the time from one step to the next
(gfem/solvers.py:83-95, 601-604).  ``save`` writes exactly those (from a
``StaticSolver.solve`` callback or the state after a step) to one compressed NumPy
archive; ``load`` returns them as device tensors, ready for
``StaticSolver.solve(step, u0=..., states=..., fext0=...)``.
"""
import numpy as np
import torch


def _host(t):
    return t.detach().cpu().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)


def save(path, u, states, time=0.0, fext=None, **meta):
    """Write u (ndof,), the per-block material states and optional fext (ndof,) with
    the analysis time and scalar metadata."""
    arrays = {"u": _host(u), "time": np.float64(time), "nblocks": np.int64(len(states))}
    for i, s in enumerate(states):
        arrays[f"state_{i}"] = _host(s)
    if fext is not None:
        arrays["fext"] = _host(fext)
    for k, v in meta.items():
        arrays[f"meta_{k}"] = np.asarray(v)
    np.savez_compressed(path, **arrays)


def load(path, device="cuda"):
    """(u, states, time, fext or None, metadata dict) of a checkpoint; tensors on
    ``device``."""
    with np.load(path) as f:
        u = torch.as_tensor(f["u"], device=device)
        states = [torch.as_tensor(f[f"state_{i}"], device=device) for i in range(int(f["nblocks"]))]
        fext = torch.as_tensor(f["fext"], device=device) if "fext" in f.files else None
        meta = {k[5:]: f[k][()] for k in f.files if k.startswith("meta_")}
        return u, states, float(f["time"]), fext, meta


def callback(path_pattern):
    """A ``StaticSolver.solve`` callback writing one checkpoint per converged
    increment: ``path_pattern`` formatted with the increment count and time."""
    count = {"n": 0}

    def cb(t, u, states):
        count["n"] += 1
        save(path_pattern.format(inc=count["n"], t=t), u, states, time=t, increment=count["n"])
    return cb
