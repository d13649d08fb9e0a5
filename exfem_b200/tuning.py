"""Autotuner of the matrix-free product's tile size, per element type.

The tile size (elements per tile: 128 or 256) is fixed when a block is created
(``exfem_set_tile``, process-wide per element type): larger tiles share more
nodes between elements (fewer node-list entries, less partial-sum traffic) but
hold more shared memory per CTA (fewer resident CTAs).  Which wins depends on the
element type and the device, so :func:`autotune` measures it: for each element
type it builds a representative jittered box mesh with each candidate tile size,
times the FP32 product with CUDA events and keeps the fastest.  Results are kept
per (device name, element type) for the process and applied with
``exfem_set_tile``; :func:`apply` sets a known choice without measuring.
No counterpart in the reference.
"""
import ctypes as C

import numpy as np
import torch

from . import _lib, elements, mesh
from ._lib import check, lib
from .materials import LinearElastic
from .model import Block

CANDIDATES = (128, 256)
_cache = {}


def current(etype):
    t = C.c_int()
    check(lib.exfem_get_tile(etype.code, C.byref(t)))
    return t.value


def apply(etype, tile):
    check(lib.exfem_set_tile(etype.code, int(tile)))


def _mesh(etype, n):
    X, c = mesh.box_hex(1.0, 1.0, 1.0, n, n, n)
    X = mesh.jitter_interior(X, 1.0 / n, 0.1, 0)
    if etype.name == "C3D10":
        X, c = mesh.tet4_to_tet10(*mesh.hex_to_tet4(X, c))
    return X, c


def _time_product(blk, ndof, reps):
    v = torch.randn(ndof, dtype=torch.float32, device="cuda", generator=torch.Generator("cuda").manual_seed(0))
    y = torch.empty_like(v)
    s = torch.cuda.current_stream()
    run = lambda: check(lib.exfem_tangent_matvec(blk.handle, _lib.F32, v.data_ptr(), y.data_ptr(), 1, s.cuda_stream))
    for _ in range(3):
        run()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        run()
    e1.record(s)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def autotune(etypes=(elements.HEX8, elements.TET10), n=None, reps=20, candidates=CANDIDATES, verbose=False):
    """Measure every candidate tile size per element type and apply the fastest.
    n: hexahedra per edge of the test cube (default: about 1M elements, larger
    than L2).  Returns {element type name: (tile, {tile: ms})}."""
    _lib.require_cuda()
    dev = torch.cuda.get_device_name()
    out = {}
    for et in etypes:
        key = (dev, et.name)
        if key not in _cache:
            nn_ = n or (100 if et.name == "C3D8" else 56)
            X, c = _mesh(et, nn_)
            fixed = np.zeros(3 * len(X), bool)
            fixed[: 3 * (nn_ + 1) ** 2] = True                   # one clamped face
            saved = current(et)
            times = {}
            try:
                for tile in candidates:
                    apply(et, tile)
                    blk = Block(c, et, LinearElastic(1000.0, 0.3), X=X)
                    blk.set_fixed(fixed)
                    times[tile] = _time_product(blk, 3 * len(X), reps)
                    del blk
            finally:
                apply(et, saved)
            _cache[key] = (min(times, key=times.get), times)
            if verbose:
                print(f"autotune {et.name}: {times} -> tile {_cache[key][0]}", flush=True)
        tile, times = _cache[key]
        apply(et, tile)
        out[et.name] = (tile, times)
    return out
