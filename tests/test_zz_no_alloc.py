"""The allocation-free V-cycle entry point, called through the C ABI.

``exfem_amg_vcycle_noalloc`` serves callers that must not allocate device memory
during a call (code recording a CUDA graph by stream capture, hosts whose device
memory belongs to another allocator).  It must give the same result as
``exfem_amg_vcycle`` on two calls in a row (the second call reuses the static
scratch the first one left behind), in FP64 and FP32, with and without the
matrix-free level-0 operator, and must reject a hierarchy too large for its
static scratch with a clear error.  The same holds on a hierarchy set up on the
device; one set up without its mesh-level matrix is refused, before any launch,
when no level-0 block is given.  A call on a hierarchy it has not seen before
leaves the device's free memory unchanged.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = a.double().cpu().numpy(), b.double().cpu().numpy()
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _model():
    import exfem_b200 as xf
    from exfem_b200 import mesh
    X, c = mesh.box_hex(100.0, 20.0, 20.0, 20, 4, 4)
    m = xf.Model(X)
    m.add_block(c, xf.HEX8, xf.LinearElastic(210000.0, 0.3))
    fixed = np.zeros(m.ndof, bool)
    fix = mesh.nodes_where(X, lambda x, y, z: x < 1e-9)
    for d in range(3):
        fixed[fix * 3 + d] = True
    return m, X, fixed


def _hierarchy():
    from exfem_b200 import linalg
    m, X, fixed = _model()
    ops = m.stiffness_ops(torch.zeros(m.ndof, dtype=torch.float64, device="cuda"), m.init_state())
    A = linalg.bc_matrix(linalg.ops_assemble(ops, m.ndof), (~fixed).astype(float))
    return m, fixed, linalg.AMG(A, X)


def _device_hierarchy(keep_level0):
    """Hierarchy set up on the GPU (the set-up the solvers use by default)."""
    from exfem_b200 import linalg
    m, X, fixed = _model()
    blk = m.blocks[0]
    blk.set_fixed(fixed)
    Ke = blk.stiffness(torch.zeros(m.ndof, dtype=torch.float64, device="cuda"), blk.init_state())
    return m, fixed, linalg.DeviceAMG(blk, Ke, keep_level0=keep_level0)


def _call(amg, r, z, level0=None, dinv0=None):
    from exfem_b200 import _lib
    code = _lib.F64 if r.dtype == torch.float64 else _lib.F32
    return _lib.lib.exfem_amg_vcycle_noalloc(amg.handle, code, r.data_ptr(), z.data_ptr(),
                                             level0.handle if level0 is not None else None,
                                             dinv0.data_ptr() if dinv0 is not None else None,
                                             torch.cuda.current_stream().cuda_stream)


def _noalloc(amg, r, level0=None, dinv0=None):
    from exfem_b200 import _lib
    z = torch.empty_like(r)
    st = _call(amg, r, z, level0, dinv0)
    assert st == _lib.OK, _lib.last_error()
    return z


def _dinv0(blk, fixed, dtype=torch.float64):
    d = blk.tangent_diagonal()
    return torch.where(torch.as_tensor(fixed, device="cuda"), torch.ones_like(d), 1.0 / d).to(dtype)


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 1e-6)])
def test_noalloc_vcycle_matches_vcycle_twice(cuda, dtype, tol):
    m, fixed, amg = _hierarchy()
    rng = np.random.default_rng(0)
    for call in range(2):
        r = torch.as_tensor(rng.standard_normal(m.ndof) * (~fixed), dtype=dtype, device="cuda")
        z_ref = amg.vcycle(r)
        z = _noalloc(amg, r)
        torch.cuda.synchronize()
        assert _rel(z, z_ref) < tol, (call, _rel(z, z_ref))


def test_noalloc_vcycle_matrix_free_level0(cuda):
    m, fixed, amg = _hierarchy()
    blk = m.blocks[0]
    blk.set_fixed(fixed)
    dinv0 = _dinv0(blk, fixed)
    rng = np.random.default_rng(1)
    for call in range(2):
        r = torch.as_tensor(rng.standard_normal(m.ndof) * (~fixed), device="cuda")
        z_ref = amg.vcycle(r, blk, dinv0)
        z = _noalloc(amg, r, blk, dinv0)
        torch.cuda.synchronize()
        assert _rel(z, z_ref) < 1e-12, (call, _rel(z, z_ref))
    blk.set_fixed(None)


def test_noalloc_vcycle_rejects_oversized_hierarchy(cuda):
    from exfem_b200 import _lib
    n = 400_000                                 # 6 FP64 level vectors alone need 19.2 MB
    ptr = np.arange(n + 1, dtype=np.int64)
    idx = np.arange(n, dtype=np.int32)
    one = np.ones(n)
    pptr = np.arange(n + 1, dtype=np.int64)
    pidx = np.zeros(n, dtype=np.int32)
    rptr = np.array([0, n], dtype=np.int64)
    h = C.c_void_p()
    assert _lib.lib.exfem_amg_create(C.byref(h)) == _lib.OK
    try:
        assert _lib.lib.exfem_amg_add_level(h, n, 1, ptr.ctypes.data, idx.ctypes.data, one.ctypes.data,
                                            pptr.ctypes.data, pidx.ctypes.data, one.ctypes.data,
                                            rptr.ctypes.data, idx.ctypes.data, one.ctypes.data,
                                            one.ctypes.data, 1.1) == _lib.OK
        ainv = np.ones(1)
        assert _lib.lib.exfem_amg_set_coarse(h, 1, ainv.ctypes.data) == _lib.OK
        r = torch.ones(n, dtype=torch.float64, device="cuda")
        z = torch.empty_like(r)
        st = _lib.lib.exfem_amg_vcycle_noalloc(h, _lib.F64, r.data_ptr(), z.data_ptr(), None, None,
                                               torch.cuda.current_stream().cuda_stream)
        assert st == _lib.ERR_ARG
        assert "static scratch" in _lib.last_error()
    finally:
        _lib.lib.exfem_amg_destroy(h)


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 1e-6)])
def test_noalloc_vcycle_device_hierarchy_twice(cuda, dtype, tol):
    """A hierarchy set up on the GPU with its mesh-level matrix kept: stored level 0
    and matrix-free level 0, two calls in a row each."""
    m, fixed, amg = _device_hierarchy(keep_level0=True)
    blk = m.blocks[0]
    dinv0 = _dinv0(blk, fixed, dtype)
    rng = np.random.default_rng(2)
    for call in range(2):
        r = torch.as_tensor(rng.standard_normal(m.ndof) * (~fixed), dtype=dtype, device="cuda")
        for lv0, d0 in ((None, None), (blk, dinv0)):
            z_ref = amg.vcycle(r, lv0, d0)
            z = _noalloc(amg, r, lv0, d0)
            torch.cuda.synchronize()
            assert _rel(z, z_ref) < tol, (call, lv0 is not None, _rel(z, z_ref))


def test_noalloc_vcycle_refuses_level0_without_matrix(cuda):
    """The solvers' default device set-up stores no mesh-level matrix: without a
    level-0 block the call is refused with an argument error (nothing launched, the
    output untouched), as exfem_amg_vcycle refuses it; with the block it runs."""
    from exfem_b200 import _lib
    m, fixed, amg = _device_hierarchy(keep_level0=False)
    assert amg._export(0, 0)[0].nnz == 0                 # level 0 stores no matrix
    r = torch.ones(m.ndof, dtype=torch.float64, device="cuda")
    z = torch.full_like(r, 7.0)
    torch.cuda.synchronize()
    assert _call(amg, r, z) == _lib.ERR_ARG
    assert "no stored matrix" in _lib.last_error()
    torch.cuda.synchronize()
    assert bool(torch.all(z == 7.0))
    blk = m.blocks[0]
    dinv0 = _dinv0(blk, fixed)
    z_ref = amg.vcycle(r * torch.as_tensor(~fixed, device="cuda"), blk, dinv0)
    z = _noalloc(amg, r * torch.as_tensor(~fixed, device="cuda"), blk, dinv0)
    torch.cuda.synchronize()
    assert _rel(z, z_ref) < 1e-12


def test_noalloc_vcycle_leaves_free_memory_unchanged(cuda):
    """The first call on a hierarchy it has not seen allocates nothing: the device's
    free memory is the same before and after it (kernels are loaded by a call on
    another hierarchy first, so module loading does not count)."""
    m, fixed, amg0 = _hierarchy()
    r = torch.as_tensor(np.random.default_rng(3).standard_normal(m.ndof) * (~fixed), device="cuda")
    _noalloc(amg0, r)
    _, _, amg = _hierarchy()
    z = torch.empty_like(r)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    from exfem_b200 import _lib
    assert _call(amg, r, z) == _lib.OK, _lib.last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert _rel(z, amg.vcycle(r)) < 1e-12
