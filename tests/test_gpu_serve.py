"""Served request stream on the device: every result against the oracle (a sparse
direct FP64 solve of the oracle's element matrices) to 1e-8, and the same request
alone and inside a mix of concurrent requests on other meshes (bit-identical: every
reduction of the path has a fixed order)."""
import numpy as np
import pytest
import torch

from exfem_b200 import batch, elements, linalg, mesh, serve
from exfem_b200.materials import J2Plasticity, LinearElastic
from exfem_b200.solvers import Step

pytestmark = pytest.mark.gpu


def _linear_spec(key, n, etype, E, nu):
    p = batch.cantilever(*n, 5.0, LinearElastic(E, nu), [[0.0, 0.0, -500.0]], etype=etype)
    return serve.MeshSpec(key, p.X, p.conn, etype, p.material, p.fixed), p.rhs[0]


def _j2_spec(key):
    X, c = mesh.box_hex(40.0, 10.0, 10.0, 8, 2, 2)
    fix = mesh.nodes_where(X, lambda x, y, z: x < 1e-9)
    tip = mesh.nodes_where(X, lambda x, y, z: x > 40.0 - 1e-9)
    fixed = np.zeros(3 * len(X), bool)
    for d in range(3):
        fixed[3 * fix + d] = True
    mat = J2Plasticity(210e3, 0.3, [[250.0, 0.0], [1250.0, 1.0]])
    step = Step(bcs=[(fix, d, 0.0) for d in range(3)] + [(tip, 2, -0.6)], dt_init=0.2, dt_max=0.2)
    return serve.MeshSpec(key, X, c, elements.HEX8, mat, fixed), step


def _direct(spec, rhs):
    from test_gpu_batch import oracle_direct
    return oracle_direct(spec.X, spec.conn, spec.etype.name, spec.material.E, spec.material.nu, spec.fixed, rhs)


def _mix():
    reqs = []
    for i, (n, et, E, nu) in enumerate([((10, 3, 2), elements.HEX8, 210e3, 0.3),
                                        ((3, 2, 2), elements.TET10, 70e3, 0.33),
                                        ((16, 4, 3), elements.HEX8, 120e3, 0.27),
                                        ((6, 2, 2), elements.TET10, 95e3, 0.35)]):
        spec, rhs = _linear_spec(f"lin{i}", n, et, E, nu)
        for s in (1.0, -0.5, 2.0):
            reqs.append((spec, rhs * s))
    return reqs


def test_served_results_match_direct_and_alone(cuda):
    reqs = _mix()
    j2spec, step = _j2_spec("j2")
    # residual tolerance 1e-10: the displacement error of these cantilevers stays
    # below 1e-8 (condition numbers up to ~1e5)
    with serve.SolveServer(slots=4, setup_workers=0, tol=1e-10) as srv:
        futs = [srv.submit(serve.SolveRequest(sp, rhs=r)) for sp, r in reqs]
        futs.append(srv.submit(serve.SolveRequest(j2spec, step=step)))
        out = [f.result(timeout=600) for f in futs]
        st = serve.latency_stats(srv.completed)
        assert st["n"] == len(reqs) + 1
        # requests ran concurrently on several slots
        assert len({r.info["slot"] for r in srv.completed}) > 1
    for (sp, r), (x, info) in zip(reqs, out[:-1]):
        xd = _direct(sp, r)
        assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-8, (np.linalg.norm(x - xd) / np.linalg.norm(xd), info)
    assert out[-1][1]["increments"] >= 3
    # the same requests alone (one slot, nothing else on the server)
    for k in (0, 7, 11):
        sp, r = reqs[k]
        with serve.SolveServer(slots=1, setup_workers=0, tol=1e-10) as srv:
            xa, _ = srv.submit(serve.SolveRequest(sp, rhs=r)).result(timeout=600)
        np.testing.assert_array_equal(xa, out[k][0])
    with serve.SolveServer(slots=1, setup_workers=0) as srv:
        ua, _ = srv.submit(serve.SolveRequest(j2spec, step=step)).result(timeout=600)
    np.testing.assert_array_equal(ua, out[-1][0])


def test_c_abi_request_queue(cuda):
    """The request queue of the C ABI (exfem_queue_*), as a host that is not Python
    drives it: right-hand sides for two resident mixed-solver handles submitted,
    polled, waited for and collected, one request withdrawn before it starts; every
    result equals the same handle's direct mixed solve bit for bit, and to 1e-8 the
    oracle's direct solution."""
    import ctypes as C

    from exfem_b200 import _lib
    from exfem_b200._lib import lib
    from exfem_b200.model import Block
    specs = [_linear_spec("q0", (12, 3, 2), elements.HEX8, 210e3, 0.3),
             _linear_spec("q1", (4, 2, 2), elements.TET10, 95e3, 0.35)]
    solvers = []
    for sp, _ in specs:
        blk = Block(sp.conn, sp.etype, sp.material, X=sp.X)
        blk.set_fixed(sp.fixed)
        Ke = blk.stiffness(torch.zeros(sp.ndof, dtype=torch.float64, device="cuda"), blk.init_state())
        amg = linalg.DeviceAMG(blk, Ke)
        solvers.append((blk, amg, linalg.NativeSolver(blk, "mf32", "amg", amg)))
    q = C.c_void_p()
    assert lib.exfem_queue_create(2, C.byref(q)) == _lib.OK
    got = {}
    try:
        ids, want = [], []
        for k in range(6):
            (sp, rhs), (_, _, ns) = specs[k % 2], solvers[k % 2]
            b = np.ascontiguousarray(rhs * (1.0 + 0.5 * k))
            i = C.c_int64()
            assert lib.exfem_queue_submit(q, ns._h, b.ctypes.data, 1e-10, C.byref(i)) == _lib.OK, _lib.last_error()
            ids.append(i.value)
            want.append((sp, b))
        wd = C.c_int()
        assert lib.exfem_queue_cancel(q, ids[5], C.byref(wd)) == _lib.OK
        for k, i in enumerate(ids):
            st = C.c_int()
            assert lib.exfem_queue_wait(q, i, 120.0, C.byref(st)) == _lib.OK
            if k == 5 and wd.value:
                assert st.value == _lib.REQ_CANCELLED
                assert lib.exfem_queue_result(q, i, None, None, None, None) == _lib.ERR_ARG
                continue
            assert st.value == _lib.REQ_DONE, (k, st.value, _lib.last_error())
            sp, b = want[k]
            x = np.empty(sp.ndof)
            it, ps, rr = C.c_int(), C.c_int(), C.c_double()
            assert lib.exfem_queue_result(q, i, x.ctypes.data, C.byref(it), C.byref(ps), C.byref(rr)) == _lib.OK
            assert rr.value <= 1e-10 and it.value > 0
            got[k] = x
        st = C.c_int()
        assert lib.exfem_queue_poll(q, ids[0], C.byref(st), None, None) == _lib.ERR_ARG     # already collected
    finally:
        assert lib.exfem_queue_destroy(q) == _lib.OK
    # the handles are free again once the queue is gone: direct solves to compare with
    for k, x in got.items():
        sp, b = want[k]
        xd, _, _, _ = solvers[k % 2][2].mixed(torch.as_tensor(b, device="cuda"), tol=1e-10)
        np.testing.assert_array_equal(x, xd.cpu().numpy())
        xo = _direct(sp, b)
        assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-8
