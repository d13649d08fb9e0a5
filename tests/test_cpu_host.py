"""CPU: mesh fixtures, host index builders through the C ABI, exported symbols,
host smoothed-aggregation set-up, and the world-size-2 replicas path (gloo)."""
import ctypes as C
import json
import os
import re
import subprocess
import sys

import numpy as np
import pytest
import scipy.sparse as sp

from exfem_b200 import _lib, linalg, mesh
from helpers import tet10_box
from oracle import fem

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "mesh_fixtures.npz")


def test_mesh_generators_match_reference_fixtures():
    """Fixtures produced by the reference's gfem/mesh.py (tests/golden/make_golden.py)."""
    g = np.load(GOLDEN)
    cases = {"c1": (100.0, 20.0, 20.0, 20, 4, 4), "small": (1.0, 1.0, 1.0, 2, 3, 4), "cant": (10.0, 1.0, 1.0, 20, 2, 2)}
    for name, args in cases.items():
        X, c = mesh.box_hex(*args)
        np.testing.assert_array_equal(X, g[f"{name}_hex_X"])
        np.testing.assert_array_equal(c, g[f"{name}_hex_conn"])
    for name in ("t", "tj"):
        Xh = g[f"{name}_hexX"]
        _, c = mesh.box_hex(1.0, 1.0, 1.0, 3, 3, 3)
        X4, c4 = mesh.hex_to_tet4(Xh, c)
        np.testing.assert_array_equal(c4, g[f"{name}_tet4"])
        X10, c10 = mesh.tet4_to_tet10(X4, c4)
        np.testing.assert_array_equal(c10, g[f"{name}_tet10"])
        np.testing.assert_array_equal(X10, g[f"{name}_X10"])


def test_library_exports_every_declared_symbol():
    header = open(os.path.join(ROOT, "include", "exfem_b200.h")).read()
    header = re.sub(r"/\*.*?\*/", "", header, flags=re.S)
    names = set(re.findall(r"\bint\s+(exfem_\w+)\s*\(", header)) | set(re.findall(r"\bconst char\*\s+(exfem_\w+)\s*\(", header))
    assert len(names) > 30
    lib = C.CDLL(_lib.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.EXPORTED) <= names


def _host_plan(c, nn):
    c32 = np.ascontiguousarray(c, dtype=np.int32)
    vmax = C.c_int()
    assert _lib.lib.exfem_host_gather_plan(nn, len(c), c.shape[1], c32.ctypes.data, None, C.byref(vmax)) == 0
    plan = np.empty((nn, vmax.value), np.int32)
    assert _lib.lib.exfem_host_gather_plan(nn, len(c), c.shape[1], c32.ctypes.data, plan.ctypes.data, C.byref(vmax)) == 0
    return plan


@pytest.mark.parametrize("kind", ["hex", "tet"])
def test_host_gather_plan_and_colouring_bit_exact(kind):
    if kind == "hex":
        X, c = mesh.box_hex(1, 1, 1, 5, 4, 3)
    else:
        X, c = tet10_box(1, 1, 1, 3, 3, 2)
    np.testing.assert_array_equal(_host_plan(c, len(X)), fem.gather_plan([c], len(X)))
    col = np.empty(len(c), np.int32)
    nc = C.c_int()
    c32 = np.ascontiguousarray(c, dtype=np.int32)
    assert _lib.lib.exfem_host_colouring(len(X), len(c), c.shape[1], c32.ctypes.data, col.ctypes.data, C.byref(nc)) == 0
    np.testing.assert_array_equal(col, fem.greedy_colouring(c, len(X)))
    assert nc.value == col.max() + 1


def _host_order(X, c, ncorner):
    order = np.empty(len(c), np.int32)
    c32 = np.ascontiguousarray(c, dtype=np.int32)
    X = np.ascontiguousarray(X, dtype=np.float64)
    assert _lib.lib.exfem_host_tile_order(len(X), len(c), c.shape[1], ncorner, X.ctypes.data, c32.ctypes.data,
                                          order.ctypes.data) == 0
    return order


@pytest.mark.parametrize("kind", ["hex", "tet", "union"])
def test_host_tile_order_bit_exact(kind):
    """The native Morton tile order equals the oracle's restatement; components
    (here several meshes in one block) stay contiguous."""
    if kind == "hex":
        X, c = mesh.box_hex(1, 1, 1, 9, 5, 4)
        X = mesh.jitter_interior(X, 1.0 / 9, 0.1, 2)
        nc = 8
    elif kind == "tet":
        X, c = tet10_box(1, 1, 1, 4, 3, 3)
        nc = 4
    else:
        X1, c1 = mesh.box_hex(1, 1, 1, 6, 2, 2)
        X2, c2 = mesh.box_hex(2, 1, 1, 3, 3, 1)
        X = np.concatenate([X1, X2, X1])
        c = np.concatenate([c1, c2 + len(X1), c1 + len(X1) + len(X2)])
        nc = 8
    order = _host_order(X, c, nc)
    np.testing.assert_array_equal(order, fem.tile_order(X, c, nc))
    np.testing.assert_array_equal(np.sort(order), np.arange(len(c)))
    if kind == "union":
        n1, n2 = len(c1), len(c2)
        np.testing.assert_array_equal(np.sort(order[:n1]), np.arange(n1))
        np.testing.assert_array_equal(np.sort(order[n1:n1 + n2]), np.arange(n1, n1 + n2))


def test_host_tile_pairs_bit_exact_and_oriented():
    """Face pairs of the C3D10 tile order equal the oracle's restatement; paired
    elements share their face at local corners (0,1,2) <-> (1,0,2), every element
    keeps its node set and stays positively oriented, and mid-nodes follow corners."""
    X, c = tet10_box(1, 1, 1, 4, 3, 3)
    order = _host_order(X, c, 4)
    o, ct = order.copy(), np.empty_like(c, dtype=np.int32)
    c32 = np.ascontiguousarray(c, dtype=np.int32)
    assert _lib.lib.exfem_host_tile_pairs(len(c), c32.ctypes.data, o.ctypes.data, ct.ctypes.data) == 0
    wo, wc = fem.tile_pairs(order, c)
    np.testing.assert_array_equal(o, wo)
    np.testing.assert_array_equal(ct, wc)
    np.testing.assert_array_equal(np.sort(o), np.arange(len(c)))
    for p, e in enumerate(o):
        assert sorted(ct[p]) == sorted(c[e])
        x = X[ct[p, :4]]
        assert np.linalg.det(np.stack([x[1] - x[0], x[2] - x[0], x[3] - x[0]])) > 0
        for k, (a, b) in enumerate([(0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3)]):
            np.testing.assert_allclose(X[ct[p, 4 + k]], 0.5 * (X[ct[p, a]] + X[ct[p, b]]), atol=1e-12)
    paired = sum(ct[2 * j, 0] == ct[2 * j + 1, 1] and ct[2 * j, 1] == ct[2 * j + 1, 0] and ct[2 * j, 2] == ct[2 * j + 1, 2]
                 for j in range(len(c) // 2))
    assert paired >= 0.9 * (len(c) // 2)          # Kuhn tets pair up almost completely


def test_host_gather_plan_rejects_bad_connectivity():
    c = np.array([[0, 1, 2, 3, 4, 5, 6, 99]], np.int32)
    vmax = C.c_int()
    assert _lib.lib.exfem_host_gather_plan(8, 1, 8, c.ctypes.data, None, C.byref(vmax)) == _lib.ERR_ARG
    assert "outside" in _lib.last_error()


def test_standard_aggregation_partitions_the_graph():
    X, c = mesh.box_hex(1, 1, 1, 6, 5, 4)
    rows = np.repeat(c, 8, axis=1).ravel()
    cols = np.tile(c, (1, 8)).ravel()
    S = sp.csr_matrix((np.ones(len(rows)), (rows, cols)), shape=(len(X), len(X)))
    S.sum_duplicates()
    agg, nagg = linalg._aggregate(S)
    assert agg.min() >= 0 and agg.max() == nagg - 1
    assert np.bincount(agg).min() >= 1
    # every aggregate is connected through the graph (a root and its neighbours)
    for a in range(nagg):
        members = np.nonzero(agg == a)[0]
        sub = S[members][:, members]
        ncomp, _ = sp.csgraph.connected_components(sub, directed=False)
        assert ncomp == 1


def test_sa_hierarchy_properties():
    """Host set-up: P interpolates the rigid-body modes at the tentative stage,
    coarse operators are symmetric Galerkin products, sizes shrink to <= 300."""
    import torch
    X, c = mesh.box_hex(10.0, 2.0, 2.0, 12, 3, 3)
    m = fem.Model(X)
    m.add_block(c, fem.HEX8, fem.LinearElastic(200e3, 0.3))
    ops = [(d, K.numpy()) for d, K in m.stiffness_ops(torch.zeros(m.ndof, dtype=torch.float64), m.init_state())]
    free = np.ones(m.ndof)
    fix = mesh.nodes_where(X, lambda x, y, z: x < 1e-9)
    for d in range(3):
        free[fix * 3 + d] = 0
    A = linalg.bc_matrix(fem.ops_assemble(ops, m.ndof), free)
    B = linalg.rigid_body_modes(X)
    levels, Ac = linalg.sa_hierarchy(A, B, 3, 300)
    assert len(levels) >= 1 and Ac.shape[0] <= 300
    for Al, P in levels:
        assert abs(Al - Al.T).max() <= 1e-9 * abs(Al).max()
    S = linalg._strength_graph(A, 3)
    agg, nagg = linalg._aggregate(S)
    T, Bc = linalg._fit_candidates(agg, nagg, B, 3)
    free_nodes = np.nonzero(agg[np.arange(m.ndof) // 3] >= 0)[0]
    np.testing.assert_allclose((T @ Bc)[free_nodes], B[free_nodes], atol=1e-9 * np.abs(B).max())


def test_bench_replicas_world_size_two_gloo(tmp_path):
    """The multi-GPU path is replicas: max-over-ranks timing and rank-0 output.
    Exercised with two gloo ranks on the CPU."""
    code = r'''
import os, torch, torch.distributed as dist
dist.init_process_group("gloo")
r, w = dist.get_rank(), dist.get_world_size()
t = torch.tensor([1.0 + r])
dist.all_reduce(t, op=dist.ReduceOp.MAX)
assert float(t) == float(w)
units = torch.tensor([100.0])
dist.all_reduce(units)
if r == 0:
    print("OK", float(units) / float(t))
dist.destroy_process_group()
'''
    f = tmp_path / "rep.py"
    f.write_text(code)
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT="29571")
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
                        "--master-addr", "127.0.0.1", "--master-port", "29571", str(f)],
                       capture_output=True, text=True, env=env, timeout=300)
    assert "OK 100.0" in r.stdout, r.stderr[-2000:]


def test_batch_host_setups_in_spawned_workers():
    """Per-problem host hierarchies of a batch (element stiffness from the oracle):
    spawned worker processes give the same hierarchy as the in-process set-up, and
    a problem below the coarse size has no level (it is relayed in the union)."""
    import torch
    from exfem_b200 import batch
    from exfem_b200.materials import LinearElastic
    probs = [batch.cantilever(14, 3, 3, 5.0, LinearElastic(150e3, 0.3), [[0, 0, -100.0]]),
             batch.cantilever(2, 1, 1, 5.0, LinearElastic(80e3, 0.3), [[0, 0, -100.0]])]
    stiff = []
    for p in probs:
        m = fem.Model(p.X)
        m.add_block(p.conn, fem.HEX8, fem.LinearElastic(p.material.E, p.material.nu))
        (d, K), = m.stiffness_ops(torch.zeros(m.ndof, dtype=torch.float64), m.init_state())
        stiff.append((np.asarray(d), K.numpy()))
    a = batch.host_setups(probs, workers=0, stiffness=stiff)
    b = batch.host_setups(probs, workers=2, stiffness=stiff)
    assert len(a[0]["levels"]) >= 1 and len(a[1]["levels"]) == 0
    for ha, hb in zip(a, b):
        np.testing.assert_array_equal(ha["coarse_inv"], hb["coarse_inv"])
        for la, lb in zip(ha["levels"], hb["levels"]):
            assert (la["P"] != lb["P"]).nnz == 0 and la["rho"] == lb["rho"]


def test_batch_union_levels_equal_scipy_block_diag():
    """The union level arrays written by shifting each problem's CSR arrays equal
    SciPy's block_diag of the same blocks (canonicalised: summed duplicates, sorted
    indices, explicit zeros kept), for unsorted and duplicated entries, identity
    relays, empty rows and all-zero blocks given by their shape; the transpose
    blocks give the union's transpose."""
    from exfem_b200 import batch
    rng = np.random.default_rng(5)
    blocks = []
    for n, m in ((7, 3), (1, 1), (12, 5), (4, 4), (9, 2)):
        nnz = 3 * n
        r, c = rng.integers(0, n, nnz), rng.integers(0, m, nnz)
        v = rng.standard_normal(nnz)
        v[::5] = 0.0                                         # explicit zeros stay
        o = np.argsort(r, kind="stable")                     # rows in order, columns as drawn
        blocks.append(sp.csr_matrix((v[o], c[o], np.searchsorted(r[o], np.arange(n + 1))), shape=(n, m)))
    blocks.insert(2, sp.identity(3, format="csr"))
    blocks.append(sp.csr_matrix((4, 2)))                     # empty rows
    before = [(B.indptr.copy(), B.indices.copy(), B.data.copy()) for B in blocks]
    ref = sp.block_diag(blocks, format="csr")
    ref.sum_duplicates()
    ref.sort_indices()
    p, i, v = batch._block_diag_csr(blocks)
    for B, (bp, bi, bv) in zip(blocks, before):               # the inputs are left as they were
        assert np.array_equal(B.indptr, bp) and np.array_equal(B.indices, bi) and np.array_equal(B.data, bv)
    assert p.dtype == np.int64 and i.dtype == np.int32 and v.dtype == np.float64
    np.testing.assert_array_equal(p, ref.indptr)
    np.testing.assert_array_equal(i, ref.indices)
    np.testing.assert_array_equal(v, ref.data)
    rt = ref.T.tocsr()
    rt.sort_indices()
    p, i, v = batch._block_diag_csr([B.T for B in blocks])
    np.testing.assert_array_equal(p, rt.indptr)
    np.testing.assert_array_equal(i, rt.indices)
    np.testing.assert_array_equal(v, rt.data)
    p, i, v = batch._block_diag_csr([(3, 3), (2, 2)])
    np.testing.assert_array_equal(p, np.zeros(6, np.int64))
    assert i.size == 0 and v.size == 0


def test_random_cantilevers_follow_the_stated_ranges():
    from exfem_b200 import batch
    probs = batch.random_cantilevers(40, seed=3)
    for p in probs:
        ne = len(p.conn)
        assert 4 * 2 * 2 <= ne <= 64 * 16 * 16
        assert 70e3 <= p.material.E <= 210e3 and 0.25 <= p.material.nu <= 0.35
        assert p.rhs.shape == (4, p.ndof)
        tot = p.rhs.reshape(4, -1, 3).sum(1)
        mags = np.abs(tot).max(1)
        assert np.all((mags >= 100.0) & (mags <= 1000.0))
        np.testing.assert_allclose(np.sign(tot).astype(int), [[1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, -1]])


def test_skin_and_pressure_vector_match_oracle():
    """Config-3 load set-up: skin of a jittered C3D10 box, its z = 1 sub-surface and
    the equivalent nodal forces of a -1 pressure against the oracle's restatement of
    gfem/surfaces.py:182-242 and gfem/loads.py:37-49 (facets bit for bit, forces to
    1e-14 of the largest: the closed-form shape-function derivatives round
    differently from the oracle's AD ones in the last bit); the C3D8 skin
    (QUAD4 facets) against the closed form: a pressure -p on the unit cube's top face
    gives a total force p along +z and nothing else."""
    from types import SimpleNamespace

    from exfem_b200 import elements, loads, mesh, surfaces
    from oracle import loads as oloads
    X, c = tet10_box(1.0, 1.0, 1.0, 3, 3, 3, frac=0.1, seed=7)
    blk = SimpleNamespace(conn=c, etype=elements.TET10)
    top = mesh.nodes_where(X, lambda x, y, z: z > 1 - 1e-9)
    sk = surfaces.skin(X, [blk])
    osk = oloads.skin_tet10(X, c)
    assert len(sk.groups) == 1 and sk.groups[0][0] is surfaces.TRI6
    np.testing.assert_array_equal(sk.groups[0][1], osk)
    sub = surfaces.sub_surface(sk, top)
    osub = oloads.sub_surface(osk, top, len(X))
    np.testing.assert_array_equal(sub.groups[0][1], osub)
    f = loads.pressure_vector(X, sub, -1.0)
    fo = oloads.pressure_vector(X, osub, -1.0)
    np.testing.assert_allclose(f, fo, rtol=0, atol=1e-14 * np.abs(fo).max())
    assert abs(f.reshape(-1, 3)[:, 2].sum() - 1.0) < 1e-12
    Xh, ch = mesh.box_hex(1.0, 1.0, 1.0, 3, 3, 3)
    Xh = mesh.jitter_interior(Xh, [1 / 3] * 3, 0.1, 3)
    skh = surfaces.skin(Xh, [SimpleNamespace(conn=ch, etype=elements.HEX8)])
    assert len(skh) == 6 * 9 and skh.groups[0][0] is surfaces.QUAD4
    toph = mesh.nodes_where(Xh, lambda x, y, z: z > 1 - 1e-9)
    fh = loads.pressure_vector(Xh, surfaces.sub_surface(skh, toph), -2.5).reshape(-1, 3)
    np.testing.assert_allclose(fh.sum(0), [0.0, 0.0, 2.5], atol=1e-12)
    w, area, nsum = skh.integrate(Xh)
    assert abs(area - 6.0) < 1e-12 and np.abs(nsum).max() < 1e-12 and abs(w.sum() - 6.0) < 1e-12
    ft = loads.traction_vector(Xh, surfaces.sub_surface(skh, toph), [1.0, 0.0, 0.0]).reshape(-1, 3)
    np.testing.assert_allclose(ft.sum(0), [1.0, 0.0, 0.0], atol=1e-12)


def test_deck_reader_fixture():
    """Input-deck reader (gfem/io/inp.py semantics) on the committed C3D10 fixture
    (tests/golden/make_deck.py): nodes, connectivity in deck order through the
    labels, generated and listed node sets, the element-face surface, the encastre,
    the concentrated tip load and the pressure vector of the surface against the
    oracle's skin / sub-surface / pressure restatement."""
    import importlib.util

    from exfem_b200 import deck
    from oracle import loads as oloads
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    spec = importlib.util.spec_from_file_location("make_deck", os.path.join(here, "make_deck.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    ref = mk.case()
    d = deck.InpDeck(os.path.join(here, "cantilever_c3d10.inp"))
    np.testing.assert_array_equal(d.X, ref["X"])
    np.testing.assert_array_equal(d.node_ids, ref["node_labels"])
    assert len(d.blocks) == 1 and d.blocks[0]["etype"].name == "C3D10"
    np.testing.assert_array_equal(d.blocks[0]["conn"], ref["conn"])
    np.testing.assert_array_equal(d.blocks[0]["labels"], ref["elem_labels"])
    np.testing.assert_array_equal(np.sort(d.node_indices("FIX")), np.sort(ref["fix"]))
    np.testing.assert_array_equal(d.node_indices("FIRST_NODES"), np.arange(10))
    m = d.blocks[0]["material"]
    assert (m.E, m.nu) == (mk.E, mk.NU)
    (st,) = d.step_objects()
    assert st.name == "Load" and st.T == 1.0 and st.max_inc == 100
    fixed = {(int(n), k) for nodes, k, v in st.bcs for n in nodes if v == 0.0}
    assert fixed == {(int(n), k) for n in ref["fix"] for k in range(3)}
    assert [(list(n), k, v) for n, k, v in st.loads] == [([ref["tip"]], 2, mk.TIP_LOAD)]
    top = np.nonzero(ref["X"][:, 2] > 1 - 1e-9)[0]
    skin = oloads.skin_tet10(ref["X"], ref["conn"])
    fo = oloads.pressure_vector(ref["X"], oloads.sub_surface(skin, top, len(ref["X"])), mk.PRESSURE)
    (f,) = st.dloads
    np.testing.assert_allclose(f, fo, rtol=0, atol=1e-13 * np.abs(fo).max())
    assert abs(f.reshape(-1, 3)[:, 2].sum() - (-mk.PRESSURE) * 4.0) < 1e-12


# the reference checkout (its example decks are read where they lie, when present)
REF_DIR = os.environ.get("EXFEM_REFERENCE_DIR",
                         os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))),
                                      "reference"))


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF_DIR, "examples", "decks")),
                    reason="reference decks not present")
def test_deck_reader_reference_examples():
    """The reference's own static C3D10 example decks parse: node and element counts
    against a plain count of their data lines, one static step each, the bracket's
    concentrated loads and the plate's pressure (total force along +x)."""
    from exfem_b200 import deck
    for name, nload, ndl in (("bracket", 113, 0), ("plate_hole", 0, 1)):
        path = os.path.join(REF_DIR, "examples", "decks", f"{name}.inp")
        counts, card = {"NODE": 0, "ELEMENT": 0}, None
        with open(path) as fh:
            for line in fh:
                s = line.strip()
                if s.startswith("**") or not s:
                    continue
                if s.startswith("*"):
                    card = s[1:].split(",")[0].strip().upper()
                elif card in counts:
                    counts[card] += 1
        d = deck.InpDeck(path)
        assert len(d.X) == counts["NODE"] and sum(len(b["conn"]) for b in d.blocks) == counts["ELEMENT"]
        (st,) = d.step_objects()
        assert len(st.loads) == nload and len(st.dloads) == ndl and len(st.bcs) > 0
        if ndl:
            assert st.dloads[0].reshape(-1, 3).sum(0)[0] > 0


def test_device_setup_host_steps():
    """Host graph steps of the device smoothed-aggregation set-up, checked on CPU:
    the node adjacency against a brute-force set union over the elements, the
    tentative prolongator against the host set-up's NumPy modified Gram-Schmidt
    (linalg._fit_candidates) on a real aggregation of a C3D10 mesh with rigid-body
    modes, and the regularised Cholesky inverse of the coarsest matrix against
    NumPy."""
    X, c = tet10_box(2.0, 1.0, 1.0, 4, 2, 2)
    nn, ne = len(X), len(c)
    conn = np.ascontiguousarray(c, dtype=np.int32)
    nnz, ptr = C.c_int64(), np.zeros(nn + 1, np.int64)
    _lib.check(_lib.lib.exfem_host_node_adjacency(nn, ne, 10, conn.ctypes.data, C.byref(nnz), ptr.ctypes.data, None))
    idx = np.zeros(nnz.value, np.int32)
    _lib.check(_lib.lib.exfem_host_node_adjacency(nn, ne, 10, conn.ctypes.data, C.byref(nnz), ptr.ctypes.data,
                                                  idx.ctypes.data))
    nb = [set() for _ in range(nn)]
    for row in c:
        for a in row:
            nb[a].update(int(b) for b in row)
    for n in range(nn):
        np.testing.assert_array_equal(idx[ptr[n]:ptr[n + 1]], sorted(nb[n] | {n}))
    # aggregation of the adjacency graph, tentative prolongator with rigid-body modes
    agg = np.zeros(nn, np.int32)
    nagg = C.c_int64()
    _lib.check(_lib.lib.exfem_host_standard_aggregation(nn, ptr.ctypes.data, idx.ctypes.data, agg.ctypes.data,
                                                        C.byref(nagg)))
    B = np.ascontiguousarray(linalg.rigid_body_modes(X))
    Q = np.zeros((3 * nn, 6))
    Bc = np.zeros((nagg.value * 6, 6))
    _lib.check(_lib.lib.exfem_host_fit_candidates(nn, 3, 6, agg.ctypes.data, nagg.value, B.ctypes.data, Q.ctypes.data,
                                                  Bc.ctypes.data))
    T, Bc_ref = linalg._fit_candidates(agg, nagg.value, B, 3)
    Qref = np.zeros_like(Q)
    Td = T.tocoo()
    Qref[Td.row, Td.col % 6] = Td.data
    np.testing.assert_allclose(Q, Qref, rtol=0, atol=1e-13)
    np.testing.assert_allclose(Bc, Bc_ref, rtol=0, atol=1e-12 * np.abs(Bc_ref).max())
    # coarsest inverse
    rng = np.random.default_rng(4)
    M = rng.standard_normal((30, 30))
    A = M @ M.T + 30 * np.eye(30)
    Ainv = np.zeros_like(A)
    _lib.check(_lib.lib.exfem_host_coarse_inverse(30, np.ascontiguousarray(A).ctypes.data, Ainv.ctypes.data))
    ref = np.linalg.inv(A + 1e-13 * np.abs(A).max() * np.eye(30))
    np.testing.assert_allclose(Ainv, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


def test_deck_reader_step_semantics(tmp_path):
    """Boundary conditions and loads across steps as the reference reader carries
    them (gfem/io/inp.py:518-616): *INCLUDE, GENERATE sets, DOF ranges with a value,
    symmetry keywords, accumulation from step to step, OP=NEW, a later value of the
    same node and DOF winning, and the static time increments."""
    from exfem_b200 import deck
    nodes = "\n".join(f"{10 + i}, {i % 3}.0, {(i // 3) % 3}.0, {i // 9}.0" for i in range(27))
    (tmp_path / "nodes.inp").write_text("*NODE, NSET=ALLN\n" + nodes + "\n")
    conn = [[0, 1, 4, 3, 9, 10, 13, 12], [1, 2, 5, 4, 10, 11, 14, 13], [3, 4, 7, 6, 12, 13, 16, 15],
            [4, 5, 8, 7, 13, 14, 17, 16], [9, 10, 13, 12, 18, 19, 22, 21], [10, 11, 14, 13, 19, 20, 23, 22],
            [12, 13, 16, 15, 21, 22, 25, 24], [13, 14, 17, 16, 22, 23, 26, 25]]
    elems = "\n".join(f"{100 + e}, " + ", ".join(str(10 + n) for n in row) for e, row in enumerate(conn))
    text = f"""*HEADING
semantics
*INCLUDE, INPUT=nodes.inp
*ELEMENT, TYPE=C3D8R, ELSET=EALL
{elems}
*NSET, NSET=BASE, GENERATE
10, 18, 1
*NSET, NSET=TOPC
36
*SOLID SECTION, ELSET=EALL, MATERIAL=AL
*MATERIAL, NAME=AL
*ELASTIC
70000., 0.33
*PLASTIC
100., 0.
200., 0.5
*BOUNDARY
BASE, ZSYMM
*STEP, NAME=one
*STATIC
0.1, 1., 1e-4, 0.25
*BOUNDARY
10, 1, 2
*CLOAD
TOPC, 3, -1.5
36, 1, 2.0
*END STEP
*STEP, NAME=two
*STATIC
*BOUNDARY
36, 1, 2, 0.25
*CLOAD
TOPC, 3, -3.0
*END STEP
*STEP, NAME=three
*STATIC
*BOUNDARY, OP=NEW
11, 3, 3, 0.5
*CLOAD, OP=NEW
TOPC, 2, 1.0
*END STEP
"""
    path = tmp_path / "sem.inp"
    path.write_text(text)
    d = deck.InpDeck(str(path))
    assert len(d.X) == 27 and len(d.blocks) == 1 and d.blocks[0]["etype"].name == "C3D8"
    m = d.blocks[0]["material"]
    assert type(m).__name__ == "J2Plasticity"
    one, two, three = d.step_objects()
    flat = lambda items: {(int(n), k): v for ns, k, v in items for n in ns}
    base = {(n, 2): 0.0 for n in range(9)}
    assert (one.dt_init, one.T, one.dt_min, one.dt_max) == (0.1, 1.0, 1e-4, 0.25)
    assert flat(one.bcs) == {**base, (0, 0): 0.0, (0, 1): 0.0}
    assert flat(one.loads) == {(26, 2): -1.5, (26, 0): 2.0}
    assert flat(two.bcs) == {**base, (0, 0): 0.0, (0, 1): 0.0, (26, 0): 0.25, (26, 1): 0.25}
    assert flat(two.loads) == {(26, 2): -3.0, (26, 0): 2.0}
    assert flat(three.bcs) == {**base, (1, 2): 0.5}
    assert flat(three.loads) == {(26, 1): 1.0}


@pytest.mark.parametrize("kind", ["hex", "tet"])
def test_lumped_mass_matches_oracle(kind):
    """HRZ-lumped mass of the modal analysis (gfem/model.py:120-124, 501-510) against
    the oracle's restatement on jittered C3D8 and C3D10 meshes: 1e-13 relative, and
    the total equals density x volume."""
    from types import SimpleNamespace

    from exfem_b200 import eigen, elements
    from oracle import fem as ofem
    if kind == "hex":
        X, c = mesh.box_hex(3.0, 1.0, 1.0, 6, 2, 2)
        X = mesh.jitter_interior(X, [0.5, 0.5, 0.5], 0.1, 5)
        pet, oet = elements.HEX8, ofem.HEX8
    else:
        X, c = tet10_box(3.0, 1.0, 1.0, 3, 2, 2)
        pet, oet = elements.TET10, ofem.TET10
    rho = 7.85e-9
    mat = SimpleNamespace(density=rho)
    m = eigen.lumped_mass_host(X, [SimpleNamespace(conn=c, etype=pet, material=mat)])
    om = ofem.Model(X)
    om.add_block(c, oet, ofem.LinearElastic(210e3, 0.3, density=rho))
    mo = ofem.lumped_mass(om)
    np.testing.assert_allclose(m, mo, rtol=1e-13, atol=0)
    assert abs(m.sum() / 3 - rho * 3.0) < 1e-12 * rho * 3.0
    assert (m > 0).all()


def test_checkpoint_roundtrip(tmp_path):
    """Checkpoint / resume data of a static analysis (the reference's State fields,
    gfem/solvers.py:83-95): displacement, per-block material states, external force,
    time and metadata survive a save / load round trip bit for bit, and the
    per-increment callback writes one file per converged increment."""
    import torch

    from exfem_b200 import checkpoint
    rng = np.random.default_rng(0)
    u = torch.as_tensor(rng.standard_normal(30))
    states = [torch.as_tensor(rng.standard_normal((4, 8, 19))), torch.as_tensor(rng.standard_normal((2, 4, 1)))]
    fext = torch.as_tensor(rng.standard_normal(30))
    path = tmp_path / "ck.npz"
    checkpoint.save(path, u, states, time=0.75, fext=fext, increment=3)
    u2, s2, t2, f2, meta = checkpoint.load(path, device="cpu")
    assert torch.equal(u2, u) and all(torch.equal(a, b) for a, b in zip(s2, states)) and torch.equal(f2, fext)
    assert t2 == 0.75 and int(meta["increment"]) == 3 and len(s2) == 2
    cb = checkpoint.callback(str(tmp_path / "inc{inc:03d}.npz"))
    for t in (0.25, 0.5):
        cb(t, u * t, states)
    files = sorted(p.name for p in tmp_path.glob("inc*.npz"))
    assert files == ["inc001.npz", "inc002.npz"]
    u3, _, t3, f3, meta3 = checkpoint.load(tmp_path / "inc002.npz", device="cpu")
    assert t3 == 0.5 and f3 is None and torch.equal(u3, u * 0.5) and int(meta3["increment"]) == 2


def test_vtu_writer_roundtrip(tmp_path):
    """ParaView output (gfem/io/vtk.py:24-71 format): the .vtu of a C3D8 + C3D10
    mesh parses as XML, and every binary DataArray decodes (UInt64 byte count, then
    the values) to the written points, connectivity, offsets, cell types and result
    arrays; the .pvd lists the frames."""
    import base64
    import xml.etree.ElementTree as ET
    from types import SimpleNamespace

    from exfem_b200 import elements, results
    Xh, ch = mesh.box_hex(2.0, 1.0, 1.0, 2, 1, 1)
    X10, c10 = tet10_box(1.0, 1.0, 1.0, 1, 1, 1)
    X = np.vstack([Xh, X10 + [3.0, 0.0, 0.0]])
    blocks = [SimpleNamespace(conn=ch, etype=elements.HEX8),
              SimpleNamespace(conn=c10 + len(Xh), etype=elements.TET10)]
    rng = np.random.default_rng(0)
    U = rng.standard_normal((len(X), 3))
    mises = rng.uniform(0, 300, len(ch) + len(c10))
    path = tmp_path / "f.vtu"
    results.write_vtu(path, X, blocks, point_data={"U": U}, cell_data={"MISES": mises})
    root = ET.parse(path).getroot()
    arrays = {}
    for da in root.iter("DataArray"):
        raw = base64.b64decode(da.text)
        n = int(np.frombuffer(raw[:8], np.uint64)[0])
        dt = {"Float64": np.float64, "Int64": np.int64, "UInt8": np.uint8}[da.get("type")]
        arrays[da.get("Name")] = np.frombuffer(raw[8:8 + n], dt)
    np.testing.assert_array_equal(arrays["Points"].reshape(-1, 3), X)
    np.testing.assert_array_equal(arrays["connectivity"], np.concatenate([ch.ravel(), (c10 + len(Xh)).ravel()]))
    np.testing.assert_array_equal(arrays["offsets"], np.cumsum([8] * len(ch) + [10] * len(c10)))
    np.testing.assert_array_equal(arrays["types"], [12] * len(ch) + [24] * len(c10))
    np.testing.assert_array_equal(arrays["U"].reshape(-1, 3), U)
    np.testing.assert_array_equal(arrays["MISES"], mises)
    piece = next(root.iter("Piece"))
    assert int(piece.get("NumberOfPoints")) == len(X) and int(piece.get("NumberOfCells")) == len(mises)
    results.write_pvd(tmp_path / "s.pvd", [(0.5, "f.vtu"), (1.0, "g.vtu")])
    ds = [d.attrib for d in ET.parse(tmp_path / "s.pvd").getroot().iter("DataSet")]
    assert ds == [{"timestep": "0.5", "file": "f.vtu"}, {"timestep": "1", "file": "g.vtu"}]
    with pytest.raises(ValueError):
        results.write_vtu(tmp_path / "bad.vtu", X, blocks, point_data={"U": U[:-1]})


def test_deck_reader_rejects_what_it_does_not_cover(tmp_path):
    """The deck reader refuses, with a clear error, decks outside the static solid
    path: other element types, dynamic / frequency steps, elements without a section,
    node-based surfaces."""
    from exfem_b200 import deck
    head = "*NODE\n1, 0, 0, 0\n2, 1, 0, 0\n3, 0, 1, 0\n4, 0, 0, 1\n"
    cases = {
        "S4R shell": (head + "*ELEMENT, TYPE=S4R\n1, 1, 2, 3, 4\n", NotImplementedError),
        "frequency": (head + "*ELEMENT, TYPE=C3D4\n1, 1, 2, 3, 4\n", NotImplementedError),
        "no section": (None, ValueError),
        "node surface": (None, NotImplementedError),
    }
    tet10 = ("*NODE\n" + "\n".join(f"{i + 1}, {x}, {y}, {z}" for i, (x, y, z) in enumerate(
        [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (.5, 0, 0), (.5, .5, 0), (0, .5, 0), (0, 0, .5), (.5, 0, .5),
         (0, .5, .5)])) + "\n*ELEMENT, TYPE=C3D10, ELSET=E\n1, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10\n")
    cases["no section"] = (tet10 + "*MATERIAL, NAME=M\n*ELASTIC\n1., 0.3\n", ValueError)
    cases["node surface"] = (tet10 + "*SURFACE, NAME=S, TYPE=NODE\n1, 1.\n", NotImplementedError)
    cases["frequency"] = (tet10 + "*SOLID SECTION, ELSET=E, MATERIAL=M\n*MATERIAL, NAME=M\n*ELASTIC\n1., 0.3\n"
                          "*STEP\n*FREQUENCY\n10\n*END STEP\n", NotImplementedError)
    for name, (text, exc) in cases.items():
        p = tmp_path / f"{name.replace(' ', '_')}.inp"
        p.write_text(text)
        with pytest.raises(exc):
            deck.InpDeck(str(p))


def test_coarse_inverse_singular_and_indefinite():
    """Coarsest solve of the device set-up: a singular positive semidefinite matrix
    (rigid-body null space of a floating structure) still factors through the
    1e-13 max|A| shift, and the regularised inverse solves consistent systems; an
    indefinite matrix is refused with a status instead of a wrong factor."""
    rng = np.random.default_rng(2)
    Bm = rng.standard_normal((12, 9))
    A = Bm @ Bm.T                                        # rank 9 of 12
    Ainv = np.zeros_like(A)
    _lib.check(_lib.lib.exfem_host_coarse_inverse(12, np.ascontiguousarray(A).ctypes.data, Ainv.ctypes.data))
    assert np.isfinite(Ainv).all()
    b = A @ rng.standard_normal(12)                      # in the range of A
    x = Ainv @ b
    assert np.linalg.norm(A @ x - b) < 1e-3 * np.linalg.norm(b)
    Neg = -np.eye(6)
    st = _lib.lib.exfem_host_coarse_inverse(6, np.ascontiguousarray(Neg).ctypes.data, np.zeros((6, 6)).ctypes.data)
    assert st < 0 and "positive definite" in _lib.last_error()


def _ref_fixture_cases():
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_index_fixtures.npz")
    z = np.load(path)
    names = sorted({k.split("_")[0] for k in z.files})
    return z, names


@pytest.mark.parametrize("case", ["c1", "tet10", "hex", "two", "mixed"])
def test_index_maps_and_surfaces_match_reference_output(case):
    """The gather plan (gfem/model.py:241-261) over one or several blocks, the skin
    (gfem/surfaces.py:182-221, with its outward orientation 150-162), the z = max
    sub-surface (234-242), the surface integrals (103-120) and the pressure and
    traction load vectors (gfem/loads.py:39-57), against the output of the
    reference's own code (tests/golden/make_golden.py runs it on these meshes):
    index maps and facet lists bit for bit, load vectors to 1e-14 of the largest
    entry (shape-function derivatives in closed form here, by a complex-step
    derivative there)."""
    from types import SimpleNamespace

    from exfem_b200 import elements, loads, surfaces
    from exfem_b200.model import gather_plan
    z, _ = _ref_fixture_cases()
    X = z[f"{case}_X"]
    conns = [z[f"{case}_b{i}_conn"] for i in range(int(z[f"{case}_nblk"]))]
    ets = [elements.ELEMENTS[str(z[f"{case}_b{i}_etype"])] for i in range(len(conns))]
    np.testing.assert_array_equal(gather_plan(conns, len(X)), z[f"{case}_plan"])
    blocks = [SimpleNamespace(conn=c, etype=et) for c, et in zip(conns, ets)]
    sk = surfaces.skin(X, blocks)
    top = np.nonzero(X[:, 2] > X[:, 2].max() - 1e-9)[0]
    sub = surfaces.sub_surface(sk, top)
    for tag, s in (("skin", sk), ("sub", sub)):
        assert [ft.name for ft, _ in s.groups] == list(z[f"{case}_{tag}_types"])
        for g, (_, f) in enumerate(s.groups):
            np.testing.assert_array_equal(f, z[f"{case}_{tag}_g{g}"])
    for name, got in (("pressure", loads.pressure_vector(X, sub, -1.0)),
                      ("traction", loads.traction_vector(X, sub, [1.0, 0.5, -0.25]))):
        ref = z[f"{case}_{name}"]
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-14 * np.abs(ref).max())
    w, area, nsum = sk.integrate(X)
    np.testing.assert_allclose(w, z[f"{case}_skin_w"], rtol=0, atol=1e-14 * np.abs(z[f"{case}_skin_w"]).max())
    assert abs(area - float(z[f"{case}_skin_area"])) <= 1e-13 * area
    np.testing.assert_allclose(nsum, z[f"{case}_skin_nsum"], rtol=0, atol=1e-12 * area)


def test_face_hash_counts_shared_keys():
    """exfem_host_face_once: a key that occurs once is flagged, twice or more not."""
    keys = np.array([[-1, 0, 1, 2], [0, 1, 2, 3], [-1, 0, 1, 2], [-1, 0, 1, 3], [-1, 0, 1, 2]], np.int64)
    once = np.zeros(len(keys), np.uint8)
    assert _lib.lib.exfem_host_face_once(len(keys), keys.ctypes.data, once.ctypes.data) == 0
    np.testing.assert_array_equal(once, [0, 1, 0, 1, 0])


def _host_tile_maps(conn, nn, tile):
    c32 = np.ascontiguousarray(conn, dtype=np.int32)
    nt, nl = C.c_int64(), C.c_int64()
    args = [nn, len(c32), c32.shape[1], c32.ctypes.data, tile, C.byref(nt), C.byref(nl)]
    assert _lib.lib.exfem_host_tile_maps(*args, None, None, None, None) == 0, _lib.last_error()
    ptr = np.zeros(nt.value + 1, np.int32)
    nodes = np.zeros(max(nl.value, 1), np.int32)
    nend = np.zeros(max(nl.value, 1), np.uint16)
    perm = np.zeros((nt.value, c32.shape[1] * tile), np.uint16)
    assert _lib.lib.exfem_host_tile_maps(*args, ptr.ctypes.data, nodes.ctypes.data, nend.ctypes.data,
                                         perm.ctypes.data) == 0
    return ptr, nodes[:nl.value], nend[:nl.value], perm


@pytest.mark.parametrize("kind", ["tet", "hex"])
def test_host_tile_maps_bit_exact(kind):
    """The tile maps of the matrix-free product (no counterpart in the reference),
    built by the library's threaded host code, equal the oracle's restatement bit
    for bit on a tile-ordered C3D10 (face-paired) and C3D8 mesh, both tile sizes."""
    from oracle import fem as ofem
    if kind == "tet":
        X, c = tet10_box(1.0, 1.0, 1.0, 6, 5, 5, frac=0.1, seed=2)
        order = fem.tile_order(X, c, 4)
        order, ct = fem.tile_pairs(order, c)
    else:
        X, c = mesh.box_hex(1.0, 1.0, 1.0, 10, 8, 8)
        ct = c[fem.tile_order(X, c, 8)]
    ct = np.asarray(ct)
    for tile in (128, 256):
        for g, w in zip(_host_tile_maps(ct, len(X), tile), ofem.tile_maps(ct, tile)):
            np.testing.assert_array_equal(g, w)


def test_newton_increment_checks_states_before_any_device_work():
    """The device Newton increment takes one state entry per block, and a J2 block's
    entry must hold its ne x ngp x nstate FP64 values: anything else is refused on
    the host, before a pointer reaches the library."""
    from types import SimpleNamespace as NS
    import torch
    j2 = NS(ne=2, etype=NS(ngp=8), material=NS(nstate=10), name="plastic")
    el = NS(ne=3, etype=NS(ngp=8), material=NS(nstate=1), name="elastic")
    fake = NS(blocks=[j2, el])
    u = torch.zeros(12, dtype=torch.float64)
    args = (u, u, 0.0, 1e-6, 4, True, 1e-6, 100)
    for states in ([None], [None, None], [torch.zeros(2, 8, 9, dtype=torch.float64), None],
                   [torch.zeros(2, 8, 10, dtype=torch.float32), None]):
        with pytest.raises(ValueError):
            linalg.NativeSolver.newton_increment(fake, u, states, *args)


_NULL_CALLS = r'''
import ctypes as C, json, sys
from exfem_b200 import _lib
out = {}
for name, (argt, _) in sorted(_lib._SIGS.items()):
    if name in ("exfem_version", "exfem_last_error"):
        continue
    args = [0 if t in (C.c_int, C.c_int64) else 0.0 if t is C.c_double else None for t in argt]
    st = getattr(_lib.lib, name)(*args)
    msg = _lib.lib.exfem_last_error()
    out[name] = [st, msg.decode() if msg else ""]
print(json.dumps(out))
'''


def test_every_export_refuses_null_arguments():
    """Every export called with NULL pointers and zero sizes (no GPU needed) returns
    a status without touching memory: an error with a message, except the destroy
    calls (NULL is a no-op, like free) and the host builders given nothing to do.
    Run in a child process, so that a crash fails the test instead of the run."""
    env = dict(os.environ, PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
    p = subprocess.run([sys.executable, "-c", _NULL_CALLS], capture_output=True, text=True, timeout=300, env=env,
                       cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    res = json.loads(p.stdout.strip().splitlines()[-1])
    ok_zero = {n for n in res if n.endswith("_destroy")} | {"exfem_host_face_once", "exfem_host_tile_pairs"}
    assert len(res) > 70
    for name, (st, msg) in res.items():
        if name in ok_zero:
            assert st == 0, (name, st, msg)
        else:
            assert st < 0 and msg, (name, st, msg)


def test_host_builders_refuse_invalid_sizes():
    """The host index builders given negative sizes, an unknown tile size, a tile
    order that is not a permutation or a dense block too large for the host return
    an argument error with a message instead of building a huge host array (an
    allocation error never leaves the library as a C++ exception)."""
    lib = _lib.lib
    buf = np.zeros(1 << 12, np.int64)
    b = buf.ctypes.data
    i64, i32 = C.c_int64(), C.c_int()
    calls = [
        lambda: lib.exfem_host_gather_plan(-1, 1, 8, b, b, C.byref(i32)),
        lambda: lib.exfem_host_gather_plan(8, -1, 8, b, b, C.byref(i32)),
        lambda: lib.exfem_host_colouring(-5, 1, 8, b, b, C.byref(i32)),
        lambda: lib.exfem_host_colouring(8, 1, -8, b, b, C.byref(i32)),
        lambda: lib.exfem_host_tile_order(-1, 1, 8, 8, b, b, b),
        lambda: lib.exfem_host_tile_pairs(-3, b, b, b),
        lambda: lib.exfem_host_tile_pairs(3, b, np.array([0, 0, 1], np.int32).ctypes.data, b),
        lambda: lib.exfem_host_tile_pairs(3, b, np.array([0, 5, 1], np.int32).ctypes.data, b),
        lambda: lib.exfem_host_tile_maps(8, 1, 8, b, 0, C.byref(i64), C.byref(i64), None, None, None, None),
        lambda: lib.exfem_host_tile_maps(-8, 0, 8, b, 256, C.byref(i64), C.byref(i64), None, None, None, None),
        lambda: lib.exfem_host_node_adjacency(-1, 1, 8, b, C.byref(i64), b, None),
        lambda: lib.exfem_host_standard_aggregation(-1, b, b, b, C.byref(i64)),
        lambda: lib.exfem_host_fit_candidates(2, 0, 6, b, 1, b, b, b),
        lambda: lib.exfem_host_coarse_inverse(1 << 21, b, b),
        lambda: lib.exfem_host_face_once(-4, b, b),
    ]
    for k, f in enumerate(calls):
        assert f() == _lib.ERR_ARG and _lib.last_error(), k
    # an empty slot list is a valid (empty) plan
    assert lib.exfem_host_gather_plan(4, 1, 0, b, None, C.byref(i32)) == 0 and i32.value == 1


def test_host_gather_plan_threaded_bit_exact():
    """A plan large enough to be built by several threads (over 2^21 slots, node
    numbers shuffled so that every thread's node range takes slots from all over
    the connectivity) equals the oracle's stable argsort plan."""
    X, c = mesh.box_hex(1, 1, 1, 66, 64, 64)
    perm = np.random.default_rng(4).permutation(len(X)).astype(np.int32)
    c = perm[c]
    assert c.size > 2 ** 21
    np.testing.assert_array_equal(_host_plan(c, len(X)), fem.gather_plan([c], len(X)))


def test_host_tile_order_threaded_bit_exact():
    """A tile order large enough to be sorted in several chunks and merged (three
    mesh components, jittered coordinates, over 2^17 elements) equals the oracle's
    restatement."""
    X1, c1 = mesh.box_hex(2.0, 1.0, 1.0, 64, 32, 32)
    X1 = mesh.jitter_interior(X1, 1.0 / 32, 0.1, 7)
    X2, c2 = mesh.box_hex(1.0, 1.0, 1.0, 20, 20, 20)
    X = np.concatenate([X1, X2 + 3.0, X1 - 5.0])
    c = np.concatenate([c1, c2 + len(X1), c1 + len(X1) + len(X2)])
    assert len(c) > 2 ** 17
    order = _host_order(X, c, 8)
    np.testing.assert_array_equal(order, fem.tile_order(X, c, 8))


def test_host_node_adjacency_threaded():
    """Node adjacency of a mesh large enough to be built by several threads (69k
    nodes, numbering shuffled) equals the sparsity pattern of the node-element
    incidence product, rows ascending."""
    X, c = mesh.box_hex(1, 1, 1, 40, 40, 40)
    perm = np.random.default_rng(8).permutation(len(X)).astype(np.int32)
    c = np.ascontiguousarray(perm[c])
    nn, ne = len(X), len(c)
    nnz, ptr = C.c_int64(), np.zeros(nn + 1, np.int64)
    _lib.check(_lib.lib.exfem_host_node_adjacency(nn, ne, 8, c.ctypes.data, C.byref(nnz), ptr.ctypes.data, None))
    idx = np.zeros(nnz.value, np.int32)
    _lib.check(_lib.lib.exfem_host_node_adjacency(nn, ne, 8, c.ctypes.data, C.byref(nnz), ptr.ctypes.data,
                                                  idx.ctypes.data))
    inc = sp.csr_matrix((np.ones(c.size), (c.ravel(), np.repeat(np.arange(ne), 8))), shape=(nn, ne))
    A = (inc @ inc.T + sp.identity(nn)).tocsr()
    A.sort_indices()
    np.testing.assert_array_equal(ptr, A.indptr)
    np.testing.assert_array_equal(idx, A.indices)


@pytest.mark.parametrize("nrows", [7, 120_000])
def test_host_filter_pattern(nrows):
    """The strength filter of the device set-up (the entries whose flag is set, row
    by row in order, with their positions) equals NumPy's boolean selection, on one
    thread and on several (120k rows), with empty rows and rows filtered empty."""
    rng = np.random.default_rng(nrows)
    cnt = rng.integers(0, 9, nrows)
    ptr = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
    idx = rng.integers(0, nrows, ptr[-1]).astype(np.int32)
    flag = (rng.random(ptr[-1]) < 0.7).astype(np.uint8)
    nnz = C.c_int64()
    _lib.check(_lib.lib.exfem_host_filter_pattern(nrows, ptr.ctypes.data, idx.ctypes.data, flag.ctypes.data,
                                                  C.byref(nnz), None, None, None))
    assert nnz.value == int(flag.sum())
    po, io, ko = np.empty(nrows + 1, np.int64), np.empty(nnz.value, np.int32), np.empty(nnz.value, np.int64)
    _lib.check(_lib.lib.exfem_host_filter_pattern(nrows, ptr.ctypes.data, idx.ctypes.data, flag.ctypes.data,
                                                  C.byref(nnz), po.ctypes.data, io.ctypes.data, ko.ctypes.data))
    rows = np.repeat(np.arange(nrows), cnt)
    sel = flag.astype(bool)
    np.testing.assert_array_equal(po, np.concatenate([[0], np.cumsum(np.bincount(rows[sel], minlength=nrows))]))
    np.testing.assert_array_equal(io, idx[sel])
    np.testing.assert_array_equal(ko, np.nonzero(sel)[0])
    bad = ptr.copy()
    bad[3] = bad[2] - 1
    assert _lib.lib.exfem_host_filter_pattern(nrows, bad.ctypes.data, idx.ctypes.data, flag.ctypes.data,
                                              C.byref(nnz), None, None, None) == _lib.ERR_ARG
