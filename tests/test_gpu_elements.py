"""Element kernels, index maps and EbE products on the GPU against the CPU oracle.

Bars (north star): FP64 element forces, element tangents and matvecs agree with
the oracle to 1e-12 relative (max-norm); index maps (gather plan, colouring)
bit for bit; the FP32 matrix-free product to 2e-6 relative (FP32 rounding of
O(100) terms per entry).
"""
import numpy as np
import pytest
import torch

from helpers import jittered_box, rel_err, smooth_field, tet10_box
from oracle import fem as ofem

pytestmark = pytest.mark.gpu

E, NU = 210000.0, 0.3
TABLE = [[250.0, 0.0], [1250.0, 1.0]]          # sy = 250 MPa, H = 1 GPa (config 2)


def _pair(kind, mat_kind, n=(4, 3, 3), seed=0):
    import exfem_b200 as xf
    if kind == "hex":
        X, c = jittered_box(4.0, 3.0, 3.0, *n, frac=0.15, seed=seed)
        pet, oet = xf.HEX8, ofem.HEX8
    else:
        X, c = tet10_box(2.0, 2.0, 2.0, *n, frac=0.15, seed=seed)
        pet, oet = xf.TET10, ofem.TET10
    if mat_kind == "el":
        pm, om = xf.LinearElastic(E, NU), ofem.LinearElastic(E, NU)
    else:
        pm, om = xf.J2Plasticity(E, NU, TABLE, Hk=500.0), ofem.J2Plasticity(E, NU, TABLE, Hk=500.0)
    pmod = xf.Model(X)
    pmod.add_block(c, pet, pm)
    omod = ofem.Model(X)
    omod.add_block(c, oet, om)
    return X, c, pmod, omod


def _plastic_state(pmod, omod, X, amp):
    """A nonzero history: states after one force evaluation at a yielding field."""
    u0 = smooth_field(X, amp, seed=3)
    _, s1 = omod.internal_force(torch.as_tensor(u0), omod.init_state())
    return [s.clone() for s in s1], [s.cuda() for s in s1]


@pytest.mark.parametrize("kind", ["hex", "tet"])
@pytest.mark.parametrize("mat_kind", ["el", "j2"])
def test_internal_force_and_states(cuda, kind, mat_kind):
    X, c, pmod, omod = _pair(kind, mat_kind)
    amp = 2e-3 if mat_kind == "el" else 6e-3
    if mat_kind == "j2":
        so, sp = _plastic_state(pmod, omod, X, 4e-3)
    else:
        so, sp = omod.init_state(), pmod.init_state()
    u = smooth_field(X, amp, seed=1)
    fo, sno = omod.internal_force(torch.as_tensor(u), so)
    fp, snp = pmod.internal_force(torch.as_tensor(u, device="cuda"), sp)
    assert rel_err(fp, fo) < 1e-12
    if mat_kind == "j2":
        assert rel_err(snp[0], sno[0]) < 1e-12
        assert float(sno[0][..., 9].max()) > 0          # plasticity actually active


@pytest.mark.parametrize("kind", ["hex", "tet"])
def test_colour_assembly_matches_gather(cuda, kind):
    from exfem_b200 import _lib
    X, c, pmod, omod = _pair(kind, "el")
    u = torch.as_tensor(smooth_field(X, 1e-3), device="cuda")
    s = pmod.init_state()
    f1, _ = pmod.internal_force(u, s, assembly=_lib.ASSEMBLE_GATHER)
    f2, _ = pmod.internal_force(u, s, assembly=_lib.ASSEMBLE_COLOUR)
    assert rel_err(f2, f1) < 1e-14
    f3, _ = pmod.internal_force(u, s, assembly=_lib.ASSEMBLE_COLOUR)
    assert torch.equal(f2, f3)                            # deterministic


@pytest.mark.parametrize("kind", ["hex", "tet"])
@pytest.mark.parametrize("mat_kind", ["el", "j2"])
def test_element_stiffness(cuda, kind, mat_kind):
    X, c, pmod, omod = _pair(kind, mat_kind, n=(2, 2, 2))
    if mat_kind == "j2":
        so, sp = _plastic_state(pmod, omod, X, 4e-3)
    else:
        so, sp = omod.init_state(), pmod.init_state()
    u = smooth_field(X, 6e-3, seed=2)
    Ko = omod.element_stiffness(torch.as_tensor(u), so)[0]
    Kp = pmod.element_stiffness(torch.as_tensor(u, device="cuda"), sp)[0]
    assert rel_err(Kp, Ko) < 1e-12
    K32 = pmod.element_stiffness(torch.as_tensor(u, device="cuda"), sp, dtype=torch.float32)[0]
    assert rel_err(K32.double(), Ko) < 1e-6


@pytest.mark.parametrize("kind", ["hex", "tet"])
@pytest.mark.parametrize("mat_kind", ["el", "j2"])
def test_matrix_free_tangent_matvec(cuda, kind, mat_kind):
    X, c, pmod, omod = _pair(kind, mat_kind)
    if mat_kind == "j2":
        so, sp = _plastic_state(pmod, omod, X, 4e-3)
    else:
        so, sp = omod.init_state(), pmod.init_state()
    u = smooth_field(X, 6e-3, seed=2)
    v = np.random.default_rng(5).standard_normal(pmod.ndof)
    yo = omod.tangent_jvp(torch.as_tensor(u), so, torch.as_tensor(v))
    yp = pmod.tangent_jvp(torch.as_tensor(u, device="cuda"), sp, torch.as_tensor(v, device="cuda"))
    assert rel_err(yp, yo) < 1e-12
    blk = pmod.blocks[0]
    y32 = blk.tangent_matvec(torch.as_tensor(v, device="cuda", dtype=torch.float32), apply_bc=False)
    assert rel_err(y32.double(), yo) < 2e-6


@pytest.mark.parametrize("kind", ["hex", "tet"])
def test_ebe_matvec_diagonal_and_opA(cuda, kind):
    X, c, pmod, omod = _pair(kind, "el")
    s = omod.init_state()
    u = smooth_field(X, 1e-3)
    ops = omod.stiffness_ops(torch.as_tensor(u), s)
    v = torch.as_tensor(np.random.default_rng(7).standard_normal(pmod.ndof))
    yo = ofem.ops_matvec(ops, v, omod.ndof)
    Kp = pmod.element_stiffness(torch.as_tensor(u, device="cuda"), pmod.init_state())
    yp = pmod.matvec(Kp, v.cuda())
    assert rel_err(yp, yo) < 1e-12
    assert rel_err(pmod.diagonal(Kp), ofem.ops_diagonal(ops, omod.ndof)) < 1e-12
    # opA = free*K(free*v) + fixed*v with a BC mask (solvers.py:257-267)
    fixed = np.zeros(pmod.ndof, bool)
    fixed[::7] = True
    free = torch.as_tensor((~fixed).astype(float))
    ref = free * ofem.ops_matvec(ops, free * v, omod.ndof) + (1 - free) * v
    blk = pmod.blocks[0]
    blk.set_fixed(fixed)
    assert rel_err(blk.ebe_matvec(Kp[0], v.cuda()), ref) < 1e-12
    blk.tangent_update(torch.as_tensor(u, device="cuda"), pmod.init_state()[0])
    assert rel_err(blk.tangent_matvec(v.cuda()), ref) < 1e-12
    blk.set_fixed(None)


@pytest.mark.parametrize("kind", ["hex", "tet"])
def test_index_maps_bit_exact(cuda, kind):
    X, c, pmod, omod = _pair(kind, "el", n=(5, 4, 3))
    np.testing.assert_array_equal(pmod.gather(), ofem.gather_plan([c], len(X)))
    np.testing.assert_array_equal(pmod.blocks[0].colours(), ofem.greedy_colouring(c, len(X)))
    tile, order = pmod.blocks[0].tile_order()
    want_order = ofem.tile_order(X, c, 8 if kind == "hex" else 4)
    want_conn = np.asarray(c)[want_order]
    if kind == "tet":                               # linear-elastic C3D10: face pairs
        want_order, want_conn = ofem.tile_pairs(want_order, c)
    np.testing.assert_array_equal(order, want_order)
    np.testing.assert_array_equal(pmod.blocks[0].tile_conn(), want_conn)
    for got, want in zip(pmod.blocks[0].tile_maps(), ofem.tile_maps(want_conn, tile)):
        np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("kind", ["hex", "tet"])
@pytest.mark.parametrize("mat_kind", ["el", "j2"])
def test_stresses(cuda, kind, mat_kind):
    X, c, pmod, omod = _pair(kind, mat_kind)
    if mat_kind == "j2":
        so, sp = _plastic_state(pmod, omod, X, 4e-3)
    else:
        so, sp = omod.init_state(), pmod.init_state()
    u = smooth_field(X, 5e-3, seed=4)
    ro = omod.stresses(torch.as_tensor(u), so)[0]
    rp = pmod.stresses(torch.as_tensor(u, device="cuda"), sp)[0]
    for k in ("S", "MISES", "PEEQ"):
        assert rel_err(rp[k], ro[k]) < 1e-12 or float(ro[k].abs().max()) == 0.0


def test_scale_field(cuda):
    X, c, pmod, omod = _pair("tet", "el")
    rng = np.random.default_rng(11)
    sc = np.exp(rng.uniform(0, np.log(10), size=len(c)))
    u = smooth_field(X, 1e-3)
    fo, _ = omod.internal_force(torch.as_tensor(u), omod.init_state(), scale=[sc])
    fp, _ = pmod.internal_force(torch.as_tensor(u, device="cuda"), pmod.init_state(), dict(scale=[sc]))
    assert rel_err(fp, fo) < 1e-12
    v = torch.as_tensor(rng.standard_normal(pmod.ndof))
    yo = omod.tangent_jvp(torch.as_tensor(u), omod.init_state(), v, scale=[sc])
    yp = pmod.tangent_jvp(torch.as_tensor(u, device="cuda"), pmod.init_state(), v.cuda(), dict(scale=[sc]))
    assert rel_err(yp, yo) < 1e-12


def test_autotuner_picks_a_tile_and_both_tiles_agree(cuda):
    import exfem_b200 as xf
    from exfem_b200 import tuning
    from exfem_b200.model import Block
    res = tuning.autotune((xf.TET10,), n=12, reps=3)
    tile, times = res["C3D10"]
    assert tile in tuning.CANDIDATES and set(times) == set(tuning.CANDIDATES)
    assert tuning.current(xf.TET10) == tile
    X, c = tet10_box(1, 1, 1, 4, 3, 3)
    rng = np.random.default_rng(5)
    v = torch.as_tensor(rng.standard_normal(3 * len(X)), device="cuda")
    ys = {}
    for t in tuning.CANDIDATES:
        tuning.apply(xf.TET10, t)
        blk = Block(c, xf.TET10, xf.LinearElastic(1000.0, 0.3), X=X)
        assert blk.tile_order()[0] == t
        ys[t] = blk.tangent_matvec(v.float()).double()
        y64 = blk.tangent_matvec(v)
    tuning.apply(xf.TET10, tile)
    for t in tuning.CANDIDATES:
        assert rel_err(ys[t], y64) < 2e-6


@pytest.mark.parametrize("kind", ["hex", "tet"])
@pytest.mark.parametrize("nrhs", [1, 4, 16])
def test_tensor_core_stored_ke_multi_rhs(cuda, kind, nrhs):
    """BF16 Ke x BF16 right-hand sides with FP32 accumulation (tcgen05): equal to
    the same BF16-rounded operands multiplied in FP64 up to FP32 accumulation
    (1e-5), and to the FP64 stored-Ke product within BF16 rounding (2e-2)."""
    from exfem_b200.model import Block
    X, c, pmod, omod = _pair(kind, "el", n=(5, 4, 3))
    blk = pmod.blocks[0]
    fixed = np.zeros(pmod.ndof, bool)
    fixed[::7] = True
    blk.set_fixed(fixed)
    zero = torch.zeros(pmod.ndof, dtype=torch.float64, device="cuda")
    Kb = blk.stiffness(zero, blk.init_state(), dtype=torch.bfloat16)
    K64 = blk.stiffness(zero, blk.init_state())
    rng = np.random.default_rng(nrhs)
    V = torch.as_tensor(rng.standard_normal((pmod.ndof, nrhs)), dtype=torch.float32, device="cuda")
    Y = blk.ebe_matvec_multi(Kb, V, engine="tc")
    Vb = V.to(torch.bfloat16).double()
    for r in range(nrhs):
        yb = blk.ebe_matvec(Kb.double(), Vb[:, r].contiguous())
        y64 = blk.ebe_matvec(K64, V[:, r].double().contiguous())
        # prescribed rows take v itself (FP32 V, not its BF16 rounding)
        yb[torch.as_tensor(fixed, device="cuda")] = V[torch.as_tensor(fixed, device="cuda"), r].double()
        assert rel_err(Y[:, r].double(), yb) < 1e-5
        assert rel_err(Y[:, r].double(), y64) < 2e-2
    blk.set_fixed(None)


@pytest.mark.parametrize("kind", ["hex", "tet"])
@pytest.mark.parametrize("nrhs", [1, 4, 5, 16])
def test_multi_rhs_stored_ke_product(cuda, kind, nrhs):
    """CUDA-core stored-Ke product of several right-hand sides: FP64 Ke against the
    single-right-hand-side FP64 product of each column (1e-13), FP32 Ke (1e-6) and
    BF16 Ke (against the BF16-rounded Ke in FP64, 1e-5) — prescribed rows included."""
    X, c, pmod, omod = _pair(kind, "el", n=(5, 4, 3))
    blk = pmod.blocks[0]
    fixed = np.zeros(pmod.ndof, bool)
    fixed[::7] = True
    blk.set_fixed(fixed)
    zero = torch.zeros(pmod.ndof, dtype=torch.float64, device="cuda")
    K64 = blk.stiffness(zero, blk.init_state())
    rng = np.random.default_rng(100 + nrhs)
    V = torch.as_tensor(rng.standard_normal((pmod.ndof, nrhs)), device="cuda")
    Y64 = blk.ebe_matvec_multi(K64, V)
    Y32 = blk.ebe_matvec_multi(K64.float(), V.float())
    Kb = K64.to(torch.bfloat16)
    Yb = blk.ebe_matvec_multi(Kb, V.float())
    assert Y64.dtype == torch.float64 and Y32.dtype == torch.float32 and Yb.dtype == torch.float32
    for r in range(nrhs):
        y = blk.ebe_matvec(K64, V[:, r].contiguous())
        assert rel_err(Y64[:, r], y) < 1e-13
        assert rel_err(Y32[:, r].double(), y) < 1e-6
        yb = blk.ebe_matvec(Kb.double(), V[:, r].float().double().contiguous())
        assert rel_err(Yb[:, r].double(), yb) < 1e-5
    blk.set_fixed(None)


def test_multi_rhs_product_with_unaligned_operands(cuda):
    """The C ABI takes V and Y at any element-aligned address: a V and a Y four bytes
    off a 16-byte boundary give the same product as aligned copies (the 16-byte
    loads and stores are used only where the addresses allow them)."""
    from exfem_b200 import _lib
    from exfem_b200._lib import lib
    X, c, pmod, omod = _pair("hex", "el", n=(5, 4, 3))
    blk = pmod.blocks[0]
    zero = torch.zeros(pmod.ndof, dtype=torch.float64, device="cuda")
    Kb = blk.stiffness(zero, blk.init_state(), dtype=torch.bfloat16)
    nr = 4
    V = torch.randn(pmod.ndof, nr, dtype=torch.float32, device="cuda")
    Y = blk.ebe_matvec_multi(Kb, V)
    buf = torch.zeros(2, pmod.ndof * nr + 1, dtype=torch.float32, device="cuda")
    Vu, Yu = buf[0, 1:], buf[1, 1:]
    Vu.copy_(V.reshape(-1))
    assert Vu.data_ptr() % 16 != 0 and Yu.data_ptr() % 16 != 0
    _lib.check(lib.exfem_ebe_matvec_multi(blk.handle, _lib.ptr(Kb), _lib.BF16, nr, Vu.data_ptr(), Yu.data_ptr(), 1,
                                          _lib.stream_ptr()))
    torch.testing.assert_close(Yu.reshape(pmod.ndof, nr), Y, rtol=0, atol=0)

