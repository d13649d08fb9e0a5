"""Model and element blocks on the GPU (drop-in for the solid-block part of ``gfem.model``).

Layout (gfem/model.py:1-11): one block = one element type + one material; every
element kernel is one launch over all elements of a block.  Each ``Block`` owns a
library handle holding, in HBM, the node coordinates, the connectivity, the
gather plan (bit-identical to gfem/model.py:241-261), an element colouring, the
per-element geometry streams of the matrix-free operator (FP32 and FP64) and,
for J2, the per-Gauss-point consistent-tangent data.

Public methods keep the reference's names and argument meaning:
``Model.internal_force(u, states, fields) -> (f, new_states)`` (model.py:466-477),
``element_stiffness`` (479-483), ``stiffness_ops -> [(dofs, Ke)]`` (485-486),
``tangent_jvp(u, states, v, fields)`` (488-490), ``matvec``/``diagonal``
(495-499), ``stresses`` (530-539), ``gather`` (421-429), ``init_state`` (380-381);
``Block.force``/``Block.stiff`` accept the reference's per-element gathered
arrays (model.py:70-111, 146-147).  Arrays are torch CUDA FP64 tensors (numpy
inputs are moved to the device).  There is no CPU path.
"""
import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import check, lib, ptr, stream_ptr


def gather_plan(conns, nn):
    """Atomic-free assembly plan of a list of element blocks (gfem/model.py:241-261):
    for every node the flat slots ``offset_b + e*nnode_b + a`` of the blocks'
    elements that touch it, in increasing order, padded with the total slot count
    (a zero row) to the maximum valence; (nn, vmax) int32.  The library's counting
    sort runs over the blocks' connectivities laid end to end as one slot list."""
    flat = [np.asarray(c, dtype=np.int32).reshape(-1) for c in conns]
    nslot = int(sum(f.size for f in flat))
    flat = np.ascontiguousarray(np.concatenate(flat + [np.zeros(1, np.int32)]))   # one spare entry: never empty
    vmax = C.c_int()
    check(lib.exfem_host_gather_plan(int(nn), 1, nslot, flat.ctypes.data, None, C.byref(vmax)))
    plan = np.empty((int(nn), vmax.value), np.int32)
    check(lib.exfem_host_gather_plan(int(nn), 1, nslot, flat.ctypes.data, plan.ctypes.data, C.byref(vmax)))
    return plan


def _check_thermal(material, Te, where):
    """Temperatures give a thermal strain alpha (T - T0) (gfem/model.py:54-59); the
    element kernels cover materials without thermal expansion only, so a field that
    would strain them is refused instead of ignored."""
    if Te is None or float(getattr(material, "alpha", 0.0)) == 0.0:
        return
    T = torch.as_tensor(Te, dtype=torch.float64)
    if bool(torch.any(T[..., 0] != T[..., 1])):
        raise NotImplementedError(f"{where()}: thermal strain (alpha = {material.alpha:g}, T != T0) is not covered "
                                  "by the element kernels")


def _dev(x, dtype=torch.float64):
    if isinstance(x, torch.Tensor):
        return x.to(device="cuda", dtype=dtype).contiguous()
    return torch.as_tensor(np.asarray(x), dtype=dtype, device="cuda").contiguous()


def _case_groups(nc):
    """Load cases in groups the multi-case PCG takes (16, 8, 4, 3, 2, 1 at a time)."""
    out = []
    while nc > 0:
        g = next(k for k in (16, 8, 4, 3, 2, 1) if k <= nc)
        out.append(g)
        nc -= g
    return out


class Block:
    """Element block: connectivity, element type and material (gfem/model.py:21-26,
    same positional arguments).  The global operators need the block bound to the
    model's node coordinates ``X`` (``Model.add_block`` binds it; a library handle
    then holds the device data); ``force``/``stiff`` on gathered element arrays work
    on an unbound block too."""

    def __init__(self, conn, etype, material, name="block", X=None):
        self.conn = np.ascontiguousarray(np.asarray(conn, dtype=np.int32))
        self.etype, self.material, self.name = etype, material, name
        self.ne = int(self.conn.shape[0])
        if self.ne and self.conn.shape[1] != etype.nnode:
            raise ValueError(f"{etype.name} needs {etype.nnode} nodes per element, got {self.conn.shape[1]}")
        self._h = None
        self._scale_key = None
        self._fixed_key = None
        self._local = None                  # (key, disjoint block) of the gathered-array signatures
        self.nn = 0
        if X is not None:
            self.bind(X)

    def bind(self, X):
        """Create the library handle over node coordinates X (nn, 3)."""
        _lib.require_cuda()
        if self._h is not None:
            raise RuntimeError(f"block {self.name} is already bound to node coordinates")
        X = np.ascontiguousarray(np.asarray(X, dtype=np.float64))
        self.nn = int(X.shape[0])
        h = C.c_void_p()
        m = self.material.to_c()
        check(lib.exfem_block_create(self.etype.code, C.byref(m), self.nn, X.ctypes.data, self.ne,
                                     self.conn.ctypes.data if self.ne else None, C.byref(h)))
        self._h = h
        self.conn_dev = torch.as_tensor(self.conn, device="cuda")
        return self

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib.exfem_block_destroy(h)
            self._h = None

    @property
    def handle(self):
        if self._h is None:
            raise RuntimeError(f"block {self.name} is not bound to node coordinates (Model.add_block binds it)")
        return self._h

    # ---------------- info and index maps
    def query(self):
        ne, nn, vmax, ncol, aff, nb = C.c_int64(), C.c_int64(), C.c_int(), C.c_int(), C.c_int(), C.c_int64()
        nnode, ngp, ns = C.c_int(), C.c_int(), C.c_int()
        check(lib.exfem_block_query(self.handle, C.byref(ne), C.byref(nn), C.byref(nnode), C.byref(ngp), C.byref(ns),
                                    C.byref(vmax), C.byref(ncol), C.byref(aff), C.byref(nb)))
        return dict(ne=ne.value, nn=nn.value, nnode=nnode.value, ngp=ngp.value, nstate=ns.value,
                    vmax=vmax.value, ncolour=ncol.value, affine=bool(aff.value), device_bytes=nb.value)

    def gather_plan(self):
        q = self.query()
        out = np.empty((self.nn, q["vmax"]), np.int32)
        check(lib.exfem_block_gather_plan(self.handle, out.ctypes.data))
        return out

    def colours(self):
        out = np.empty(self.ne, np.int32)
        check(lib.exfem_block_colours(self.handle, out.ctypes.data))
        return out

    def tile_maps(self):
        """(ptr, nodes, nend, perm) element-tile maps of the matrix-free operator."""
        nt, nl, mu = C.c_int64(), C.c_int64(), C.c_int()
        check(lib.exfem_block_tile_info(self.handle, C.byref(nt), C.byref(nl), C.byref(mu)))
        tile, _ = self.tile_order()
        ptr_ = np.empty(nt.value + 1, np.int32)
        nodes = np.empty(max(nl.value, 1), np.int32)
        nend = np.empty(max(nl.value, 1), np.uint16)
        perm = np.empty((nt.value, self.etype.nnode * tile), np.uint16)
        check(lib.exfem_block_tile_maps(self.handle, ptr_.ctypes.data, nodes.ctypes.data, nend.ctypes.data,
                                        perm.ctypes.data))
        return ptr_, nodes[:nl.value], nend[:nl.value], perm

    def tile_conn(self):
        """(ne, nnode) connectivity of every tile position in the tiles' numbering."""
        out = np.empty((max(self.ne, 1), self.etype.nnode), np.int32)
        check(lib.exfem_block_tile_conn(self.handle, out.ctypes.data))
        return out[:self.ne]

    def tile_order(self):
        """(tile, order): elements per tile and the tile order (position -> element)."""
        tile = C.c_int()
        order = np.empty(max(self.ne, 1), np.int32)
        check(lib.exfem_block_tile_order(self.handle, C.byref(tile), order.ctypes.data))
        return tile.value, order[:self.ne]

    def init_state(self):                                              # model.py:154-155
        return torch.zeros((self.ne, self.etype.ngp, self.material.nstate), dtype=torch.float64, device="cuda")

    def dofs(self):                                                    # model.py:157-158
        return (self.conn_dev.long()[:, :, None] * 3 + torch.arange(3, device="cuda")).reshape(self.ne, -1)

    # ---------------- parameters
    def set_scale(self, scale):
        """Per-element stiffness scale (fields["scale"], model.py:449-463)."""
        if scale is None:
            if self._scale_key is not None:
                check(lib.exfem_block_set_scale(self.handle, None))
                self._scale_key = None
            return
        s = np.ascontiguousarray(np.asarray(scale.cpu() if isinstance(scale, torch.Tensor) else scale,
                                            dtype=np.float64).reshape(-1))
        # compared with a kept copy of the last one set (a memory compare, cheaper
        # than hashing the array on every call)
        if self._scale_key is None or self._scale_key.shape != s.shape or not np.array_equal(self._scale_key, s):
            check(lib.exfem_block_set_scale(self.handle, s.ctypes.data))
            self._scale_key = s.copy()

    def set_lame(self, lam, mu):
        """Per-element Lame parameters of the matrix-free operator (a block holding
        many linear-elastic instances with their own E and nu); None, None = the
        block material's."""
        if lam is None and mu is None:
            check(lib.exfem_block_set_lame(self.handle, None, None))
            return
        lam = np.ascontiguousarray(np.asarray(lam, dtype=np.float64).reshape(-1))
        mu = np.ascontiguousarray(np.asarray(mu, dtype=np.float64).reshape(-1))
        if lam.size != self.ne or mu.size != self.ne:
            raise ValueError(f"need {self.ne} Lame pairs, got {lam.size} and {mu.size}")
        check(lib.exfem_block_set_lame(self.handle, lam.ctypes.data, mu.ctypes.data))

    def set_fixed(self, fixed):
        """Prescribed-DOF mask (ndof of this block's node set) used by opA."""
        if fixed is None:
            if self._fixed_key is not None:
                check(lib.exfem_block_set_fixed(self.handle, None))
                self._fixed_key = None
            return
        f = np.ascontiguousarray(np.asarray(fixed).reshape(-1)).view(np.uint8) if np.asarray(fixed).dtype == bool \
            else np.ascontiguousarray(np.asarray(fixed).astype(np.uint8).reshape(-1))
        if self._fixed_key is None or self._fixed_key.shape != f.shape or not np.array_equal(self._fixed_key, f):
            check(lib.exfem_block_set_fixed(self.handle, f.ctypes.data))
            self._fixed_key = f.copy()

    # ---------------- kernels on global vectors
    def internal_force(self, u, state, assembly=_lib.ASSEMBLE_GATHER, fe=None):
        u = _dev(u)
        j2 = self.material.nstate > 1
        s_old = _dev(state) if j2 else None
        s_new = torch.empty_like(s_old) if j2 else None
        f = torch.empty(3 * self.nn, dtype=torch.float64, device="cuda")
        check(lib.exfem_internal_force(self.handle, ptr(u), ptr(s_old), ptr(s_new), ptr(fe), ptr(f), assembly,
                                       stream_ptr()))
        return f, (s_new if j2 else state)

    def stiffness(self, u, state, dtype=torch.float64):
        code = {torch.float64: _lib.F64, torch.float32: _lib.F32, torch.bfloat16: _lib.BF16}[dtype]
        u = _dev(u)
        s_old = _dev(state) if self.material.nstate > 1 else None
        nd = self.etype.nd
        Ke = torch.empty((self.ne, nd, nd), dtype=dtype, device="cuda")
        check(lib.exfem_element_stiffness(self.handle, ptr(u), ptr(s_old), code, ptr(Ke), stream_ptr()))
        return Ke

    def tangent_update(self, u, state):
        if self.material.nstate > 1:
            check(lib.exfem_tangent_update(self.handle, ptr(_dev(u)), ptr(_dev(state)), stream_ptr()))

    def tangent_matvec(self, v, out=None, apply_bc=True):
        v = v.contiguous()
        code = _lib.F64 if v.dtype == torch.float64 else _lib.F32
        y = torch.empty_like(v) if out is None else out
        check(lib.exfem_tangent_matvec(self.handle, code, ptr(v), ptr(y), 1 if apply_bc else 0, stream_ptr()))
        return y

    def tangent_diagonal(self):
        d = torch.empty(3 * self.nn, dtype=torch.float64, device="cuda")
        check(lib.exfem_tangent_diagonal(self.handle, ptr(d), stream_ptr()))
        return d

    def ebe_matvec_multi(self, Ke, V, apply_bc=True, engine="cuda"):
        """Stored-Ke product of several right-hand sides, V (ndof, nrhs <= 16) ->
        (ndof, nrhs).  engine "cuda": Ke (ne, nd, nd) BF16 or FP32 with FP32 V and
        accumulation, or FP64 Ke with FP64 V; "tc": the tensor-core form, BF16 Ke,
        V rounded to BF16, FP32 accumulation."""
        if engine == "tc":
            V = V.to(torch.float32).contiguous()
            Y = torch.empty_like(V)
            check(lib.exfem_ebe_matvec_bf16_multi(self.handle, ptr(Ke.contiguous()), V.shape[1], ptr(V), ptr(Y),
                                                  1 if apply_bc else 0, stream_ptr()))
            return Y
        if engine != "cuda":
            raise ValueError(f"unknown engine {engine!r}")
        code = {torch.float64: _lib.F64, torch.float32: _lib.F32, torch.bfloat16: _lib.BF16}[Ke.dtype]
        V = V.to(torch.float64 if Ke.dtype == torch.float64 else torch.float32).contiguous()
        Y = torch.empty_like(V)
        check(lib.exfem_ebe_matvec_multi(self.handle, ptr(Ke.contiguous()), code, V.shape[1], ptr(V), ptr(Y),
                                         1 if apply_bc else 0, stream_ptr()))
        return Y

    def multi_pcg(self, Ke, B, tol=1e-8, maxiter=20000):
        """Jacobi PCG over the columns of B (ndof, ncase) at once with the stored
        FP64 Ke and this block's prescribed DOFs (gfem/optimize.py:116-143): one
        product per iteration for every case, each case with its own scalars and
        stopping test.  Returns (X, iters, relres) per case."""
        B = B.to(torch.float64)
        nc = B.shape[1]
        X = torch.empty_like(B)
        iters, rel = np.zeros(nc, np.int32), np.zeros(nc)
        j = 0
        for size in _case_groups(nc):
            Bg = B[:, j:j + size].contiguous()
            Xg = torch.empty_like(Bg)
            it = np.zeros(size, np.int32)
            rr = np.zeros(size)
            st = lib.exfem_multi_pcg(self.handle, ptr(Ke.contiguous()), size, ptr(Bg), ptr(Xg), float(tol),
                                     int(maxiter), it.ctypes.data, rr.ctypes.data, stream_ptr())
            if st < 0:
                check(st)
            X[:, j:j + size] = Xg
            iters[j:j + size], rel[j:j + size] = it, rr
            j += size
        return X, iters, rel

    def ebe_matvec(self, Ke, v, apply_bc=True):
        v = _dev(v)
        y = torch.empty_like(v)
        check(lib.exfem_ebe_matvec(self.handle, ptr(Ke.contiguous()), ptr(v), ptr(y), 1 if apply_bc else 0, stream_ptr()))
        return y

    def ebe_diagonal(self, Ke):
        d = torch.empty(3 * self.nn, dtype=torch.float64, device="cuda")
        check(lib.exfem_ebe_diagonal(self.handle, ptr(Ke.contiguous()), ptr(d), stream_ptr()))
        return d

    def geometric_stiffness(self, S):
        """Initial-stress stiffness of every element under its Cauchy stress S
        (ne, 3, 3) (gfem/model.py:113-117): Kg (ne, nd, nd) FP64."""
        S = _dev(S).reshape(self.ne, 3, 3).contiguous()
        nd = self.etype.nd
        Kg = torch.empty((self.ne, nd, nd), dtype=torch.float64, device="cuda")
        check(lib.exfem_geometric_stiffness(self.handle, ptr(S), ptr(Kg), stream_ptr()))
        return Kg

    def cauchy(self, u, state):
        S = torch.empty((self.ne, 3, 3), dtype=torch.float64, device="cuda")
        mises = torch.empty(self.ne, dtype=torch.float64, device="cuda")
        peeq = torch.empty(self.ne, dtype=torch.float64, device="cuda")
        s = _dev(state) if self.material.nstate > 1 else None
        check(lib.exfem_stresses(self.handle, ptr(_dev(u)), ptr(s), ptr(S), ptr(mises), ptr(peeq), stream_ptr()))
        return S, mises, peeq

    # ---------------- reference per-element signatures (model.py:70-111)
    def _disjoint(self, Xe):
        """A block of the same type and material whose elements own their nodes,
        over the gathered coordinates Xe (ne, nnode, 3); kept while Xe is unchanged,
        so repeated calls on one mesh build its geometry streams once."""
        Xh = np.ascontiguousarray(np.asarray(Xe.detach().cpu() if isinstance(Xe, torch.Tensor) else Xe,
                                             dtype=np.float64))
        key = (Xh.shape, hash(Xh.tobytes()))
        if self._local is None or self._local[0] != key:
            ne, nnode = Xh.shape[0], Xh.shape[1]
            conn = np.arange(ne * nnode, dtype=np.int32).reshape(ne, nnode)
            self._local = (key, Block(conn, self.etype, self.material, self.name, X=Xh.reshape(-1, 3)))
        return self._local[1]

    def _element_fields(self, b, Te, scv):
        """Stiffness scale of the gathered-array signatures; temperature and
        eigenstrain fields are checked, because the element kernels cover neither."""
        _check_thermal(self.material, Te, lambda: f"block {self.name}")
        if scv is None:
            b.set_scale(None)
            return
        scv = torch.as_tensor(scv, dtype=torch.float64)
        if scv.shape[-1] > 1 and bool(torch.any(scv[:, 1:] != 0)):
            raise NotImplementedError(f"block {self.name}: eigenstrain fields are not covered by the element kernels")
        b.set_scale(np.asarray(scv[:, 0].cpu()))

    def force(self, Xe, ue, se=None, Te=None, scv=None):
        """Element forces from gathered arrays Xe, ue (ne, nnode, 3): (fe, s_new)."""
        b = self._disjoint(Xe)
        self._element_fields(b, Te, scv)
        st = se if se is not None else b.init_state()
        fe = torch.empty((b.ne, self.etype.nnode, 3), dtype=torch.float64, device="cuda")
        _, sn = b.internal_force(_dev(ue).reshape(-1), st, fe=fe)
        return fe, sn

    def stiff(self, Xe, ue, se=None, Te=None, scv=None):
        """Element tangents from gathered arrays: Ke (ne, nd, nd)."""
        b = self._disjoint(Xe)
        self._element_fields(b, Te, scv)
        st = se if se is not None else b.init_state()
        return b.stiffness(_dev(ue).reshape(-1), st)


class Model:
    """Nodes + element blocks (gfem/model.py:270-539, solid blocks)."""

    def __init__(self, nodes):
        self.X = np.ascontiguousarray(np.asarray(nodes, dtype=np.float64))
        self.nn = int(self.X.shape[0])
        self.ndof = 3 * self.nn
        self.blocks = []
        self.nsets, self.elsets, self.surfaces = {}, {}, {}
        self.constraints, self.interactions = [], []
        self.rot_of = {}
        self.T0 = None

    def add_block(self, conn, etype, material, name=None):
        b = Block(conn, etype, material, name or f"block{len(self.blocks)}", X=self.X)
        self.blocks.append(b)
        return b

    def init_state(self):
        return [b.init_state() for b in self.blocks]

    def gather(self):
        """The gather plan over all blocks (gfem/model.py:421-429 with 241-261)."""
        if len(self.blocks) == 1:
            return self.blocks[0].gather_plan()
        return gather_plan([b.conn for b in self.blocks], self.nn)

    def dof(self, nodes, d):
        return np.asarray(nodes, dtype=np.int64).ravel() * 3 + d

    def rot_mask(self):
        return np.zeros(self.nn, bool)

    @property
    def nelem(self):
        return sum(b.ne for b in self.blocks)

    def default_fields(self):
        return dict(scale=[None] * len(self.blocks))

    def _apply_fields(self, fields):
        """fields (gfem/model.py:446-463): "scale" per block is applied; "T" (nodal
        temperatures against the initial ``T0``) and "eig" (per-element
        eigenstrains) are refused where they would change the result, because the
        element kernels cover neither."""
        fields = fields or {}
        sc = fields.get("scale") or [None] * len(self.blocks)
        for b, s in zip(self.blocks, sc):
            b.set_scale(s)
        T = fields.get("T")
        if T is not None:
            T = torch.as_tensor(T, dtype=torch.float64).reshape(-1)
            T0 = torch.zeros_like(T) if self.T0 is None else torch.as_tensor(self.T0, dtype=torch.float64).reshape(-1)
            for b in self.blocks:
                _check_thermal(b.material, torch.stack([T, T0], 1), lambda: f"block {b.name}")
        for b, e in zip(self.blocks, fields.get("eig") or []):
            if e is not None and bool(torch.any(torch.as_tensor(e) != 0)):
                raise NotImplementedError(f"block {b.name}: eigenstrain fields are not covered by the element kernels")

    # ---------- global operators
    def internal_force(self, u, states, fields=None, assembly=_lib.ASSEMBLE_GATHER):
        self._apply_fields(fields)
        u = _dev(u)
        f, new = None, []
        for b, s in zip(self.blocks, states):
            fb, sn = b.internal_force(u, s, assembly)
            f = fb if f is None else f + fb
            new.append(sn)
        if f is None:
            f = torch.zeros(self.ndof, dtype=torch.float64, device="cuda")
        return f, new

    def element_stiffness(self, u, states, fields=None, dtype=torch.float64):
        self._apply_fields(fields)
        u = _dev(u)
        return [b.stiffness(u, s, dtype) for b, s in zip(self.blocks, states)]

    def stiffness_ops(self, u, states, fields=None):
        return list(zip([b.dofs() for b in self.blocks], self.element_stiffness(u, states, fields)))

    def tangent_update(self, u, states, fields=None):
        self._apply_fields(fields)
        u = _dev(u)
        for b, s in zip(self.blocks, states):
            b.tangent_update(u, s)

    def tangent_jvp(self, u, states, v, fields=None):
        """K(u) v with the matrix-free tangent (no boundary conditions applied)."""
        self.tangent_update(u, states, fields)
        v = _dev(v)
        out = None
        for b in self.blocks:
            y = b.tangent_matvec(v, apply_bc=False)
            out = y if out is None else out + y
        return out

    def matvec(self, Kes, v):
        v = _dev(v)
        out = None
        for b, K in zip(self.blocks, Kes):
            y = b.ebe_matvec(K, v, apply_bc=False)
            out = y if out is None else out + y
        return out

    def diagonal(self, Kes):
        out = None
        for b, K in zip(self.blocks, Kes):
            d = b.ebe_diagonal(K)
            out = d if out is None else out + d
        return out

    def stresses(self, u, states, fields=None):
        self._apply_fields(fields)
        out = []
        for b, s in zip(self.blocks, states):
            S, mises, peeq = b.cauchy(u, s)
            out.append(dict(S=S, MISES=mises, PEEQ=peeq))
        return out

    def geometric_ops(self, stresses, u=None, states=None):
        """Initial-stress stiffness ops [(dofs, Kg)] of the solid blocks from their
        element stresses (``stresses()[b]["S"]``; gfem/model.py:541-553)."""
        return [(b.dofs(), b.geometric_stiffness(st["S"])) for b, st in zip(self.blocks, stresses)]

    def summary(self):
        lines = [f"{self.nn} nodes, {self.nelem} elements, {self.ndof} dofs"]
        for b in self.blocks:
            lines.append(f"  {b.name}: {b.ne} x {b.etype.name}, {b.material.describe()}")
        return "\n".join(lines)
