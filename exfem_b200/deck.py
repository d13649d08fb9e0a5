"""Abaqus-style input decks for the structural hot path (drop-in for the solid,
static part of ``gfem.io.inp``: ``read_inp(path) -> (Model, [Step])``,
gfem/io/inp.py:635-643).

Covered cards (the others are skipped; element types other than the solid C3D8 /
C3D10 families and the dynamic, heat, buckling and frequency procedures raise
``NotImplementedError``), restating the reference reader's meaning
(gfem/io/inp.py:27-60 tokenizer, 101-336 cards, 503-616 sets, surfaces and step
data):

  * ``*INCLUDE, INPUT=`` — the included file's lines in place;
  * ``*NODE`` (``NSET=``), ``*ELEMENT, TYPE=, ELSET=`` — labels are arbitrary; nodes
    are numbered in the order of the deck;
  * ``*NSET`` / ``*ELSET`` with labels, names of other sets and ``GENERATE``;
  * ``*SURFACE, TYPE=ELEMENT`` — lines ``elset-or-element, Sk`` (face k of the
    element: for C3D8 and C3D10 the faces of ``elements.HEX8`` / ``TET10``, which
    follow the same S1..S6 / S1..S4 numbering);
  * ``*SOLID SECTION, ELSET=, MATERIAL=``; ``*MATERIAL, NAME=`` with ``*ELASTIC``
    (isotropic E, nu) and ``*PLASTIC`` (isotropic hardening table: yield stress,
    plastic strain -> ``J2Plasticity``);
  * ``*STEP`` (``NAME=``, ``INC=``) ... ``*END STEP``; ``*STATIC`` (initial
    increment, step time, minimum, maximum increment; defaults 1, 1, 1e-5, 1);
  * ``*BOUNDARY`` (before the first step or inside one; ``node|nset, first dof[,
    last dof[, value]]`` or ``node|nset, ENCASTRE|PINNED|XSYMM|YSYMM|ZSYMM``;
    ``OP=NEW`` drops the boundary conditions of earlier steps);
  * ``*CLOAD`` (``node|nset, dof, value``; ``OP=NEW``) and ``*DSLOAD`` (``surface,
    P, pressure``; a pressure replaces an earlier one on the same surface).

Boundary conditions and loads carry over from step to step as in the reference
(a later value of the same node and DOF wins).
"""
import os

import numpy as np

from . import elements, loads, surfaces
from .materials import J2Plasticity, LinearElastic
from .model import Model
from .solvers import Step

_SYM = {"ENCASTRE": (0, 1, 2), "PINNED": (0, 1, 2), "XSYMM": (0,), "YSYMM": (1,), "ZSYMM": (2,)}
_UNSUPPORTED_STEPS = ("DYNAMIC", "FREQUENCY", "BUCKLE", "HEAT TRANSFER", "VISCO", "COUPLED TEMPERATURE-DISPLACEMENT")


def _lines(path):
    base = os.path.dirname(os.path.abspath(path))
    with open(path, errors="replace") as f:
        for line in f:
            s = line.strip()
            if s.upper().startswith("*INCLUDE"):
                for q in (x.strip() for x in s.split(",")[1:]):
                    if q.upper().startswith("INPUT"):
                        yield from _lines(os.path.join(base, q.split("=", 1)[1].strip().strip('"')))
                continue
            yield s


def _cards(path):
    """[(KEYWORD, {PARAM: value or True}, [[field, ...], ...])] of a deck."""
    cards = []
    for s in _lines(path):
        if not s or s.startswith("**"):
            continue
        if s.startswith("*"):
            parts = [p.strip() for p in s[1:].split(",")]
            params = {}
            for p in parts[1:]:
                if "=" in p:
                    k, v = p.split("=", 1)
                    params[k.strip().upper()] = v.strip().strip('"')
                elif p:
                    params[p.upper()] = True
            cards.append((parts[0].upper(), params, []))
        elif cards:
            cards[-1][2].append([t.strip() for t in s.rstrip(",").split(",")])
    return cards


def _num(x, default=0.0):
    try:
        return float(x)
    except (TypeError, ValueError):
        return default


def _etype(name):
    n = name.upper()
    if n.startswith("C3D10"):
        return elements.TET10
    if n.startswith("C3D8") and not n.startswith("C3D8_"):
        return elements.HEX8
    raise NotImplementedError(f"element type {name} is outside the solid C3D8 / C3D10 path")


class InpDeck:
    """The parsed deck: ``X`` (nn, 3), ``node_ids`` (labels), ``blocks`` — one
    (etype, conn (ne, nnode) node indices, element labels, material) per section —,
    ``nsets`` / ``elsets`` (labels), ``surfaces`` ({name: [(element label, face)]}),
    ``steps`` (dicts)."""

    def __init__(self, path):
        self.path = path
        self.nodes = {}                     # label -> index
        xs = []
        self.elems = {}                     # label -> (etype, node labels)
        self.nsets, self.elsets, self.surfaces = {}, {}, {}
        self.materials, self.sections = {}, []
        self.initial_bcs, self.steps = [], []
        mat = step = None
        for kw, p, data in _cards(path):
            if kw == "NODE":
                for d in data:
                    lab = int(d[0])
                    self.nodes[lab] = len(xs)
                    xs.append([_num(v) for v in (d[1:4] + ["0", "0", "0"])[:3]])
                    if "NSET" in p:
                        self.nsets.setdefault(p["NSET"].upper(), []).append(lab)
            elif kw == "ELEMENT":
                et = _etype(str(p.get("TYPE", "")))
                for d in data:
                    lab = int(d[0])
                    self.elems[lab] = (et, [int(v) for v in d[1:] if v])
                    if "ELSET" in p:
                        self.elsets.setdefault(p["ELSET"].upper(), []).append(lab)
            elif kw in ("NSET", "ELSET"):
                sets = self.nsets if kw == "NSET" else self.elsets
                name = str(p[kw]).upper()
                vals = sets.setdefault(name, [])
                if "GENERATE" in p:
                    for d in data:
                        a, b = int(d[0]), int(d[1])
                        c = int(d[2]) if len(d) > 2 and d[2] else 1
                        vals.extend(range(a, b + 1, c))
                else:
                    for d in data:
                        for v in d:
                            if not v:
                                continue
                            if v.lstrip("-").isdigit():
                                vals.append(int(v))
                            else:
                                vals.extend(sets.get(v.upper(), []))
            elif kw == "SURFACE":
                if str(p.get("TYPE", "ELEMENT")).upper() != "ELEMENT":
                    raise NotImplementedError("only element-face surfaces are supported")
                name = str(p["NAME"]).upper()
                rec = self.surfaces.setdefault(name, [])
                for d in data:
                    face = int(d[1].upper().lstrip("S")) - 1
                    ref = d[0]
                    labs = [int(ref)] if ref.isdigit() else self.elsets.get(ref.upper(), [])
                    rec.extend((lab, face) for lab in labs)
            elif kw == "SOLID SECTION":
                self.sections.append((str(p["ELSET"]).upper(), str(p["MATERIAL"]).upper()))
            elif kw == "MATERIAL":
                mat = self.materials.setdefault(str(p["NAME"]).upper(), {})
            elif kw == "ELASTIC" and mat is not None:
                flat = [_num(x) for d in data for x in d if x]
                mat["E"], mat["nu"] = flat[0], flat[1]
            elif kw == "PLASTIC" and mat is not None:
                hard = str(p.get("HARDENING", "ISOTROPIC")).upper()
                if hard != "ISOTROPIC":
                    raise NotImplementedError(f"*PLASTIC, HARDENING={hard}")
                mat["table"] = [[_num(d[0]), _num(d[1])] for d in data]
            elif kw == "STEP":
                step = dict(name=p.get("NAME", f"Step-{len(self.steps) + 1}"), max_inc=int(_num(p.get("INC", 1000))),
                            dt_init=1.0, time=1.0, dt_min=1e-5, dt_max=1.0, bc=[], bc_new=False, cload=[],
                            dsload=[], load_new=False)
            elif kw == "STATIC" and step is not None:
                if "RIKS" in p:
                    raise NotImplementedError("*STATIC, RIKS")
                vals = [_num(x) for x in data[0] if x] if data else []
                step["dt_init"], step["time"], step["dt_min"], step["dt_max"] = (vals + [1.0, 1.0, 1e-5, 1.0][len(vals):])[:4]
            elif kw in _UNSUPPORTED_STEPS and step is not None:
                raise NotImplementedError(f"*{kw} steps are outside the static structural path")
            elif kw == "BOUNDARY":
                if step is None:
                    self.initial_bcs.append(data)
                else:
                    step["bc_new"] |= str(p.get("OP", "")).upper() == "NEW"
                    step["bc"].append(data)
            elif kw == "CLOAD" and step is not None:
                step["load_new"] |= str(p.get("OP", "")).upper() == "NEW"
                step["cload"].append(data)
            elif kw == "DSLOAD" and step is not None:
                step["load_new"] |= str(p.get("OP", "")).upper() == "NEW"
                step["dsload"].append(data)
            elif kw == "END STEP" and step is not None:
                self.steps.append(step)
                step = None
        self.X = np.asarray(xs, dtype=np.float64).reshape(-1, 3)
        self.node_ids = np.array(sorted(self.nodes, key=self.nodes.get), dtype=np.int64)
        self._build_blocks()

    # ---------------------------------------------------------------- sets
    def node_indices(self, ref):
        """Node indices of a node label or an NSET name."""
        if isinstance(ref, (int, np.integer)) or str(ref).lstrip("-").isdigit():
            return np.array([self.nodes[int(ref)]], dtype=np.int64)
        labs = self.nsets.get(str(ref).upper())
        if labs is None:
            raise KeyError(f"unknown node set {ref}")
        return np.array([self.nodes[lab] for lab in labs], dtype=np.int64)

    def _build_blocks(self):
        self.blocks = []
        assigned = set()
        for elset, mname in self.sections:
            labs = [lab for lab in self.elsets.get(elset, []) if lab in self.elems]
            by_type = {}
            for lab in labs:
                by_type.setdefault(self.elems[lab][0].name, []).append(lab)
            m = self.materials.get(mname, {})
            if "E" not in m:
                raise ValueError(f"material {mname} has no *ELASTIC data")
            mat = (J2Plasticity(m["E"], m["nu"], m["table"]) if "table" in m else LinearElastic(m["E"], m["nu"]))
            for tname, tl in by_type.items():
                et = self.elems[tl[0]][0]
                conn = np.array([[self.nodes[n] for n in self.elems[lab][1][:et.nnode]] for lab in tl], dtype=np.int32)
                self.blocks.append(dict(etype=et, conn=conn, labels=np.array(tl, dtype=np.int64), material=mat,
                                        elset=elset))
                assigned.update(tl)
        missing = len(self.elems) - len(assigned)
        if missing:
            raise ValueError(f"{missing} elements have no *SOLID SECTION")
        self._where = {}
        for bi, b in enumerate(self.blocks):
            for i, lab in enumerate(b["labels"]):
                self._where[int(lab)] = (bi, i)

    # ---------------------------------------------------------------- loads
    def _bc_items(self, data):
        out = {}
        for d in data:
            if len(d) >= 2 and d[1].upper() in _SYM:
                dofs, val = _SYM[d[1].upper()], 0.0
            else:
                a = int(_num(d[1]))
                b = int(_num(d[2])) if len(d) > 2 and d[2] else a
                val = _num(d[3]) if len(d) > 3 and d[3] else 0.0
                dofs = [k - 1 for k in range(a, b + 1) if k <= 3]
            for n in self.node_indices(d[0]):
                for k in dofs:
                    out[(int(n), k)] = val
        return out

    def surface(self, name):
        """The facets of an element surface as a :class:`surfaces.Surface`, each
        oriented away from its element (gfem/surfaces.py:150-179)."""
        groups = {}
        for lab, face in self.surfaces[str(name).upper()]:
            bi, i = self._where[int(lab)]
            b = self.blocks[bi]
            loc = b["etype"].faces[face]
            g = groups.setdefault(len(loc), ([], []))
            g[0].append(b["conn"][i, loc])
            g[1].append(self.X[b["conn"][i, :b["etype"].ncorner]].mean(0))
        s = surfaces.Surface(name=name)
        for nf, (fac, cen) in groups.items():
            ft = surfaces.FACETS[nf]
            s.add(ft, surfaces.orient_outward(self.X, ft, np.asarray(fac, dtype=np.int64), np.asarray(cen)))
        return s

    def model(self):
        m = Model(self.X)
        for b in self.blocks:
            m.add_block(b["conn"], b["etype"], b["material"], name=b["elset"])
        return m

    def step_objects(self):
        """The deck's steps as :class:`solvers.Step` (boundary conditions and loads
        accumulated over the steps)."""
        bcs0 = {}
        for data in self.initial_bcs:
            bcs0.update(self._bc_items(data))
        bcs, cl, ds, out = dict(bcs0), {}, {}, []
        for st in self.steps:
            if st["bc_new"]:
                bcs = dict(bcs0)
            for data in st["bc"]:
                bcs.update(self._bc_items(data))
            if st["load_new"]:
                cl, ds = {}, {}
            for data in st["cload"]:
                for d in data:
                    for n in self.node_indices(d[0]):
                        cl[(int(n), int(_num(d[1])) - 1)] = _num(d[2])
            for data in st["dsload"]:
                for d in data:
                    if d[1].upper() != "P":
                        raise NotImplementedError(f"*DSLOAD type {d[1]}")
                    ds[d[0].upper()] = _num(d[2])
            f = np.zeros(3 * len(self.X))
            for name, pval in ds.items():
                f += loads.pressure_vector(self.X, self.surface(name), pval)
            out.append(Step(name=st["name"], time_period=st["time"], dt_init=st["dt_init"], dt_min=st["dt_min"],
                            dt_max=st["dt_max"], max_inc=st["max_inc"], bcs=_grouped(bcs), loads=_grouped(cl),
                            dloads=[f] if ds else []))
        return out


def _grouped(items):
    """{(node, dof): value} -> [(nodes, dof, value)], one entry per (dof, value)."""
    g = {}
    for (n, k), v in items.items():
        g.setdefault((k, v), []).append(n)
    return [(np.array(sorted(ns), dtype=np.int64), k, v) for (k, v), ns in g.items()]


def read_inp(path):
    """(Model, [Step]) of an input deck (gfem/io/inp.py:639-643)."""
    d = InpDeck(path)
    return d.model(), d.step_objects()
