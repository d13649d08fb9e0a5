"""Writes tests/golden/cantilever_c3d10.inp, the input-deck fixture of the deck
reader tests: a jittered C3D10 cantilever 4 x 1 x 1 (4 x 2 x 2 hexahedra, Kuhn
split) with non-contiguous node and element labels, node sets (one generated),
an element-face surface on the top face written per face index, a material,
a section and one static step with an encastre, a pressure on the surface and a
concentrated tip load.  ``case()`` returns the arrays the deck is written from,
so the tests can check the reader against them.

Run: python tests/golden/make_deck.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from exfem_b200 import elements, mesh  # noqa: E402

DECK = os.path.join(HERE, "cantilever_c3d10.inp")
E, NU, PRESSURE, TIP_LOAD = 210000.0, 0.3, -2.0, -5.0


def case():
    X, c = mesh.box_hex(4.0, 1.0, 1.0, 4, 2, 2)
    X = mesh.jitter_interior(X, [1.0, 0.5, 0.5], 0.1, 3)
    X, c = mesh.tet4_to_tet10(*mesh.hex_to_tet4(X, c))
    node_labels = 1000 + 2 * np.arange(len(X))
    elem_labels = 1 + 3 * np.arange(len(c))
    fix = np.nonzero(X[:, 0] < 1e-9)[0]
    tip = int(np.nonzero((X[:, 0] > 4 - 1e-9) & (X[:, 1] > 1 - 1e-9) & (X[:, 2] > 1 - 1e-9))[0][0])
    top = set(np.nonzero(X[:, 2] > 1 - 1e-9)[0].tolist())
    faces = []                                   # (element index, face index) on z = 1
    for e, row in enumerate(c):
        for k, loc in enumerate(elements.TET10.faces):
            if all(int(row[a]) in top for a in loc[:3]):
                faces.append((e, k))
    return dict(X=X, conn=c, node_labels=node_labels, elem_labels=elem_labels, fix=fix, tip=tip, top_faces=faces)


def write(path=DECK):
    d = case()
    X, c, nl, el = d["X"], d["conn"], d["node_labels"], d["elem_labels"]
    out = ["*HEADING", "deck reader fixture: C3D10 cantilever", "** units: N, mm", "*NODE"]
    out += [f"{nl[i]}, {X[i, 0]:.17g}, {X[i, 1]:.17g}, {X[i, 2]:.17g}" for i in range(len(X))]
    out.append("*ELEMENT, TYPE=C3D10, ELSET=BODY")
    out += [f"{el[e]}, " + ", ".join(str(nl[n]) for n in c[e]) for e in range(len(c))]
    out.append("*NSET, NSET=FIX")
    fl = [str(nl[n]) for n in d["fix"]]
    out += [", ".join(fl[i:i + 8]) for i in range(0, len(fl), 8)]
    out += ["*NSET, NSET=TIP", str(nl[d["tip"]])]
    out += ["*NSET, NSET=FIRST_NODES, GENERATE", f"{nl[0]}, {nl[9]}, 2"]
    by_face = {}
    for e, k in d["top_faces"]:
        by_face.setdefault(k, []).append(el[e])
    for k in sorted(by_face):
        out.append(f"*ELSET, ELSET=_TOP_S{k + 1}")
        labs = [str(x) for x in by_face[k]]
        out += [", ".join(labs[i:i + 8]) for i in range(0, len(labs), 8)]
    out.append("*SURFACE, NAME=TOP, TYPE=ELEMENT")
    out += [f"_TOP_S{k + 1}, S{k + 1}" for k in sorted(by_face)]
    out += ["*SOLID SECTION, ELSET=BODY, MATERIAL=STEEL", ",", "*MATERIAL, NAME=STEEL", "*DENSITY", "7.85e-09,",
            "*ELASTIC", f"{E:g}, {NU:g}", "*STEP, NAME=Load, NLGEOM=NO, INC=100", "*STATIC", "1, 1, 1e-05, 1",
            "*BOUNDARY, OP=NEW", "FIX, ENCASTRE", "*DSLOAD, OP=NEW", f"TOP, P, {PRESSURE:g}", "*CLOAD",
            f"TIP, 3, {TIP_LOAD:g}", "*OUTPUT, FIELD, VARIABLE=PRESELECT", "*END STEP"]
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


if __name__ == "__main__":
    write()
    print("wrote", DECK)
