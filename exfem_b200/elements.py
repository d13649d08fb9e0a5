"""Element types of the hot path (drop-in names of ``gfem.elements``).

Only the two solid elements the structural hot path covers are provided:

  * ``HEX8`` — "C3D8", 8-node hexahedron, 2x2x2 Gauss points at the corners
    scaled by 1/sqrt(3), unit weights, B-bar for small strain
    (gfem/elements.py:113-125, ``fbar=True``);
  * ``TET10`` — "C3D10", 10-node tetrahedron, 4-point rule with barycentric
    a = 0.5854101966249685, b = 0.1381966011250105, weights 1/24
    (gfem/elements.py:166-179).

The shape-function arithmetic itself lives in the CUDA kernels
(``csrc/element_math.cuh``); these objects carry the identifiers and the
topology the host code needs.
"""
from . import _lib


class ElementType:
    def __init__(self, name, code, nnode, ngp, ncorner, faces, fbar=False):
        self.name, self.code = name, code
        self.nnode, self.ngp, self.ncorner = nnode, ngp, ncorner
        self.faces = [list(f) for f in faces]
        self.fbar = fbar
        self.nd = 3 * nnode

    def __repr__(self):
        return f"<ElementType {self.name}>"


HEX_FACES = [[0, 1, 2, 3], [4, 7, 6, 5], [0, 4, 5, 1], [1, 5, 6, 2], [2, 6, 7, 3], [3, 7, 4, 0]]
TET10_FACES = [[0, 1, 2, 4, 5, 6], [0, 3, 1, 7, 8, 4], [1, 3, 2, 8, 9, 5], [2, 3, 0, 9, 7, 6]]

HEX8 = ElementType("C3D8", _lib.C3D8, 8, 8, 8, HEX_FACES, fbar=True)
TET10 = ElementType("C3D10", _lib.C3D10, 10, 4, 4, TET10_FACES)

# gfem/elements.py:194-197 aliases that map onto the two covered types
ELEMENTS = {"C3D8": HEX8, "C3D8H": HEX8, "C3D8R": HEX8, "C3D8I": HEX8,
            "C3D10": TET10, "C3D10M": TET10, "C3D10H": TET10}
BY_NNODE = {8: HEX8, 10: TET10}
