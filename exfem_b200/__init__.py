"""exfem_b200 — B200-native structural hot path of EXFEM (``gfem`` 0.3.0).

Hand-written sm_100a CUDA kernels (``csrc/``, built into ``libexfem_b200.so``
behind the C ABI in ``include/exfem_b200.h``) for the C3D8 (B-bar) and C3D10
element force / tangent kernels with linear-elastic and J2 materials, the
element-by-element matrix-free tangent product, the smoothed-aggregation
V-cycle, PCG with device-resident scalars and graph-captured iterations, and
FP32-inside-FP64 iterative refinement.  The Python modules mirror the
reference's element, material, model, linear-algebra and static-solver
interfaces so its Newton loop can run on them unchanged.
"""
from . import _lib  # noqa: F401  (fails loudly when the CUDA library is missing)
from .elements import ELEMENTS, HEX8, TET10  # noqa: F401
from . import checkpoint, deck, eigen, loads, optimize, results, surfaces  # noqa: F401
from .linalg import AMG, DeviceAMG, NativeSolver, pcg  # noqa: F401
from .materials import J2Plasticity, LinearElastic, from_props  # noqa: F401
from .model import Block, Model  # noqa: F401
from .solvers import Monitor, State, StaticSolver, Step  # noqa: F401

__version__ = "0.1.0"
