"""ctypes binding of ``libexfem_b200.so`` (the C ABI in include/exfem_b200.h).

The library is built in-tree by ``python -m exfem_b200.build``.  There is no
fallback: if the shared library is missing or cannot be loaded, importing this
module raises, and every public operation of the package fails with it.
"""
import ctypes as C
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libexfem_b200.so")

OK, NOT_CONVERGED = 0, 1
ERR_ARG, ERR_CUDA, ERR_OOM, ERR_TIMEOUT, ERR_NONFINITE, ERR_UNSUPPORTED = -1, -2, -3, -4, -5, -6
C3D8, C3D10 = 0, 1
LINEAR_ELASTIC, J2 = 0, 1
F64, F32, BF16 = 0, 1, 2
ASSEMBLE_GATHER, ASSEMBLE_COLOUR = 0, 1
OP_EBE_F64, OP_MF_F64, OP_MF_F32, OP_CSR_F64 = 0, 1, 2, 3
PC_NONE, PC_JACOBI, PC_AMG, PC_CHEBY = 0, 1, 2, 3
REQ_PENDING, REQ_RUNNING, REQ_DONE, REQ_FAILED, REQ_CANCELLED = 0, 1, 2, 3, 4
MAX_TABLE = 32


class Material(C.Structure):
    _fields_ = [("kind", C.c_int), ("E", C.c_double), ("nu", C.c_double), ("Hk", C.c_double),
                ("ntab", C.c_int), ("sy_tab", C.c_double * MAX_TABLE), ("ep_tab", C.c_double * MAX_TABLE)]


class ExfemError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"exfem status {status}: {msg}")
        self.status = status


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m exfem_b200.build` "
                          "(the CUDA library is required; there is no CPU fallback)")
    return C.CDLL(LIB_PATH)


lib = _load()

P, I64, I32, D, VP = C.c_void_p, C.c_int64, C.c_int, C.c_double, C.c_void_p
_SIGS = {
    "exfem_version": ([], C.c_int),
    "exfem_last_error": ([], C.c_char_p),
    "exfem_block_create": ([C.c_int, C.POINTER(Material), I64, P, I64, P, C.POINTER(VP)], C.c_int),
    "exfem_block_destroy": ([VP], C.c_int),
    "exfem_block_query": ([VP, C.POINTER(I64), C.POINTER(I64), C.POINTER(I32), C.POINTER(I32), C.POINTER(I32),
                           C.POINTER(I32), C.POINTER(I32), C.POINTER(I32), C.POINTER(I64)], C.c_int),
    "exfem_block_gather_plan": ([VP, P], C.c_int),
    "exfem_block_colours": ([VP, P], C.c_int),
    "exfem_block_tile_info": ([VP, C.POINTER(I64), C.POINTER(I64), C.POINTER(I32)], C.c_int),
    "exfem_block_tile_maps": ([VP, P, P, P, P], C.c_int),
    "exfem_block_tile_order": ([VP, C.POINTER(I32), P], C.c_int),
    "exfem_set_tile": ([I32, I32], C.c_int),
    "exfem_get_tile": ([I32, C.POINTER(I32)], C.c_int),
    "exfem_block_set_scale": ([VP, P], C.c_int),
    "exfem_block_set_fixed": ([VP, P], C.c_int),
    "exfem_block_set_lame": ([VP, P, P], C.c_int),
    "exfem_internal_force": ([VP, P, P, P, P, P, C.c_int, VP], C.c_int),
    "exfem_element_stiffness": ([VP, P, P, C.c_int, P, VP], C.c_int),
    "exfem_tangent_update": ([VP, P, P, VP], C.c_int),
    "exfem_tangent_matvec": ([VP, C.c_int, P, P, C.c_int, VP], C.c_int),
    "exfem_tangent_diagonal": ([VP, P, VP], C.c_int),
    "exfem_ebe_matvec": ([VP, P, P, P, C.c_int, VP], C.c_int),
    "exfem_ebe_matvec_bf16_multi": ([VP, P, I32, P, P, I32, VP], C.c_int),
    "exfem_ebe_matvec_multi": ([VP, VP, C.c_int, C.c_int, VP, VP, C.c_int, VP], C.c_int),
    "exfem_multi_pcg": ([VP, VP, C.c_int, VP, VP, C.c_double, C.c_int, VP, VP, VP], C.c_int),
    "exfem_ebe_diagonal": ([VP, P, P, VP], C.c_int),
    "exfem_stresses": ([VP, P, P, P, P, P, VP], C.c_int),
    "exfem_geometric_stiffness": ([VP, P, P, VP], C.c_int),
    "exfem_amg_create": ([C.POINTER(VP)], C.c_int),
    "exfem_amg_destroy": ([VP], C.c_int),
    "exfem_amg_add_level": ([VP, I64, I64, P, P, P, P, P, P, P, P, P, P, D], C.c_int),
    "exfem_amg_set_coarse": ([VP, I64, P], C.c_int),
    "exfem_amg_set_level_rows": ([VP, C.c_int, P], C.c_int),
    "exfem_amg_set_coarse_blocks": ([VP, I64, P, P], C.c_int),
    "exfem_amg_vcycle": ([VP, C.c_int, P, P, VP, P, VP], C.c_int),
    "exfem_amg_vcycle_noalloc": ([VP, C.c_int, P, P, VP, P, VP], C.c_int),
    "exfem_solver_create": ([VP, C.c_int, C.c_int, VP, C.POINTER(VP)], C.c_int),
    "exfem_solver_destroy": ([VP], C.c_int),
    "exfem_solver_set_ke": ([VP, P], C.c_int),
    "exfem_solver_refresh_diagonal": ([VP, VP], C.c_int),
    "exfem_solver_cheby_bound": ([VP, C.POINTER(D)], C.c_int),
    "exfem_solver_set_graph": ([VP, C.c_int, C.c_int], C.c_int),
    "exfem_solver_set_loop": ([VP, C.c_int], C.c_int),
    "exfem_newton_increment": ([VP, VP, VP, VP, VP, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int, VP, VP, VP,
                                VP, VP, VP, VP, VP], C.c_int),
    "exfem_solver_pcg": ([VP, P, P, D, C.c_int, C.POINTER(I32), C.POINTER(D), VP], C.c_int),
    "exfem_solver_mixed": ([VP, P, P, D, D, C.c_int, C.c_int, C.POINTER(I32), C.POINTER(I32), C.POINTER(D), VP],
                           C.c_int),
    "exfem_amg_replicate": ([VP, C.c_int, P, C.c_int, P], C.c_int),
    "exfem_batch_create": ([VP, VP, C.c_int, P, C.POINTER(VP)], C.c_int),
    "exfem_batch_destroy": ([VP], C.c_int),
    "exfem_batch_solve": ([VP, P, P, D, D, C.c_int, C.c_int, P, C.POINTER(I32), P, VP], C.c_int),
    "exfem_host_gather_plan": ([I64, I64, C.c_int, P, P, C.POINTER(I32)], C.c_int),
    "exfem_host_colouring": ([I64, I64, C.c_int, P, P, C.POINTER(I32)], C.c_int),
    "exfem_host_standard_aggregation": ([I64, P, P, P, C.POINTER(I64)], C.c_int),
    "exfem_host_node_adjacency": ([I64, I64, I32, P, C.POINTER(I64), P, P], C.c_int),
    "exfem_host_fit_candidates": ([I64, I32, I32, P, I64, P, P, P], C.c_int),
    "exfem_host_coarse_inverse": ([I64, P, P], C.c_int),
    "exfem_host_filter_pattern": ([I64, P, P, P, C.POINTER(I64), P, P, P], C.c_int),
    "exfem_host_tile_order": ([I64, I64, I32, I32, P, P, P], C.c_int),
    "exfem_host_tile_pairs": ([I64, P, P, P], C.c_int),
    "exfem_host_face_once": ([I64, P, P], C.c_int),
    "exfem_host_tile_maps": ([I64, I64, I32, P, I32, C.POINTER(I64), C.POINTER(I64), P, P, P, P], C.c_int),
    "exfem_block_status": ([VP, VP], C.c_int),
    "exfem_amg_setup_block": ([VP, VP, P, I32, I32, VP], C.c_int),
    "exfem_amg_setup_blocks": ([VP, I32, P, P, I32, I32, VP], C.c_int),
    "exfem_solver_add_block": ([VP, VP], C.c_int),
    "exfem_solver_set_ke_block": ([VP, I32, P], C.c_int),
    "exfem_amg_info": ([VP, I32, P, P, P], C.c_int),
    "exfem_amg_export_level": ([VP, I32, I32, P, P, P, P, P, P, P], C.c_int),
    "exfem_amg_export_coarse": ([VP, P, P], C.c_int),
    "exfem_solver_set_mixed_mode": ([VP, I32, D], C.c_int),
    "exfem_selftest_bounded_wait": ([I32, VP], C.c_int),
    "exfem_block_tile_conn": ([VP, P], C.c_int),
    "exfem_queue_create": ([I32, C.POINTER(VP)], C.c_int),
    "exfem_queue_destroy": ([VP], C.c_int),
    "exfem_queue_submit": ([VP, VP, P, D, C.POINTER(I64)], C.c_int),
    "exfem_queue_poll": ([VP, I64, C.POINTER(I32), C.POINTER(I32), C.POINTER(D)], C.c_int),
    "exfem_queue_wait": ([VP, I64, D, C.POINTER(I32)], C.c_int),
    "exfem_queue_result": ([VP, I64, P, C.POINTER(I32), C.POINTER(I32), C.POINTER(D)], C.c_int),
    "exfem_queue_cancel": ([VP, I64, C.POINTER(I32)], C.c_int),
}
for _name, (_args, _res) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.argtypes = _args
    _f.restype = _res

EXPORTED = tuple(_SIGS)


def last_error():
    m = lib.exfem_last_error()
    return m.decode() if m else ""


def check(status, allow=(OK,)):
    """Raise ExfemError for a negative status; return the status otherwise."""
    if status < 0 or (status not in allow and status != NOT_CONVERGED):
        raise ExfemError(status, last_error())
    return status


def ptr(t):
    """Raw address of a tensor / ndarray (None -> NULL)."""
    if t is None:
        return None
    if isinstance(t, torch.Tensor):
        return t.data_ptr()
    return t.ctypes.data


def stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("exfem_b200 device operations need a CUDA GPU (sm_100a)")
