"""ctypes binding of libf3r_b200.so (the C ABI in include/f3r_b200.h).

The library is loaded from this package directory and nowhere else; a missing
library raises instead of falling back to anything.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libf3r_b200.so")

F3R_SUCCESS = 0
STATUS = {0: "SUCCESS", 1: "INVALID_VALUE", 2: "CUDA", 3: "OUT_OF_MEMORY", 5: "BREAKDOWN", 7: "TIMEOUT",
          8: "UNSUPPORTED", 9: "NO_DEVICE"}
F64, F32, F16 = 0, 1, 2
SELL_INDEX16 = 1 << 8
SELL_CSR = 1 << 10
FORMAT_SELL, FORMAT_CSR = 0, 1
SELL_ALIGNED = 1 << 9
PRECOND_SDAINV, PRECOND_ILU0_BJ, PRECOND_ILU0_JACOBI, PRECOND_ILU0_BAJ, PRECOND_ILU0_LEVEL = 0, 1, 2, 3, 4
TRSV_LOWER, TRSV_LOWER_D, TRSV_D_UPPER = 0, 1, 2
TRSV_JACOBI, TRSV_BAJ = 0, 1


class F3RError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"f3r_b200 {STATUS.get(status, status)}: {msg}")
        self.status = status


class CSR(C.Structure):
    _fields_ = [("nrows", C.c_int32), ("ncols", C.c_int32), ("nnz", C.c_int32),
                ("rptr", C.POINTER(C.c_int32)), ("idx", C.POINTER(C.c_int32)), ("val", C.POINTER(C.c_double))]


class Params(C.Structure):
    _fields_ = [("m_outer", C.c_int32), ("max_restarts", C.c_int32), ("m2", C.c_int32), ("m3", C.c_int32),
                ("m4", C.c_int32), ("c", C.c_int32), ("precond", C.c_int32), ("ilu_blocks", C.c_int32),
                ("sdainv_tol", C.c_double), ("acc", C.c_double), ("sell_c", C.c_int32), ("sell_sigma", C.c_int32),
                ("rel_tol", C.c_double), ("half_scale_log2", C.c_int32), ("use_graphs", C.c_int32),
                ("sell_index16", C.c_int32), ("static_weight", C.c_double), ("trsv_iters", C.c_int32),
                ("format", C.c_int32), ("trsv_omega", C.c_double), ("inner_sstep", C.c_int32),
                ("sell_align", C.c_int32), ("sell_autotune", C.c_int32), ("half_m", C.c_int32),
                ("diag_load", C.c_int32), ("reserved", C.c_int32 * 5)]


class Result(C.Structure):
    _fields_ = [("is_solved", C.c_int32), ("res_iter", C.c_int32), ("res_nrm2", C.c_double),
                ("impl_rel_res", C.c_double), ("expl_rel_res", C.c_double), ("restarts", C.c_int32),
                ("reserved0", C.c_int32), ("inner_applications", C.c_int64), ("solve_seconds", C.c_double),
                ("kernel_launches", C.c_int64)]


class SellInfo(C.Structure):
    _fields_ = [("nrows", C.c_int32), ("ncols", C.c_int32), ("nnz", C.c_int32), ("slice_height", C.c_int32),
                ("sigma", C.c_int32), ("nslices", C.c_int32), ("nnz_padded", C.c_int64), ("max_width", C.c_int32),
                ("dtypes", C.c_int32), ("index_bits", C.c_int32)]


class TuneEntry(C.Structure):
    _fields_ = [("warps", C.c_int32), ("stages", C.c_int32), ("kc", C.c_int32), ("index_bits", C.c_int32),
                ("is_default", C.c_int32), ("reserved", C.c_int32), ("microseconds", C.c_double),
                ("gbs_algorithmic", C.c_double)]


COND_FN = C.CFUNCTYPE(C.c_int, C.c_int32, C.c_double, C.c_void_p)

_vp = C.c_void_p
_pp = C.POINTER(C.c_void_p)

# name -> (restype, argtypes); every entry point of include/f3r_b200.h
SIGNATURES = {
    "f3r_last_error_string": (C.c_char_p, []),
    "f3r_status_string": (C.c_char_p, [C.c_int]),
    "f3r_host_matrix_from_csr": (C.c_int, [C.POINTER(CSR), _pp]),
    "f3r_host_matrix_view": (C.c_int, [_vp, C.POINTER(CSR)]),
    "f3r_host_matrix_destroy": (None, [_vp]),
    "f3r_problem_stencil27": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_double, _pp]),
    "f3r_problem_diffusion7": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_uint64, _pp]),
    "f3r_host_scaling": (C.c_int, [_vp]),
    "f3r_host_spmv": (C.c_int, [C.POINTER(CSR), _vp, _vp]),
    "f3r_random_uniform": (C.c_int, [C.c_uint64, C.c_double, C.c_double, C.c_int64, _vp]),
    "f3r_mm_read": (C.c_int, [C.c_char_p, C.POINTER(_vp)]),
    "f3r_trsv_create": (C.c_int, [_vp, C.POINTER(CSR), C.c_int32, C.c_int32, C.c_int32, C.c_double, C.POINTER(_vp)]),
    "f3r_trsv_solve": (C.c_int, [_vp, _vp, _vp]),
    "f3r_trsv_destroy": (None, [_vp]),
    "f3r_mm_read_vector": (C.c_int, [C.c_char_p, C.c_int64, _vp]),
    "f3r_mm_read_rhs": (C.c_int, [C.c_char_p, C.c_int64, _vp, C.POINTER(C.c_int32)]),
    "f3r_mm_write": (C.c_int, [C.c_char_p, C.POINTER(CSR)]),
    "f3r_mm_write_vector": (C.c_int, [C.c_char_p, C.c_int64, _vp]),
    "f3r_host_sdainv": (C.c_int, [C.POINTER(CSR), C.c_double, C.c_double, _pp, _pp]),
    "f3r_host_ilu0_bj": (C.c_int, [C.POINTER(CSR), C.c_int32, C.c_double, _pp, _pp]),
    "f3r_context_create": (C.c_int, [C.c_int32, _pp]),
    "f3r_context_destroy": (None, [_vp]),
    "f3r_context_set_stream": (C.c_int, [_vp, _vp]),
    "f3r_context_synchronize": (C.c_int, [_vp]),
    "f3r_sell_create": (C.c_int, [_vp, C.POINTER(CSR), C.c_int32, C.c_int32, C.c_int32, _pp]),
    "f3r_sell_info_get": (C.c_int, [_vp, C.POINTER(SellInfo)]),
    "f3r_sell_destroy": (None, [_vp]),
    "f3r_sell_tune": (C.c_int, [_vp, C.c_int, C.c_int32, C.POINTER(TuneEntry), C.c_int32, C.POINTER(C.c_int32)]),
    "f3r_sell_operate": (C.c_int, [_vp, C.c_int, C.c_int, _vp, C.c_int, _vp]),
    "f3r_sell_compute_residual": (C.c_int, [_vp, C.c_int, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp]),
    "f3r_context_wait_probe": (C.c_int, [_vp, C.c_int32, C.c_int32]),
    "f3r_dot": (C.c_int, [_vp, C.c_int, C.c_int64, _vp, _vp, C.POINTER(C.c_double)]),
    "f3r_dot_noalloc": (C.c_int, [C.c_int, C.c_int64, _vp, _vp, _vp, _vp]),
    "f3r_params_default": (None, [C.POINTER(Params)]),
    "f3r_solver_create": (C.c_int, [_vp, C.POINTER(CSR), C.POINTER(Params), _pp]),
    "f3r_solver_solve": (C.c_int, [_vp, _vp, _vp, COND_FN, _vp, C.POINTER(Result)]),
    "f3r_solver_solve_multi": (C.c_int, [_vp, C.c_int32, _vp, C.c_int64, _vp, C.c_int64, COND_FN, _vp,
                                         C.POINTER(Result)]),
    "f3r_solve_batch": (C.c_int, [C.c_int32, C.POINTER(_vp), C.POINTER(C.c_int32), C.POINTER(_vp),
                                  C.POINTER(C.c_int64), C.POINTER(_vp), C.POINTER(C.c_int64), COND_FN, _vp,
                                  C.POINTER(Result)]),
    "f3r_solver_info": (C.c_int, [_vp, C.POINTER(SellInfo), C.POINTER(C.c_int32)]),
    "f3r_solver_operate": (C.c_int, [_vp, C.c_int, C.c_int, _vp, C.c_int, _vp]),
    "f3r_solver_destroy": (None, [_vp]),
    "f3r_solver_create_factors": (C.c_int, [_vp, C.POINTER(CSR), C.POINTER(Params), C.POINTER(CSR), C.POINTER(CSR),
                                            _pp]),
    "f3r_batch_create": (C.c_int, [_vp, C.c_int32, C.POINTER(C.POINTER(CSR)), C.POINTER(Params),
                                   C.POINTER(C.POINTER(CSR)), C.POINTER(C.POINTER(CSR)), _pp]),
    "f3r_batch_solve": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(_vp), COND_FN, _vp, C.POINTER(Result)]),
    "f3r_batch_info": (C.c_int, [_vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "f3r_batch_destroy": (None, [_vp]),
    "f3r_learned_create": (C.c_int, [_vp, C.c_int32, C.c_uint64, _pp]),
    "f3r_learned_destroy": (None, [_vp]),
    "f3r_learned_params": (C.c_int, [_vp, _vp, C.c_int32, C.POINTER(C.c_int64)]),
    "f3r_learned_set_data": (C.c_int, [_vp, C.POINTER(CSR), C.c_int32, C.c_int32, C.POINTER(CSR), C.POINTER(CSR),
                                       C.c_int32, _vp, _vp]),
    "f3r_learned_evaluate": (C.c_int, [_vp, C.POINTER(C.c_double), _vp]),
    "f3r_learned_train": (C.c_int, [_vp, C.c_int32, C.c_double, _vp]),
    "f3r_learned_correct": (C.c_int, [_vp, C.POINTER(CSR), C.c_int32, C.c_int32, C.POINTER(CSR), C.POINTER(CSR),
                                      C.c_int32, _vp, _vp, _vp]),
    "f3r_learned_time_inference": (C.c_int, [_vp, C.POINTER(CSR), C.c_int32, C.c_int32, C.POINTER(CSR),
                                             C.POINTER(CSR), C.c_int32, C.c_int32, C.POINTER(C.c_double)]),
}

_lib = None


def lib() -> C.CDLL:
    """Load libf3r_b200.so from the package directory (raises if absent)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m f3r_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != F3R_SUCCESS:
        msg = lib().f3r_last_error_string()
        raise F3RError(status, msg.decode() if msg else "")
