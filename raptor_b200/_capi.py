"""ctypes binding of include/raptor_b200.h (libraptor_b200.so, in-tree).

Loading fails loudly when the library has not been built: there is no
Python or CPU fallback for any computation.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libraptor_b200.so")

RB_OK = 0
STATUS = {
    0: "RB_OK", -1: "RB_ERR_INVALID", -2: "RB_ERR_CUDA", -3: "RB_ERR_OOM",
    -4: "RB_ERR_BREAKDOWN", -5: "RB_ERR_NOT_CONVERGED", -6: "RB_ERR_NO_DEVICE",
}


class RaptorError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (STATUS.get(code, "?"), code, msg))
        self.code = code


class NotConverged(RaptorError):
    pass


class Breakdown(RaptorError):
    pass


class AmgOpts(C.Structure):
    _fields_ = [
        ("solver", C.c_int), ("strength_type", C.c_int), ("interp_type", C.c_int),
        ("relax_type", C.c_int), ("num_smooth_sweeps", C.c_int), ("max_coarse", C.c_int),
        ("max_levels", C.c_int), ("max_iterations", C.c_int), ("strong_threshold", C.c_double),
        ("relax_weight", C.c_double), ("solve_tol", C.c_double), ("interp_filter", C.c_double),
        ("prolong_weight", C.c_double), ("prolong_smooth_steps", C.c_int),
        ("precision", C.c_int), ("jacobi_compat", C.c_int), ("seed_offset", C.c_int),
        ("fuse_coarse", C.c_int), ("use_graphs", C.c_int), ("const_coef", C.c_int),
        ("coarsen_type", C.c_int), ("num_variables", C.c_int),
    ]


_P = C.c_void_p
_PP = C.POINTER(C.c_void_p)
_D = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_I = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64 = C.c_int64

# name -> (restype, argtypes)
SIGNATURES = {
    "rb_last_error": (C.c_char_p, []),
    "rb_version": (C.c_char_p, []),
    "rb_init": (C.c_int, [C.c_int]),
    "rb_set_stream": (C.c_int, [_P]),
    "rb_synchronize": (C.c_int, []),
    "rb_vec_gather": (C.c_int, [_P, _P, C.c_int, _P]),
    "rb_vec_scatter_add": (C.c_int, [_P, _P, _P, C.c_int]),
    "rb_petsc_read_host": (C.c_int, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                     C.POINTER(_i64), _P, _P, _P]),
    "rb_petsc_write_host": (C.c_int, [C.c_char_p, C.c_int, C.c_int, _i64, _P, _P, _P]),
    "rb_write_petsc": (C.c_int, [_P, C.c_char_p]),
    "rb_csr_create": (C.c_int, [C.c_int, C.c_int, _i64, _P, _P, _P, C.c_int, _PP]),
    "rb_csr_destroy": (C.c_int, [_P]),
    "rb_csr_info": (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(_i64)]),
    "rb_csr_download": (C.c_int, [_P, _P, _P, _P]),
    "rb_csr_device_arrays": (C.c_int, [_P, _PP, _PP, _PP]),
    "rb_csr_sort_diag_first": (C.c_int, [_P]),
    "rb_csr_transpose": (C.c_int, [_P, _PP]),
    "rb_bsr_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _i64, _P, _P, _P, C.c_int,
                                _PP]),
    "rb_bsr_destroy": (C.c_int, [_P]),
    "rb_bsr_info": (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                              C.POINTER(C.c_int), C.POINTER(_i64)]),
    "rb_bsr_download": (C.c_int, [_P, _P, _P, _P]),
    "rb_bsr_spmv": (C.c_int, [_P, _P, _P]),
    "rb_bsr_spmv_append": (C.c_int, [_P, _P, _P]),
    "rb_bsr_residual": (C.c_int, [_P, _P, _P, _P]),
    "rb_bsr_spmv_T": (C.c_int, [_P, _P, _P]),
    "rb_bsr_to_csr": (C.c_int, [_P, _PP]),
    "rb_vec_create": (C.c_int, [C.c_int, _PP]),
    "rb_vec_destroy": (C.c_int, [_P]),
    "rb_vec_size": (C.c_int, [_P, C.POINTER(C.c_int)]),
    "rb_vec_upload": (C.c_int, [_P, _D]),
    "rb_vec_download": (C.c_int, [_P, _D]),
    "rb_vec_set": (C.c_int, [_P, C.c_double]),
    "rb_vec_device_ptr": (C.c_int, [_P, _PP]),
    "rb_vec_copy": (C.c_int, [_P, _P]),
    "rb_vec_axpy": (C.c_int, [_P, _P, C.c_double]),
    "rb_vec_scale": (C.c_int, [_P, C.c_double]),
    "rb_vec_dot": (C.c_int, [_P, _P, C.POINTER(C.c_double)]),
    "rb_vec_norm2": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "rb_spmv": (C.c_int, [_P, _P, _P]),
    "rb_residual": (C.c_int, [_P, _P, _P, _P]),
    "rb_spmv_T": (C.c_int, [_P, _P, _P]),
    "rb_spmv_append": (C.c_int, [_P, _P, _P]),
    "rb_diffusion_stencil_2d": (C.c_int, [C.c_double, C.c_double, _D]),
    "rb_laplace_stencil_27pt": (C.c_int, [_D]),
    "rb_stencil_grid": (C.c_int, [_D, _I, C.c_int, _PP]),
    "rb_read_petsc": (C.c_int, [C.c_char_p, _PP]),
    "rb_read_mm": (C.c_int, [C.c_char_p, _PP]),
    "rb_read_par_mm": (C.c_int, [C.c_char_p, _PP]),
    "rb_write_mm": (C.c_int, [C.c_void_p, C.c_char_p]),
    "rb_mm_read_host": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.POINTER(C.c_int),
                                  C.POINTER(C.c_int), C.POINTER(C.c_int64), C.c_void_p,
                                  C.c_void_p, C.c_void_p]),
    "rb_mm_write_host": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int64, C.c_void_p,
                                   C.c_void_p, C.c_void_p]),
    "rb_strength": (C.c_int, [_P, C.c_int, C.c_double, _PP]),
    "rb_split_pmis": (C.c_int, [_P, _P, _I]),
    "rb_split": (C.c_int, [_P, C.c_int, _P, _I]),
    "rb_interpolation": (C.c_int, [_P, _P, _I, C.c_int, C.c_double, _PP]),
    "rb_mis2": (C.c_int, [_P, _P, _I]),
    "rb_aggregate": (C.c_int, [_P, _P, _I, _P, _I, C.POINTER(C.c_int)]),
    "rb_fit_candidates": (C.c_int, [C.c_int, C.c_int, _I, _D, _D, _PP]),
    "rb_jacobi_prolongation": (C.c_int, [_P, _P, C.c_double, C.c_int, _PP]),
    "rb_spgemm": (C.c_int, [_P, _P, _PP]),
    "rb_rap": (C.c_int, [_P, _P, C.c_int, _PP]),
    "rb_amg_default_opts": (None, [C.POINTER(AmgOpts)]),
    "rb_amg_setup": (C.c_int, [_P, C.POINTER(AmgOpts), _P, _PP]),
    "rb_amg_destroy": (C.c_int, [_P]),
    "rb_amg_num_levels": (C.c_int, [_P, C.POINTER(C.c_int)]),
    "rb_amg_level_info": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int), C.POINTER(_i64), C.POINTER(_i64)]),
    "rb_amg_level_matrix": (C.c_int, [_P, C.c_int, C.c_int, _PP]),
    "rb_amg_level_states": (C.c_int, [_P, C.c_int, _I]),
    "rb_amg_cycle": (C.c_int, [_P, _P, _P]),
    "rb_amg_solve": (C.c_int, [_P, _P, _P, C.POINTER(C.c_int), _P, C.c_int]),
    "rb_amg_cycle_profile": (C.c_int, [_P, _P, C.c_int, C.POINTER(C.c_int)]),
    "rb_amg_time_operator": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]),
    "rb_amg_setup_seconds": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "rb_amg_level_lanes": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "rb_amg_level_storage": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int)]),
    "rb_amg_level_const_coef": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int)]),
    "rb_amg_tail_info": (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "rb_amg_level_fused_first": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int)]),
    "rb_amg_tail_timings": (C.c_int, [_P, _D, C.c_int, C.POINTER(C.c_int)]),
    "rb_residual_norm_noalloc": (C.c_int, [C.c_int, _P, _P, _P, _P, _P, _P, _P]),
    "rb_launch_count": (C.c_int, [C.POINTER(C.c_int64)]),
    "rb_device_alloc_count": (C.c_int, [C.POINTER(C.c_int64)]),
    "rb_pcg": (C.c_int, [_P, _P, _P, _P, C.c_double, C.c_int, C.c_int, _P, C.c_int, C.POINTER(C.c_int)]),
    "rb_fv_assemble": (C.c_int, [C.c_int, C.c_int, _P, _PP]),
    "rb_fv_backward": (C.c_int, [C.c_int, C.c_int, _P, _P, _P, _P]),
    "rb_sddmm": (C.c_int, [_P, _P, _P, C.c_double, _P]),
    "rb_adjoint_solve": (C.c_int, [_P, _P, _P, _P, C.c_double, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "rb_batch_setup": (C.c_int, [C.c_int, _P, _P, _PP]),
    "rb_batch_destroy": (C.c_int, [_P]),
    "rb_batch_info": (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int64), C.POINTER(C.c_int)]),
    "rb_batch_offsets": (C.c_int, [_P, _P, _P]),
    "rb_batch_cycle": (C.c_int, [_P, _P, _P]),
    "rb_batch_pcg": (C.c_int, [_P, _P, _P, C.c_double, C.c_int, _I, _D]),
    "rb_batch_host_waits": (C.c_int, [_P, C.POINTER(C.c_int)]),
    "rb_amg_cycle_block": (C.c_int, [_P, _P, _P, C.c_int]),
    "rb_pcg_block": (C.c_int, [_P, _P, _P, _P, C.c_int, C.c_double, C.c_int, _I, _D]),
    "rb_cg": (C.c_int, [_P, _P, _P, C.c_double, C.c_int, _P, C.c_int, C.POINTER(C.c_int)]),
    "rb_bicgstab": (C.c_int, [_P, _P, _P, _P, C.c_double, C.c_int, _P, C.c_int, C.POINTER(C.c_int)]),
}

_lib = None


def lib():
    """Load libraptor_b200.so (raises ImportError when it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libraptor_b200.so is not built; run `python -m raptor_b200.build` "
                              "(the library has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error():
    return (lib().rb_last_error() or b"").decode()


def check(code):
    if code != RB_OK:
        msg = last_error()
        if code == -5:
            raise NotConverged(code, msg)
        if code == -4:
            raise Breakdown(code, msg)
        raise RaptorError(code, msg)
    return code


def exported_symbols():
    return list(SIGNATURES)
