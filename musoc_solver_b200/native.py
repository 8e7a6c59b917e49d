"""ctypes binding of ``libsevp_b200.so`` (declared in ``include/sevp_b200.h``).

The library is the product: every computation below runs in its sm_100a
kernels.  If the library is missing or no CUDA device is present the calls
fail loudly; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsevp_b200.so")

SEVP_OK = 0
SEVP_MAXITER = 1
SEVP_BREAKDOWN = 2
SEVP_NONFINITE = 3
SEVP_TIMEOUT = 4
SEVP_BAD_ARG = 5
SEVP_CUDA_ERROR = 6
SEVP_SINGULAR = 7
SEVP_NONSYMMETRIC = 8

METHOD_PCG = 0   # PCG, two grid passes per iteration
METHOD_CHEB = 1  # one-launch Chebyshev iteration (mixed precision, needs bounds)

PASS_A_TILES = 0    # stencil pass on tensor-copied shared-memory tiles
PASS_A_COLUMNS = 1  # stencil pass walking columns with warp shuffles
PASS_B_REGISTERS = 0  # tile pass loading each task into registers
PASS_B_STAGED = 1     # tile pass with tensor-copied shared-memory task stages

GUESS_ZERO, GUESS_PREVIOUS, GUESS_LINEAR, GUESS_LEARNED = 0, 1, 2, 3


class SevpError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = f"{what}: {status_string(status)} (status {status})"
        err = last_error()
        if err:
            msg += f" [{err}]"
        super().__init__(msg)


class Tiling(C.Structure):
    _fields_ = [("tile_m", C.c_int), ("tile_h", C.c_int), ("sub_rows", C.c_int),
                ("sub_rows_by_tile_row", C.POINTER(C.c_int)),
                ("sub_rows_by_tile", C.POINTER(C.c_int)), ("growth_limit", C.c_double)]


class SolveOpts(C.Structure):
    _fields_ = [("precision", C.c_int), ("tol", C.c_double), ("max_iter", C.c_int),
                ("inner_tol", C.c_double), ("use_guess", C.c_int), ("check_every", C.c_int),
                ("precond_fp32", C.c_int), ("tol_abs", C.c_int), ("method", C.c_int),
                ("restart_inner", C.c_int)]


class FsOptions(C.Structure):
    """sevp_fs_options: the options of p_sevp_pcg_."""
    _fields_ = [("precision", C.c_int), ("tol_abs", C.c_int), ("tol", C.c_double),
                ("max_iter", C.c_int), ("inner_tol", C.c_double), ("tile_m", C.c_int),
                ("tile_h", C.c_int), ("growth_limit", C.c_double), ("schwarz", C.c_int),
                ("verify", C.c_int), ("method", C.c_int)]


class Report(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("refinements", C.c_int),
                ("rel_residual", C.c_double), ("abs_residual", C.c_double), ("bnorm", C.c_double),
                ("ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None

# Exported symbols with their ctypes signatures.  Fortran-style entry points
# take every argument by reference.
P = C.c_void_p
IP = C.POINTER(C.c_int)
DP = C.POINTER(C.c_double)
_SIGS = {
    # native API
    "sevp_status_string": ([C.c_int], C.c_char_p),
    "sevp_last_error": ([], C.c_char_p),
    "sevp_last_status": ([], C.c_int),
    "sevp_set_periodic_we": ([C.c_int], None),
    "sevp_get_periodic_we": ([], C.c_int),
    "sevp_dropin_cache": ([C.c_int], C.c_int),
    "sevp_fs_default_options": ([P], None),
    "sevp_fs_set_options": ([P], C.c_int),
    "sevp_fs_last_report": ([P], C.c_int),
    "sevp_fs_release": ([], C.c_int),
    "sevp_row_symmetrize": ([P] * 5 + [C.c_int, C.c_int, C.c_int, P, P], C.c_int),
    "sevp_block_partition": ([C.c_int, C.c_int, C.c_int, P], C.c_int),
    "sevp_prep_assemble": ([C.c_int] * 4 + [P] * 8 + [C.c_int, C.c_float, C.c_int] + [P] * 6,
                           C.c_int),
    "sevp_prep_assemble_host": ([C.c_int] * 4 + [P] * 8 + [C.c_int, C.c_float, C.c_int] + [P] * 5,
                                C.c_int),
    "sevp_create": ([C.POINTER(P), C.c_int, C.c_int, C.c_int, P], C.c_int),
    "sevp_destroy": ([P], C.c_int),
    "sevp_set_operator": ([P, P, P, P, P, P, C.POINTER(Tiling)], C.c_int),
    "sevp_set_residual_operator": ([P, P, P, P, P, P, P], C.c_int),
    "sevp_set_chebyshev_bounds": ([P, C.c_double, C.c_double], C.c_int),
    "sevp_estimate_bounds": ([P, P, DP, DP, IP], C.c_int),
    "sevp_cheb_step": ([P, C.c_int, C.c_double, C.c_double, C.c_double] + [P] * 5, C.c_int),
    "sevp_influence_bytes": ([P], C.c_longlong),
    "sevp_set_influence_fp32": ([P, C.c_double], C.c_int),
    "sevp_influence_fp32_groups": ([P, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                    C.POINTER(C.c_longlong)], C.c_int),
    "sevp_solve": ([P, P, P, C.POINTER(SolveOpts), C.POINTER(Report)], C.c_int),
    "sevp_solve_host": ([P, P, P, C.POINTER(SolveOpts), C.POINTER(Report)], C.c_int),
    "sevp_apply": ([P, P, P], C.c_int),
    "sevp_precondition": ([P, P, P], C.c_int),
    "sevp_precondition_f32": ([P, P, P], C.c_int),
    "sevp_relative_residual": ([P, P, P, DP], C.c_int),
    "sevp_kernel_launches": ([P], C.c_longlong),
    "sevp_tile_layout": ([P, IP, IP, IP], C.c_int),
    "sevp_operator_symmetric": ([P], C.c_int),
    "sevp_set_full_coefficients": ([P, C.c_int], C.c_int),
    "sevp_set_graphs": ([P, C.c_int], C.c_int),
    "sevp_set_pass_a_kernel": ([P, C.c_int], C.c_int),
    "sevp_set_pass_b_kernel": ([P, C.c_int], C.c_int),
    "sevp_pass_b_kernel_used": ([P], C.c_int),
    "sevp_set_resume_check": ([P, C.c_double], C.c_int),
    "sevp_pass_a_f32": ([P, P, P, C.c_double, P, P, P], C.c_int),
    "sevp_pass_a_f64": ([P, P, P, C.c_double, P, P, P], C.c_int),
    "sevp_set_schwarz": ([P, C.c_int], C.c_int),
    "sevp_schwarz_shift": ([P], C.c_int),
    "sevp_record_coefficients": ([P, C.c_int], C.c_int),
    "sevp_step_history": ([P, P, P], C.c_int),
    "sevp_step_host": ([P, P, P, C.c_int, P, P], C.c_int),
    "sevp_step_prefetch": ([P, P], C.c_int),
    "sevp_step_submit": ([P, P, P, C.c_int, P, P], C.c_int),
    "sevp_step_wait": ([P], C.c_int),
    "sevp_read_coefficients": ([P, DP, DP, C.c_int, C.POINTER(C.c_int)], C.c_int),
    "sevp_schwarz_influence_bytes": ([P], C.c_longlong),
    "sevp_inprod_noalloc": ([P, P, C.c_int, C.c_int, P, P], C.c_int),
    "sevp_fs_mask": ([C.c_int, C.c_int, P, P, P, P, C.c_int, P], C.c_int),
    "sevp_fs_rhs": ([C.c_int, C.c_int, C.c_int] + [P] * 11, C.c_int),
    "sevp_fs_correct": ([C.c_int, C.c_int, C.c_int, P, C.c_float] + [P] * 10 + [C.c_int, P, P],
                        C.c_int),
    "sevp_fs_barotropic": ([P, C.c_int, C.c_int, C.c_int] + [P] * 15 + [C.c_float, C.c_int,
                                                                      C.c_float, C.c_int] + [P] * 7,
                           C.c_int),
    "sevp_evp_write": ([C.c_char_p, C.c_int, C.c_int] + [P] * 6 + [P, C.c_longlong, P, C.c_longlong,
                                                                P, C.c_int], C.c_int),
    "sevp_evp_write_sub": ([C.c_char_p, C.c_int, C.c_int] + [P] * 6 + [P, C.c_longlong, P,
                                                                    C.c_longlong, P, C.c_int,
                                                                    C.c_longlong], C.c_int),
    "sevp_evp_read": ([C.c_char_p, C.c_int, C.c_int] + [P] * 6 + [P, C.c_longlong, P, C.c_longlong,
                                                               P, C.c_int, P], C.c_int),
    "sevp_profile": ([P, C.c_int], C.c_int),
    "sevp_set_warmstart": ([P, P, P, C.c_int], C.c_int),
    "sevp_solve_step": ([P, P, P, P, P, C.c_int, C.POINTER(SolveOpts), C.POINTER(Report)], C.c_int),
    "sevp_solve_step_host": ([P, P, P, P, P, C.c_int, C.POINTER(SolveOpts), C.POINTER(Report)],
                             C.c_int),
    "sevp_profile_read": ([P, DP, C.POINTER(C.c_longlong)], C.c_int),
    # Fortran-compatible drop-ins (all pointers)
    "rep1_": ([P] * 17, None),
    "rep_": ([P] * 17, None),
    "repbir_": ([P] * 19, None),
    "repbir_period_": ([P] * 19, None),
    "pre1_": ([P] * 12, None),
    "pre_": ([P] * 13, None),
    "matinv_": ([P] * 2, None),
    "p_sqprod_": ([P] * 9, None),
    "p_sqprod_t_": ([P] * 9, None),
    "p_inprod_": ([P] * 5, None),
    "solver_boundary_update_": ([P] * 3, None),
    "p_bicgstab_le_": ([P] * 14, None),
    "p_sevp_pcg_": ([P] * 14, None),
    "p_csi_": ([P] * 16, None),
    "lanczos_": ([P] * 9, None),
    "sevp_bir_sweeps_": ([P] * 17, None),
    "sevp_pre_strips_": ([P] * 12, None),
}


def exported_symbols():
    return list(_SIGS)


def lib():
    """Loads the library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run musoc_solver_b200.build.build()")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            if not hasattr(L, name):
                continue
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def status_string(s: int) -> str:
    return lib().sevp_status_string(int(s)).decode()


def last_error() -> str:
    return lib().sevp_last_error().decode()


def check(status: int, what: str):
    if status != SEVP_OK:
        raise SevpError(status, what)


# ------------------------------------------------------------- helpers
def ptr(a) -> int:
    """Raw pointer of a numpy array or a torch tensor (device or host)."""
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a.data_ptr())


def iref(v: int):
    return C.byref(C.c_int(int(v)))


def dref(v: float):
    return C.byref(C.c_double(float(v)))
