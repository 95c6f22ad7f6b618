"""ctypes binding of ``libblocksp_b200.so`` (the C ABI in include/blocksp_b200.h).

The library is loaded from this package directory only: an in-tree build made
by ``blocksp_b200.build``.  There is no fallback implementation; if the
library is missing or no GPU is present, calls fail loudly.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libblocksp_b200.so"

BSP_OK = 0
STATUS_NAMES = {
    0: "OK", 1: "ZERO_PIVOT", 2: "NOT_SPD", 3: "BREAKDOWN", 4: "MAXIT", 5: "NAN",
    6: "TIMEOUT", 7: "CUDA_ERROR", 8: "INVALID", 9: "NO_DEVICE", 10: "OUT_OF_MEMORY",
}
BSP_F64, BSP_F32, BSP_BF16 = 0, 1, 2
PC_NONE, PC_DIAG_LU, PC_DIAG_CHOL, PC_SOR_LU, PC_SOR_CHOL, PC_ILU0, PC_ICHOL0 = range(7)
PC_LEARNED_LLT, PC_LEARNED_LU = 7, 8
PREC_F64, PREC_F32, PREC_BF16 = 0, 1, 2
STOP_REFERENCE, STOP_TRUE_RESIDUAL = 0, 1
LEARNED_LU, LEARNED_LLT = 0, 1


class BspError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{where}: {name}" + (f" ({detail})" if detail else ""))


class PrecondParams(C.Structure):
    _fields_ = [("kind", C.c_int), ("sor_w", C.c_double), ("sor_nu", C.c_int),
                ("sor_type", C.c_int), ("precision", C.c_int)]


class SolveOpts(C.Structure):
    _fields_ = [("tol", C.c_double), ("max_iters", C.c_int), ("restart", C.c_int), ("k", C.c_int),
                ("print_iters", C.c_int), ("stop_rule", C.c_int), ("precision", C.c_int),
                ("inner_tol", C.c_double), ("max_outer", C.c_int), ("print_eig_info", C.c_int)]


class SolveInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("iters", C.c_int), ("n_hist", C.c_int),
                ("n_restarts", C.c_int), ("n_outer", C.c_int), ("inner_iters", C.c_int),
                ("res0", C.c_double), ("final_res", C.c_double), ("true_rel_res", C.c_double),
                ("setup_ms", C.c_double), ("solve_ms", C.c_double)]


class BatchOpts(C.Structure):
    _fields_ = [("tol", C.c_double), ("max_iters", C.c_int), ("mode", C.c_int),
                ("check_every", C.c_int), ("hist_cap", C.c_int), ("retune", C.c_int)]


class BatchInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("n_pairs", C.c_int), ("n_converged", C.c_int),
                ("iters_max", C.c_int), ("iters_total", C.c_longlong), ("graph_iters", C.c_int),
                ("setup_ms", C.c_double), ("solve_ms", C.c_double)]


_P = C.c_void_p
_I = C.c_int
_I64 = C.c_int64
_D = C.c_double
_PD = C.POINTER(C.c_double)

# name -> (restype, argtypes); every symbol declared in include/blocksp_b200.h
SIGNATURES: dict[str, tuple] = {
    "bsp_abi_version": (_I, []),
    "bsp_launch_count": (C.c_uint64, []),
    "bsp_status_string": (C.c_char_p, [_I]),
    "bsp_last_error": (C.c_char_p, [_P]),
    "bsp_device_count": (_I, [C.POINTER(_I)]),
    "bsp_handle_create": (_I, [_I, _P, C.POINTER(_P)]),
    "bsp_handle_destroy": (_I, [_P]),
    "bsp_handle_sync": (_I, [_P]),
    "bsp_handle_stream": (_P, [_P]),
    "bsp_handle_set_spin_limit": (_I, [_P, C.c_uint]),
    "bsp_release_cached_memory": (_I, [_I]),
    "bsp_cached_memory": (_I, [_I, C.POINTER(_I64)]),
    "bsp_matrix_create": (_I, [_P, _I, _I, _I, _I64, _P, _P, _P, C.POINTER(_P)]),
    "bsp_matrix_create_complex": (_I, [_P, _I, _I, _I, _I64, _P, _P, _P, C.POINTER(_P)]),
    "bsp_matrix_complex_bs": (_I, [_P, C.POINTER(_I)]),
    "bsp_matrix_create_dev": (_I, [_P, _I, _I, _I, _I64, _P, _P, _P, C.POINTER(_P)]),
    "bsp_matrix_destroy": (_I, [_P]),
    "bsp_matrix_info": (_I, [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I), C.POINTER(_I64)]),
    "bsp_matrix_device_ptrs": (_I, [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]),
    "bsp_matrix_make_lowp": (_I, [_P, _I]),
    "bsp_bsmv_dev": (_I, [_P, _P, _I, _I, _I, _D, _P, _D, _P, _P]),
    "bsp_bsmv": (_I, [_P, _P, _I, _I, _D, _P, _D, _P]),
    "bsp_dot_dev": (_I, [_P, _I64, _P, _P, _P]),
    "bsp_dot": (_I, [_P, _I64, _P, _P, _PD]),
    "bsp_axpy_dev": (_I, [_P, _I64, _D, _P, _P]),
    "bsp_dot_noalloc": (_I, [_P, _I64, _P, _P, _P]),
    "bsp_precond_create": (_I, [_P, _P, C.POINTER(PrecondParams), C.POINTER(_P)]),
    "bsp_precond_destroy": (_I, [_P]),
    "bsp_precond_apply_dev": (_I, [_P, _P, _P]),
    "bsp_precond_apply": (_I, [_P, _P, _P]),
    "bsp_precond_export": (_I, [_P, _P, _I64]),
    "bsp_precond_info": (_I, [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I), C.POINTER(_I64)]),
    "bsp_pcg_dev": (_I, [_P, _P, _P, _P, _P, C.POINTER(SolveOpts), _P, _I, C.POINTER(SolveInfo)]),
    "bsp_pgmres_dev": (_I, [_P, _P, _P, _P, _P, C.POINTER(SolveOpts), _P, _I, C.POINTER(SolveInfo)]),
    "bsp_pcg": (_I, [_P, _P, _P, _P, _P, C.POINTER(SolveOpts), _P, _I, C.POINTER(SolveInfo)]),
    "bsp_pgmres": (_I, [_P, _P, _P, _P, _P, C.POINTER(SolveOpts), _P, _I, C.POINTER(SolveInfo)]),
    "bsp_true_residual_dev": (_I, [_P, _P, _P, _P, _PD]),
    "bsp_batch_create": (_I, [_P, _I, _P, _P, _P, _P, _P, _P, C.POINTER(_P)]),
    "bsp_batch_destroy": (_I, [_P]),
    "bsp_batch_tuning": (_I, [_P, _P, _P, _P, _P, _P, _P, _P]),
    "bsp_batch_pcg_dev": (_I, [_P, _P, _I, _P, _P, C.POINTER(BatchOpts), C.POINTER(BatchInfo)]),
    "bsp_batch_pcg": (_I, [_P, _P, _I, _P, _P, C.POINTER(BatchOpts), C.POINTER(BatchInfo)]),
    "bsp_batch_results": (_I, [_P, _I, _P, _P, _P, _P, _I]),
    "bsp_learned_create": (_I, [_P, _I, _I, C.POINTER(_P)]),
    "bsp_learned_destroy": (_I, [_P]),
    "bsp_learned_set_form": (_I, [_P, _I]),
    "bsp_learned_set_relax": (_I, [_P, C.c_double]),
    "bsp_learned_get_relax": (_I, [_P, C.POINTER(C.c_double)]),
    "bsp_learned_param_count": (_I, [_P, C.POINTER(_I64)]),
    "bsp_learned_set_params": (_I, [_P, _P, _I64]),
    "bsp_learned_get_params": (_I, [_P, _P, _I64]),
    "bsp_learned_get_grads": (_I, [_P, _P, _I64]),
    "bsp_learned_forward": (_I, [_P, _P, _P, _P]),
    "bsp_learned_ilu_factors": (_I, [_P, _P, _P]),
    "bsp_learned_loss_grad": (_I, [_P, _P, _P, _P, _I, _P, _PD]),
    "bsp_learned_adam_step": (_I, [_P, _P, _D, _D, _D, _D]),
    "bsp_learned_probes": (_I, [_P, _P, _P, _P, _I, _P]),
    "bsp_learned_precond": (_I, [_P, _P, _P, _I, C.POINTER(_P)]),
    "bsp_learned_smooth": (_I, [_P, _P, _P, _I, _I, _P]),
    "bsp_arnoldi_eigenvalues": (_I, [_P, _P, _P, _I, _I, _I, _I, _P, _P, C.POINTER(_I)]),
    "bsp_bs_id": (_I, [_P, _I, _I, C.POINTER(_P)]),
    "bsp_bs_tr": (_I, [_P, _P, C.POINTER(_P)]),
    "bsp_bsmm": (_I, [_P, _P, _P, _I, C.POINTER(_P)]),
    "bsp_matrix_add": (_I, [_P, _D, _P, _D, _P, C.POINTER(_P)]),
    "bsp_matrix_export": (_I, [_P, _P, _P, _P]),
    "bsp_mtx_read_matrix": (_I, [C.c_char_p, _I, _I, _I, _I, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I64),
                                 _P, _P, _P]),
    "bsp_mtx_read_vector": (_I, [C.c_char_p, _I, _I, _I, C.POINTER(_I64), _P]),
}

_lib = None


def load() -> C.CDLL:
    """Load the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH.name} is not built; run `python -m blocksp_b200.build` "
                "(the solve path has no CPU fallback)")
        lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def exported_symbols() -> list[str]:
    lib = load()
    return [n for n in SIGNATURES if getattr(lib, n, None) is not None]


def check(status: int, where: str, handle=None) -> None:
    if status != BSP_OK:
        lib = load()
        msg = lib.bsp_last_error(handle)
        raise BspError(status, where, msg.decode() if msg else "")
