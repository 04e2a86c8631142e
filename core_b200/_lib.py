"""ctypes binding of libunwrap_b200.so (the C ABI declared in include/unwrap_b200.h).

Loading the library needs no GPU; every compute entry point needs one.  There
is no CPU fallback: if the library is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libunwrap_b200.so")

UNW_OK = 0
UNW_W_NUMERIC = 1
UNW_E_ARG = -1
UNW_E_WORKSPACE = -2
UNW_E_CUDA = -3
UNW_E_UNSUPPORTED = -4
UNW_E_OVERFLOW = -5

UNW_F_CONGRUENT = 1
UNW_F_NO_GRAPH = 2
UNW_F_PROFILE = 4
UNW_F_FIXED_ITERS = 8
UNW_F_MIXED = 16
UNW_F_COL_TC = 32
UNW_F_COL_FFT = 64
UNW_F_COL_NO_TMA = 128
UNW_F_COL_TMA = 256
UNW_F_MV_NO_TMA = 512

PROF_NAMES = ["bbox", "setup", "row_rho", "col", "row_inv", "matvec", "row_upd", "row_r0", "head", "elem", "post"]
PROF_N = len(PROF_NAMES)

UNW_S_DCT_INIT_NONFINITE = 1
UNW_S_REVERTED = 2
UNW_S_NONFINITE_OUT = 4
UNW_S_ALL_NAN = 8
UNW_S_TC_TIMEOUT = 16


class UnwParams(C.Structure):
    _fields_ = [("max_iter", C.c_int32), ("tol", C.c_float), ("cg_max_iter", C.c_int32),
                ("cg_tol", C.c_float), ("epsilon", C.c_float), ("conncomp_size", C.c_int32),
                ("flags", C.c_int32), ("check_every", C.c_int32)]


class UnwStats(C.Structure):
    _fields_ = [("irls_iters", C.c_int32), ("cg_iters_total", C.c_int32), ("cg_iters_last", C.c_int32),
                ("n_components", C.c_int32), ("n_labels", C.c_int32), ("status", C.c_int32),
                ("bbox", C.c_int32 * 4), ("rel_change", C.c_double), ("best_residual", C.c_double),
                ("k_median", C.c_double), ("cg_iters", C.c_int32 * 64),
                ("prof_ms", C.c_float * 16), ("prof_launches", C.c_int32 * 16),
                ("col_path", C.c_int32), ("tune_ms", C.c_float * 2), ("col_tma", C.c_int32),
                ("resid_rel", C.c_double)]

    def as_dict(self):
        n = min(self.irls_iters, 64)
        return dict(irls_iters=self.irls_iters, cg_iters_total=self.cg_iters_total,
                    cg_iters_last=self.cg_iters_last, n_components=self.n_components,
                    n_labels=self.n_labels, status=self.status, bbox=tuple(self.bbox),
                    rel_change=self.rel_change, best_residual=self.best_residual,
                    k_median=self.k_median, cg_iters=list(self.cg_iters[:n]),
                    prof_ms=list(self.prof_ms[:PROF_N]), prof_launches=list(self.prof_launches[:PROF_N]),
                    col_path=self.col_path, tune_ms=list(self.tune_ms), col_tma=self.col_tma,
                    resid_rel=self.resid_rel)


UNW_LINK_C_LINE = 1


class UnwLinkParams(C.Structure):
    _fields_ = [("min_size", C.c_int32), ("max_neighbors", C.c_int32), ("window", C.c_int32), ("flags", C.c_int32)]


class UnwLinkPair(C.Structure):
    _fields_ = [("comp_i", C.c_int32), ("comp_j", C.c_int32), ("yi", C.c_int32), ("xi", C.c_int32),
                ("yj", C.c_int32), ("xj", C.c_int32), ("d2", C.c_int64), ("blocked", C.c_int32),
                ("n_i", C.c_int32), ("n_j", C.c_int32), ("nf_i", C.c_int32), ("nf_j", C.c_int32),
                ("mean_i", C.c_float), ("mean_j", C.c_float), ("pad", C.c_int32)]


class UnwGrid(C.Structure):
    _fields_ = [("phase", C.c_void_p), ("phase_pitch", C.c_int64), ("weight", C.c_void_p),
                ("weight_pitch", C.c_int64), ("H", C.c_int64), ("W", C.c_int64),
                ("out_u", C.c_void_p), ("out_u_pitch", C.c_int64), ("out_cc", C.c_void_p),
                ("out_cc_pitch", C.c_int64)]


class UnwAdjGrid(C.Structure):
    _fields_ = [("phase", C.c_void_p), ("phase_pitch", C.c_int64), ("weight", C.c_void_p),
                ("weight_pitch", C.c_int64), ("H", C.c_int64), ("W", C.c_int64),
                ("u", C.c_void_p), ("u_pitch", C.c_int64), ("grad_u", C.c_void_p), ("grad_u_pitch", C.c_int64),
                ("grad_phase", C.c_void_p), ("grad_phase_pitch", C.c_int64),
                ("grad_weight", C.c_void_p), ("grad_weight_pitch", C.c_int64)]


# every symbol include/unwrap_b200.h declares, with its ctypes signature
SIGNATURES = {
    "unw_abi_version": (C.c_int, []),
    "unw_last_error": (C.c_char_p, []),
    "unw_workspace_bytes": (C.c_size_t, [C.c_int64, C.c_int64]),
    "unw_batch_workspace_bytes": (C.c_size_t, [C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "unw_solve_f32": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int64, C.c_int64,
                                C.POINTER(UnwParams), C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                C.c_void_p, C.c_size_t, C.POINTER(UnwStats), C.c_void_p]),
    "unw_solve_batch": (C.c_int, [C.c_int32, C.POINTER(UnwGrid), C.POINTER(UnwParams), C.c_void_p,
                                  C.c_size_t, C.POINTER(UnwStats), C.c_void_p]),
    "unw_setup_gradients": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]),
    "unw_apply_laplacian": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p,
                                      C.c_void_p, C.c_size_t, C.c_void_p]),
    "unw_apply_preconditioner": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p,
                                           C.c_size_t, C.c_void_p]),
    "unw_apply_preconditioner_mixed": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_int32,
                                                 C.c_void_p, C.c_size_t, C.c_void_p]),
    "unw_apply_preconditioner_noalloc": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p]),
    "unw_adjoint_workspace_bytes": (C.c_size_t, [C.c_int64, C.c_int64]),
    "unw_adjoint_batch_workspace_bytes": (C.c_size_t, [C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "unw_adjoint_batch": (C.c_int, [C.c_int32, C.POINTER(UnwAdjGrid), C.POINTER(UnwParams), C.c_void_p,
                                    C.c_size_t, C.POINTER(UnwStats), C.c_void_p]),
    "unw_goldstein_workspace_bytes": (C.c_size_t, [C.c_int64, C.c_int64, C.c_int32, C.c_int32]),
    "unw_goldstein_c64": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int64, C.c_int64,
                                    C.c_int32, C.c_int32, C.c_float, C.c_void_p, C.c_int64, C.c_void_p,
                                    C.c_size_t, C.c_void_p]),
    "unw_link_workspace_bytes": (C.c_size_t, [C.c_int64, C.c_int64, C.c_int32]),
    "unw_link_pairs_f32": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int64, C.c_int64,
                                     C.POINTER(UnwLinkParams), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                     C.POINTER(C.c_int32), C.c_void_p, C.c_int32, C.POINTER(C.c_int32),
                                     C.c_void_p, C.c_size_t, C.c_void_p]),
    "unw_link_apply_f32": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_void_p, C.c_int32,
                                     C.c_void_p, C.c_int64, C.c_void_p, C.c_size_t, C.c_int32, C.c_void_p]),
    "unw_link_offsets": (C.c_int, [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_int32, C.c_void_p]),
    "unw_adjoint_f32": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int64, C.c_int64,
                                  C.POINTER(UnwParams), C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                  C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_size_t,
                                  C.POINTER(UnwStats), C.c_void_p]),
}

_lock = threading.Lock()
_lib = None


def load():
    """Load the shared library once; raise if it has not been built."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(f"{LIB_PATH} is missing: build it with `python -m core_b200._build`")
            lib = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
        return _lib


def last_error():
    return load().unw_last_error().decode(errors="replace")


def check(rc, what="unw call"):
    """Map negative return codes to Python exceptions (positive codes are warnings)."""
    if rc >= 0:
        return rc
    msg = f"{what}: {last_error()}"
    if rc == UNW_E_ARG:
        raise ValueError(msg)
    if rc == UNW_E_OVERFLOW:
        raise OverflowError(msg)
    if rc == UNW_E_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise RuntimeError(msg)
