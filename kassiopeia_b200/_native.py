"""ctypes binding of libkemcu.so (the C ABI in include/kemcu.h).

The shared library is built in-tree by ``kassiopeia_b200.build.build()``. Loading fails
loudly when it is missing: there is no CPU fallback anywhere in this package.
"""

from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libkemcu.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "kemcu.h")

OK, EINVAL, ECUDA, ENONFINITE, ENOTCONVERGED, ETIMEOUT, ENOMEM, ESTATE = 0, -1, -2, -3, -4, -5, -6, -7
FP64, MIXED, FP32 = 0, 1, 2
FIELD_AND_POTENTIAL, POTENTIAL, FIELD = 0, 1, 2
SOLVE_PLAIN, SOLVE_MIXED, SOLVE_ASSEMBLED, SOLVE_ASSEMBLED_FP64, SOLVE_FP32, SOLVE_FFTM = 0, 1, 2, 3, 4, 5
TRACK_ACTIVE, TRACK_HIT, TRACK_MAX_STEPS, TRACK_LEFT, TRACK_NONFINITE = 0, 1, 2, 3, 4
KRYLOV_GMRES, KRYLOV_BICGSTAB = 0, 1
PRECON_NONE, PRECON_JACOBI, PRECON_IMPLICIT_KRYLOV = 0, 1, 2

_ERRNAMES = {EINVAL: "EINVAL", ECUDA: "ECUDA", ENONFINITE: "ENONFINITE", ENOTCONVERGED: "ENOTCONVERGED",
             ETIMEOUT: "ETIMEOUT", ENOMEM: "ENOMEM", ESTATE: "ESTATE"}


class KemcuError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"kemcu error {code} ({_ERRNAMES.get(code, '?')}): {message}")
        self.code = code


class Config(C.Structure):
    _fields_ = [("device", C.c_int), ("one_over_four_pi_eps0", C.c_double), ("eps0", C.c_double),
                ("assembled_budget_bytes", C.c_size_t), ("autotune", C.c_int)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("outer", C.c_int), ("fp64_matvecs", C.c_int), ("low_matvecs", C.c_int),
                ("rel_residual", C.c_double), ("rel_residual_estimate", C.c_double), ("seconds", C.c_double)]


class RhStats(C.Structure):
    _fields_ = [("subiterations", C.c_longlong), ("iterations", C.c_int), ("rel_residual", C.c_double),
                ("seconds", C.c_double)]


class HitModel(C.Structure):
    _fields_ = [("sphere_radius", C.c_double), ("max_radius", C.c_double)]


class TrackStats(C.Structure):
    _fields_ = [("steps", C.c_longlong), ("field_evals", C.c_longlong), ("hit", C.c_int), ("max_steps", C.c_int),
                ("left", C.c_int), ("nonfinite", C.c_int), ("active", C.c_int), ("seconds", C.c_double)]


class FftmParams(C.Structure):
    _fields_ = [("degree", C.c_int), ("top_level_divisions", C.c_int), ("divisions", C.c_int),
                ("zeromask", C.c_int), ("maximum_tree_depth", C.c_int), ("insertion_ratio", C.c_double),
                ("region_expansion_factor", C.c_double), ("world_center", C.c_double * 3),
                ("world_length", C.c_double), ("near_analytic", C.c_int)]



class KrylovParams(C.Structure):
    _fields_ = [("solver", C.c_int), ("mode", C.c_int), ("tolerance", C.c_double), ("max_iterations", C.c_int),
                ("iterations_between_restarts", C.c_int), ("preconditioner", C.c_int),
                ("preconditioner_mode", C.c_int), ("preconditioner_tolerance", C.c_double),
                ("max_preconditioner_iterations", C.c_int)]


ITER_CB = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_double)

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lib = None


def header_symbols() -> list[str]:
    """Every function the C header declares (the ABI surface the library must export)."""
    txt = open(HEADER).read()
    decl = r"^\s*(?:int|void|double|size_t|unsigned\s+long\s+long|const\s+char\s*\*)\s*(kemcu_[a-z0-9_]+)\s*\("
    return sorted(set(re.findall(decl, txt, flags=re.M)))


def header_constant(name: str) -> int:
    """Value of an integer #define of the C header (literals, u suffixes, <<, *, /, +, - and
    other such defines), so that tests follow the header instead of restating its numbers."""
    txt = open(HEADER).read()
    defs = dict(re.findall(r"^\s*#define\s+(KEMCU_[A-Z0-9_]+)\s+(.+?)\s*(?:/\*.*)?$", txt, flags=re.M))

    def value(n, depth=0):
        if n not in defs or depth > 8:
            raise KeyError(f"{n} is not an integer #define of {HEADER}")
        expr = re.sub(r"\b(\d+)[uUlL]+\b", r"\1", defs[n])
        expr = re.sub(r"\bKEMCU_[A-Z0-9_]+\b", lambda m: str(value(m.group(0), depth + 1)), expr)
        if not re.fullmatch(r"[0-9\s()+\-*/<>]+", expr):
            raise ValueError(f"{n}: cannot evaluate {defs[n]!r}")
        return int(eval(expr.replace("/", "//"), {"__builtins__": {}}))

    return value(name)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with kassiopeia_b200.build.build() "
                          "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.kemcu_default_config.argtypes = [C.POINTER(Config)]
    L.kemcu_default_config.restype = None
    L.kemcu_create.argtypes = [C.POINTER(vp), C.POINTER(Config)]
    L.kemcu_destroy.argtypes = [vp]
    L.kemcu_last_error.argtypes = [vp]
    L.kemcu_last_error.restype = C.c_char_p
    L.kemcu_last_kernel_ms.argtypes = [vp]
    L.kemcu_last_kernel_ms.restype = C.c_double
    L.kemcu_set_geometry.argtypes = [vp, C.c_size_t, _ip, _ip, _dp, _dp]
    L.kemcu_num_elements.argtypes = [vp]
    L.kemcu_num_elements.restype = C.c_size_t
    L.kemcu_set_sigma.argtypes = [vp, _dp]
    L.kemcu_get_sigma.argtypes = [vp, _dp]
    L.kemcu_rhs.argtypes = [vp, _dp]
    L.kemcu_field.argtypes = [vp, _dp, C.c_size_t, _dp, C.c_int, C.c_int]
    L.kemcu_field_dev.argtypes = [vp, C.c_void_p, C.c_size_t, C.c_void_p, C.c_int, C.c_int]
    L.kemcu_field_dev_noalloc.argtypes = [vp, C.c_void_p, C.c_size_t, C.c_void_p, C.c_int, C.c_int]
    L.kemcu_matrix_element.argtypes = [vp, C.c_size_t, C.c_size_t, _dp]
    L.kemcu_matvec.argtypes = [vp, _dp, _dp, C.c_int, C.c_int, C.c_int]
    L.kemcu_gmres.argtypes = [vp, _dp, _dp, C.c_int, C.c_double, C.c_int, C.c_int, C.POINTER(SolveStats)]
    L.kemcu_set_iteration_callback.argtypes = [vp, ITER_CB, C.c_void_p]
    L.kemcu_robin_hood.argtypes = [vp, _dp, _dp, C.c_double, C.c_int, C.c_longlong, C.c_int, C.POINTER(RhStats)]
    L.kemcu_set_iteration_callback.restype = None
    L.kemcu_track_rk8.argtypes = [vp, _dp, _ip, _ip, C.c_size_t, C.c_double, C.c_int, C.c_int, C.c_double,
                                  C.c_double, C.POINTER(HitModel), C.c_int, C.POINTER(TrackStats), _dp]
    L.kemcu_field_vjp.argtypes = [vp, _dp, C.c_size_t, _dp, _dp, _dp, C.c_int]
    L.kemcu_rule_nodes.argtypes = [C.c_int, _dp]
    L.kemcu_launch_count.argtypes = [vp]
    L.kemcu_launch_count.restype = C.c_ulonglong
    L.kemcu_band_histogram.argtypes = [vp, _dp, C.c_size_t, C.POINTER(C.c_longlong)]
    L.kemcu_fma_peak.argtypes = [vp, _dp, _dp]
    L.kemcu_selftest_timeout.argtypes = [vp, C.c_int]
    L.kemcu_tune_field.argtypes = [vp, C.c_void_p, C.c_size_t, C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                   C.POINTER(C.c_float)]
    L.kemcu_field_variant.argtypes = [vp, C.c_size_t, C.c_int, C.POINTER(C.c_int)]
    L.kemcu_field_variant_info.argtypes = [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.kemcu_field_variant_count.argtypes = []
    L.kemcu_fftm_default_params.argtypes = [C.POINTER(FftmParams)]
    L.kemcu_fftm_default_params.restype = None
    L.kemcu_fftm_configure.argtypes = [vp, C.POINTER(FftmParams)]
    L.kemcu_fftm_configure_preconditioner.argtypes = [vp, C.POINTER(FftmParams)]
    L.kemcu_krylov_default_params.argtypes = [C.POINTER(KrylovParams)]
    L.kemcu_krylov_default_params.restype = None
    L.kemcu_krylov_solve.argtypes = [vp, _dp, _dp, C.c_int, C.POINTER(KrylovParams), C.POINTER(SolveStats)]
    L.kemcu_fftm_field.argtypes = [vp, _dp, C.c_size_t, _dp, C.c_int]
    L.kemcu_fftm_field_dev.argtypes = [vp, C.c_void_p, C.c_size_t, C.c_void_p, C.c_int]
    L.kemcu_fftm_info.argtypes = [vp, _dp, _ip]
    L.kemcu_fftm_matvec.argtypes = [vp, _dp, _dp, C.c_int]
    L.kemcu_fm_moments.argtypes = [vp, C.c_int, _dp, _dp]
    L.kemcu_fm_local_field.argtypes = [vp, C.c_int, _dp, _dp, C.c_size_t, _dp, _dp]
    L.kemcu_fm_response.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp]
    _lib = L
    return L
