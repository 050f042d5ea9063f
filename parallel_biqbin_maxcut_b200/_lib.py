"""ctypes binding to libbqb_gpu.so (the product library).

The library is built in-tree by ``parallel_biqbin_maxcut_b200.build``.  There
is no CPU fallback: if the library is missing or no CUDA device is usable,
``load()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libbqb_gpu.so")
NMAX = 1024

_lib = None


class Problem(C.Structure):
    _fields_ = [("L", C.POINTER(C.c_double)), ("n", C.c_int), ("NIneq", C.c_int),
                ("NPentIneq", C.c_int), ("NHeptaIneq", C.c_int), ("bundle", C.c_int)]


class TriIneq(C.Structure):
    _fields_ = [("i", C.c_int), ("j", C.c_int), ("k", C.c_int), ("type", C.c_int),
                ("value", C.c_double), ("y", C.c_double)]


class PentIneq(C.Structure):
    _fields_ = [("type", C.c_int), ("permutation", C.c_int * 5),
                ("value", C.c_double), ("y", C.c_double)]


class HeptIneq(C.Structure):
    _fields_ = [("type", C.c_int), ("permutation", C.c_int * 7),
                ("value", C.c_double), ("y", C.c_double)]


class BabNode(C.Structure):
    _fields_ = [("xfixed", C.c_int * NMAX), ("sol", C.c_int * NMAX),
                ("fracsol", C.c_double * NMAX), ("level", C.c_int),
                ("upper_bound", C.c_double)]


class Params(C.Structure):
    """BiqBinParameters, src/biqbin.h:49-84 (same order and types)."""
    _fields_ = [("init_bundle_iter", C.c_int), ("max_bundle_iter", C.c_int),
                ("triag_iter", C.c_int), ("pent_iter", C.c_int), ("hept_iter", C.c_int),
                ("max_outer_iter", C.c_int), ("extra_iter", C.c_int),
                ("violated_TriIneq", C.c_double), ("TriIneq", C.c_int),
                ("adjust_TriIneq", C.c_int), ("PentIneq", C.c_int), ("HeptaIneq", C.c_int),
                ("Pent_Trials", C.c_int), ("Hepta_Trials", C.c_int),
                ("include_Pent", C.c_int), ("include_Hepta", C.c_int), ("root", C.c_int),
                ("use_diff", C.c_int), ("time_limit", C.c_int), ("branchingStrategy", C.c_int)]


# Reference defaults (src/biqbin.h:49-78) and the shipped `params` file
# values the reference tests use (init_bundle_iter 5, violated_TriIneq 0.05).
PARAM_DEFAULTS = dict(init_bundle_iter=3, max_bundle_iter=15, triag_iter=5, pent_iter=5,
                      hept_iter=5, max_outer_iter=20, extra_iter=10, violated_TriIneq=1e-3,
                      TriIneq=5000, adjust_TriIneq=1, PentIneq=5000, HeptaIneq=5000,
                      Pent_Trials=60, Hepta_Trials=50, include_Pent=1, include_Hepta=1, root=0,
                      use_diff=1, time_limit=0, branchingStrategy=1)
PARAMS_FILE = dict(PARAM_DEFAULTS, init_bundle_iter=5, violated_TriIneq=0.05)

D = C.POINTER(C.c_double)
I = C.POINTER(C.c_int)

# name -> (restype, argtypes)
SIGNATURES = {
    "ipm_mc_pk": (None, [D, C.c_int, D, D, C.c_int]),
    "op_B": (None, [C.POINTER(Problem), D, D]),
    "op_Bt": (None, [C.POINTER(Problem), D, D]),
    "diag": (None, [D, D, C.c_int]),
    "Diag": (None, [D, D, C.c_int]),
    "fct_eval": (C.c_double, [C.POINTER(Problem), D, D, D]),
    "solve_lambda": (None, [C.c_int, D, D, D]),
    "lambda_eta": (None, [C.POINTER(Problem), D, D, D, D, D, D, D]),
    "bundle_method": (None, [C.POINTER(Problem), D, C.c_int]),
    "evaluateTriangleInequality": (C.c_double, [D, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    "getViolated_TriangleInequalities": (C.c_double, [D, C.c_int, C.POINTER(TriIneq), I]),
    "updateTriangleInequalities": (C.c_double, [C.POINTER(Problem), D, I, I]),
    "getViolated_PentagonalInequalities": (C.c_double, [D, C.c_int, C.POINTER(PentIneq), I]),
    "updatePentagonalInequalities": (C.c_double, [C.POINTER(Problem), D, I, I, C.c_int]),
    "getViolated_HeptagonalInequalities": (C.c_double, [D, C.c_int, C.POINTER(HeptIneq), I]),
    "updateHeptagonalInequalities": (C.c_double, [C.POINTER(Problem), D, I, I, C.c_int]),
    "qap_simulated_annealing": (C.c_double, [I, C.c_int, D, C.c_int, I]),
    "runHeuristic": (C.c_double, [C.POINTER(Problem), C.POINTER(Problem), C.POINTER(BabNode), I]),
    "runHeuristic_unpacked": (C.c_double, [D, C.c_int, D, C.c_int, I, I, I]),
    "GW_heuristic": (C.c_double, [D, C.c_int, D, C.c_int, I, I, I, C.c_int]),
    "mc_1opt": (C.c_double, [I, D, C.c_int]),
    "update_best": (C.c_int, [I, I, D, C.c_int]),
    "bqb_init": (C.c_int, [C.c_int]),
    "bqb_last_error": (C.c_char_p, []),
    "bqb_kernel_launches": (C.c_ulonglong, []),
    "bqb_synchronize": (None, []),
    "bqb_ipm_plan_create": (C.c_void_p, [C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), I, C.c_int,
                                         C.c_void_p]),
    "bqb_ipm_plan_launch": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bqb_ipm_plan_destroy": (None, [C.c_void_p]),
    "bqb_ipm_batch_device": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), I, C.c_int,
                                       C.c_void_p, C.c_void_p]),
    "bqb_ipm_batch": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), I, C.c_int, D, I, I]),
}


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load the library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} not built: run `python -m parallel_biqbin_maxcut_b200.build`")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols(path: str = LIB_PATH) -> set[str]:
    lib = C.CDLL(path)
    return {n for n in SIGNATURES if hasattr(lib, n)}


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(D)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(I)


def colmajor(A: np.ndarray) -> np.ndarray:
    """Column-major flat copy (reference layout) of a square matrix."""
    return np.ascontiguousarray(np.asarray(A, dtype=np.float64).T).reshape(-1)


def from_colmajor(flat: np.ndarray, n: int) -> np.ndarray:
    return np.asarray(flat[: n * n]).reshape(n, n).T.copy()


def global_ptr(name: str, ctype):
    """The library's own copy of a reference global (standalone use)."""
    return ctype.in_dll(load(), name)
