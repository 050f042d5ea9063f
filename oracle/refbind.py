"""ctypes binding to the reference BiqBin C code built by ``oracle/Makefile``
into ``oracle/_ref/libbqb_ref.so`` (TEST INFRASTRUCTURE ONLY).

Exposes the reference's own entry points on inputs chosen by a test.  The
reference keeps its state in globals (src/global_var.h); ``RefLib.setup``
builds SP/PP/params/globals with the reference's own routines (see
``oracle/ref_shim.c``).  Struct layouts mirror src/biqbin.h:81-107 and
src/biqbin_cpp_api.h:27-63.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libbqb_ref.so")
REF_BAB = os.path.join(HERE, "_ref", "bqb_ref_bab")
NMAX = 1024


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


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_int))


def available() -> bool:
    return os.path.exists(REF_SO)


class RefLib:
    """One loaded copy of the reference library (its globals are process-wide)."""

    def __init__(self, path: str = REF_SO):
        os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
        self.lib = C.CDLL(path)
        L = self.lib
        L.ipm_mc_pk.argtypes = [C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double),
                                C.POINTER(C.c_double), C.c_int]
        L.op_B.argtypes = [C.POINTER(Problem), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.op_Bt.argtypes = [C.POINTER(Problem), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.fct_eval.argtypes = [C.POINTER(Problem), C.POINTER(C.c_double),
                               C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.fct_eval.restype = C.c_double
        L.getViolated_TriangleInequalities.argtypes = [C.POINTER(C.c_double), C.c_int,
                                                       C.POINTER(TriIneq), C.POINTER(C.c_int)]
        L.getViolated_TriangleInequalities.restype = C.c_double
        L.updateTriangleInequalities.argtypes = [C.POINTER(Problem), C.POINTER(C.c_double),
                                                 C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.updateTriangleInequalities.restype = C.c_double
        for nm in ("updatePentagonalInequalities", "updateHeptagonalInequalities"):
            f = getattr(L, nm)
            f.argtypes = [C.POINTER(Problem), C.POINTER(C.c_double), C.POINTER(C.c_int),
                          C.POINTER(C.c_int), C.c_int]
            f.restype = C.c_double
        L.runHeuristic_unpacked.argtypes = [C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double),
                                            C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                            C.POINTER(C.c_int)]
        L.runHeuristic_unpacked.restype = C.c_double
        L.GW_heuristic.argtypes = [C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double), C.c_int,
                                   C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int]
        L.GW_heuristic.restype = C.c_double
        L.mc_1opt.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_int]
        L.mc_1opt.restype = C.c_double
        L.solve_lambda.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                   C.POINTER(C.c_double)]
        L.lambda_eta.argtypes = [C.POINTER(Problem)] + [C.POINTER(C.c_double)] * 7
        L.bundle_method.argtypes = [C.POINTER(Problem), C.POINTER(C.c_double), C.c_int]
        L.SDPbound.argtypes = [C.POINTER(BabNode), C.POINTER(Problem), C.POINTER(Problem), C.c_int]
        L.SDPbound.restype = C.c_double
        L.Evaluate.argtypes = [C.POINTER(BabNode), C.POINTER(Problem), C.POINTER(Problem), C.c_int]
        L.Evaluate.restype = C.c_double
        L.createSubproblem.argtypes = [C.POINTER(BabNode), C.POINTER(Problem), C.POINTER(Problem)]
        L.evaluateSolution.argtypes = [C.POINTER(C.c_int)]
        L.evaluateSolution.restype = C.c_double
        L.Bab_LBGet.restype = C.c_double
        L.bqbref_setup.argtypes = [C.POINTER(C.c_double), C.c_int]
        L.bqbref_param_set.argtypes = [C.c_char_p, C.c_double]
        L.bqbref_param_get.argtypes = [C.c_char_p]
        L.bqbref_param_get.restype = C.c_double
        L.bqbref_set_lb.argtypes = [C.c_double]
        L.bqbref_set_diff.argtypes = [C.c_double]
        L.bqbref_get_diff.restype = C.c_double
        L.bqbref_sizeof_babnode.restype = C.c_size_t
        assert L.bqbref_sizeof_babnode() == C.sizeof(BabNode)
        self._setup_done = False

    # ---- globals -----------------------------------------------------
    def gptr(self, name: str, ctype):
        return C.POINTER(ctype).in_dll(self.lib, name)

    def problem(self, name: str) -> Problem:
        return C.POINTER(Problem).in_dll(self.lib, name).contents

    def setup(self, adj: np.ndarray, params: dict | None = None):
        """Default params, overrides, SP/PP from ``adj``, allocate globals."""
        if self._setup_done:
            raise RuntimeError("reference globals already allocated in this process")
        self.lib.bqbref_params_default()
        for k, v in (params or {}).items():
            if self.lib.bqbref_param_set(k.encode(), float(v)):
                raise KeyError(k)
        self._adj = np.ascontiguousarray(adj, dtype=np.float64)
        rc = self.lib.bqbref_setup(dptr(self._adj), self._adj.shape[0])
        if rc:
            raise RuntimeError("bqbref_setup failed")
        self._setup_done = True

    def param(self, name: str) -> float:
        return self.lib.bqbref_param_get(name.encode())

    def set_param(self, name: str, value) -> None:
        if self.lib.bqbref_param_set(name.encode(), float(value)):
            raise KeyError(name)

    def SP_L(self) -> np.ndarray:
        sp = self.problem("SP")
        n = sp.n
        return np.ctypeslib.as_array(sp.L, shape=(n * n,)).reshape(n, n).T.copy()

    # ---- bounding path entry points ---------------------------------
    def ipm(self, L: np.ndarray):
        n = L.shape[0]
        Lc = np.ascontiguousarray(L.T, dtype=np.float64)   # column-major
        X = np.zeros(n * n)
        phi = C.c_double()
        self.lib.ipm_mc_pk(dptr(Lc), n, dptr(X), C.byref(phi), 0)
        return X.reshape(n, n).T.copy(), phi.value

    def srand(self, seed: int):
        C.CDLL("libc.so.6").srand(seed)
