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
    "SDPbound": (C.c_double, [C.POINTER(BabNode), C.POINTER(Problem), C.POINTER(Problem), C.c_int]),
    "Evaluate": (C.c_double, [C.POINTER(BabNode), C.POINTER(Problem), C.POINTER(Problem), C.c_int]),
    "createSubproblem": (None, [C.POINTER(BabNode), C.POINTER(Problem), C.POINTER(Problem)]),
    "getFixedValue": (C.c_double, [C.POINTER(BabNode), C.POINTER(Problem)]),
    "evaluateSolution": (C.c_double, [I]),
    "updateSolution": (C.c_int, [I]),
    "getBranchingVariable": (C.c_int, [C.POINTER(BabNode)]),
    "countFixedVariables": (C.c_int, [C.POINTER(BabNode)]),
    "Bab_LBGet": (C.c_double, []),
    "Bab_LBUpd": (C.c_int, [C.c_double, C.c_void_p]),
    "Bab_numEvalNodes": (C.c_int, []),
    "readData": (C.POINTER(C.c_double), [C.c_char_p, I]),
    "process_adj_matrix": (C.c_int, [D, C.c_int]),
    "bqb_default_params": (None, [C.POINTER(Params)]),
    "bqb_read_params": (C.c_int, [C.c_char_p, C.POINTER(Params)]),
    "bqb_solve": (C.c_int, [D, C.c_int, C.c_void_p, C.c_void_p]),
    "bqb_solve_parallel": (C.c_int, [D, C.c_int, C.c_void_p, C.c_int, C.c_void_p]),
    "bqb_solve_fused": (C.c_int, [D, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "bqb_solve_device": (C.c_int, [D, C.c_int, C.c_void_p, C.c_int, C.c_void_p]),
    "bqb_bound_nodes": (C.c_int, [C.POINTER(BabNode), C.c_int, C.c_int, C.c_int,
                                  C.POINTER(C.c_void_p), D]),
    "bqb_bound_nodes_fused": (C.c_int, [C.POINTER(BabNode), C.c_int, C.c_int, D]),
    "bqb_fused_fallbacks": (C.c_longlong, []),
    "bqb_fused_submit": (C.c_longlong, [C.POINTER(BabNode), C.c_int, C.c_int]),
    "bqb_fused_collect": (C.c_int, [C.c_longlong, C.POINTER(BabNode), D]),
    "bqb_fused_stats": (None, [D]),
    "bqb_fused_stats_reset": (None, []),
    "bqb_fused_profile": (None, [D]),
    "bqb_fused_launches": (C.c_longlong, []),
    "bqb_fused_phase_calls": (None, [C.POINTER(C.c_longlong)]),
    "bqb_fused_node_times": (C.c_int, [D, C.c_int]),
    "bqb_reset_incumbent": (None, [C.c_double]),
    "bqb_set_gw_hyperplanes": (None, [C.c_int]),
    "bqb_ipm_schedule_set": (None, [C.c_int, C.c_int]),
    "bqb_sdp_certificate": (C.c_int, [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double)]),
    "bqb_ipm_dual": (C.c_int, [C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                               C.POINTER(C.c_double)]),
    "bqb_certify_enable": (None, [C.c_int]),
    "bqb_certify_stats": (None, [C.POINTER(C.c_double), C.c_int]),
    "bqb_engine_profile_enable": (None, [C.c_int]),
    "bqb_engine_profile": (None, [C.POINTER(C.c_double), C.c_int]),
    "bqb_lambda_eta_profile": (None, [C.POINTER(C.c_double), C.c_int]),
    "bqb_ipm_coop_profile_enable": (None, [C.c_int]),
    "bqb_ipm_coop_profile": (None, [C.POINTER(C.c_double), C.c_int]),
    "bqb_ipm_autotune": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "bqb_warm_train": (C.c_int, [C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int, C.c_int, C.c_int, C.c_float,
                                 C.c_uint, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "bqb_warm_grad": (C.c_int, [C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int,
                                C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "bqb_warm_predict": (C.c_int, [C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int, D]),
    "bqb_warm_set_model": (C.c_int, [C.POINTER(C.c_float)]),
    "bqb_warm_enable": (None, [C.c_int]),
    "bqb_warm_record": (None, [C.c_int]),
    "bqb_warm_dataset": (C.c_longlong, [C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_longlong]),
    "bqb_warm_dataset_clear": (None, []),
    "bqb_warm_stats": (None, [C.POINTER(C.c_longlong), C.c_int]),
    "bqb_warm_features": (C.c_int, [D, D, C.c_int, I, D, C.c_int, C.c_double, C.c_double, C.c_void_p,
                                    C.POINTER(C.c_float)]),
    "bqb_warm_dims": (None, [C.POINTER(C.c_int)]),
    "bqb_set_heuristic_hook": (None, [C.c_void_p]),
    "bqb_heuristic_runs": (C.c_longlong, [C.c_int]),
    "bqb_bundle_iterations": (C.c_longlong, [C.c_int]),
    "bqb_set_root_effort": (None, [C.c_int]),
    "bqb_set_parent_start": (None, [C.c_int]),
    "bqb_bound_trace_enable": (None, [C.c_int]),
    "bqb_bound_trace": (C.c_int, [D, C.c_int]),
    "bqb_seed_engines": (C.c_int, [C.c_uint]),
    "bqb_kgon_sa": (C.c_int, [D, C.c_int, C.c_int, C.c_int, C.c_int, C.c_ulonglong, D, I]),
    "bqb_init": (C.c_int, [C.c_int]),
    "bqb_last_error": (C.c_char_p, []),
    "bqb_kernel_launches": (C.c_ulonglong, []),
    "bqb_stream": (C.c_void_p, []),
    "bqb_stats_enable": (None, [C.c_int]),
    "bqb_stats_reset": (None, []),
    "bqb_ipm_stats": (None, [D]),
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


def fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_float))


def colmajor(A: np.ndarray) -> np.ndarray:
    """Column-major flat copy (reference layout) of a square matrix."""
    return np.ascontiguousarray(np.asarray(A, dtype=np.float64).T).reshape(-1)


def from_colmajor(flat: np.ndarray, n: int) -> np.ndarray:
    return np.asarray(flat[: n * n]).reshape(n, n).T.copy()


def global_ptr(name: str, ctype):
    """The library's own copy of a reference global (standalone use)."""
    return ctype.in_dll(load(), name)


class SolveResult(C.Structure):
    """bqb_solve_result (include/bqb_gpu.h)."""
    _fields_ = [("best_value", C.c_double), ("root_bound", C.c_double), ("nodes", C.c_int),
                ("stopped", C.c_int), ("seconds", C.c_double), ("num_vertices", C.c_int),
                ("solution", C.c_int * NMAX)]


def make_params(**overrides) -> Params:
    """Parameters as the reference tests run them (its shipped `params` file),
    with overrides."""
    p = Params()
    vals = dict(PARAMS_FILE)
    vals.update(overrides)
    for k, v in vals.items():
        setattr(p, k, v)
    return p


def solve(adj: np.ndarray, threads: int = 1, fused_batch: int = 0, fused_depth: int = 4,
          gw_hyperplanes: int = 0, device_pool: bool = False, pool_nodes: int = 0, root_effort: bool = False,
          parent_start: bool = False, **param_overrides) -> dict:
    """Solve Max-Cut on ``adj`` to optimality (best-first B&B, GPU bounding;
    ``threads`` > 1 bounds that many nodes concurrently on engines;
    ``fused_batch`` > 0 bounds batches of up to that many nodes with the
    fused node kernel, ``fused_depth`` batches in flight; ``gw_hyperplanes``
    > 0: the engines' GW rounds project that many hyperplanes at once on
    the tensor cores; ``device_pool``: the whole tree in one persistent
    launch with the open-node pool on the device); ``root_effort``: the
    root runs every outer round of SDPbound unless pruned; ``parent_start``:
    with ``threads`` > 1, each child starts from its parent's final cuts and
    multipliers)."""
    lib = load()
    lib.bqb_set_gw_hyperplanes(int(gw_hyperplanes))
    lib.bqb_set_root_effort(1 if root_effort else 0)
    lib.bqb_set_parent_start(1 if parent_start else 0)
    A = np.ascontiguousarray(adj, dtype=np.float64)
    p = make_params(**param_overrides)
    res = SolveResult()
    pp = C.cast(C.pointer(p), C.c_void_p)
    rp = C.cast(C.pointer(res), C.c_void_p)
    if device_pool:
        rc = lib.bqb_solve_device(dptr(A), A.shape[0], pp, int(pool_nodes), rp)
    elif fused_batch > 0:
        rc = lib.bqb_solve_fused(dptr(A), A.shape[0], pp, int(fused_batch), int(fused_depth), rp)
    elif threads > 1:
        rc = lib.bqb_solve_parallel(dptr(A), A.shape[0], pp, int(threads), rp)
    else:
        rc = lib.bqb_solve(dptr(A), A.shape[0], pp, rp)
    if rc != 0:
        raise RuntimeError(f"bqb_solve failed: {lib.bqb_last_error().decode()}")
    nv = A.shape[0]
    sol = np.array(res.solution[: nv - 1], dtype=np.int32)
    return dict(best_value=res.best_value, root_bound=res.root_bound, nodes=res.nodes,
                seconds=res.seconds, stopped=bool(res.stopped), x=sol,
                solution=[i + 1 for i in range(nv - 1) if sol[i] == 1])


class GlobalArrays:
    """Allocates the reference-layout globals in a library (X, Z, X_test,
    dual_gamma, ..., cut arrays) and points the library's pointer globals at
    them, as src/allocate_free.c:8-42 does.  Keeps the buffers alive.

    Capacities follow the reference (src/biqbin.h:37-42): 50,000 cuts of
    each kind and 150,000 entries in the multiplier vectors, which SDPbound
    fills up to the current number of cuts (a 343-vertex torus root holds
    about 21,000).  The host bundle arrays (X_bundle, G, lambda, F) are read
    and written only by the drop-in bundle_method, for bundles of at most
    ``bundle_cap`` elements over at most ``g_rows`` cuts; SDPbound keeps its
    bundle on the device."""

    def __init__(self, cdll, N: int, bundle_cap: int = 64, g_rows: int = 20000, list_cap: int = 20000,
                 cut_cap: int = 50000):
        self.cdll = cdll
        self.N = N
        mmax = 3 * cut_cap
        dbl = {"X": N * N, "Z": N * N, "X_test": N * N, "X_bundle": N * N * bundle_cap,
               "dual_gamma": mmax, "dgamma": mmax, "gamma_test": mmax, "eta": mmax, "g": mmax,
               "lambda": bundle_cap, "F": bundle_cap, "G": g_rows * bundle_cap}
        self.arr = {name: np.zeros(size) for name, size in dbl.items()}
        self.cuts = (TriIneq * cut_cap)()
        self.lst = (TriIneq * list_cap)()
        self.pcuts = (PentIneq * cut_cap)()
        self.plst = (PentIneq * list_cap)()
        self.hcuts = (HeptIneq * cut_cap)()
        self.hlst = (HeptIneq * list_cap)()
        self.bind()

    def bind(self) -> None:
        """Point the library's globals at these buffers (again: a solve in
        between points them at the library's own)."""
        for name, a in self.arr.items():
            C.c_void_p.in_dll(self.cdll, name).value = a.ctypes.data
        for name, obj in (("Cuts", self.cuts), ("List", self.lst), ("Pent_Cuts", self.pcuts),
                          ("Pent_List", self.plst), ("Hepta_Cuts", self.hcuts), ("Hepta_List", self.hlst)):
            C.c_void_p.in_dll(self.cdll, name).value = C.addressof(obj)

    def __getitem__(self, name):
        return self.arr[name]


def set_params(cdll, p: Params) -> None:
    Params.in_dll(cdll, "params").__init__(*[getattr(p, f) for f, _ in Params._fields_])


def autotune_ipm(sizes, path=None, reps=2) -> dict:
    """Tune the multi-CTA IPM's grid for each size in `sizes` (n > 128) on
    the GPU (bqb_ipm_autotune) and, with `path`, write the schedule as JSON
    ({"n": {"grid": g, "ms": t}}) for load_ipm_schedule."""
    import json
    lib = load()
    table = {}
    for n in sizes:
        g = C.c_int()
        ms = C.c_double()
        if lib.bqb_ipm_autotune(int(n), int(reps), C.byref(g), C.byref(ms)) == 0:
            table[str(int(n))] = {"grid": int(g.value), "ms": float(ms.value)}
    if path:
        with open(path, "w") as fh:
            json.dump(table, fh, indent=1)
    return table


def load_ipm_schedule(path) -> dict:
    """Apply a schedule written by autotune_ipm."""
    import json
    lib = load()
    with open(path) as fh:
        table = json.load(fh)
    for n, e in table.items():
        lib.bqb_ipm_schedule_set(int(n), int(e["grid"]))
    return table
