"""The reference's Python extension-module API over this library.

The reference's Python layer (``biqbin_base.py``: ``MaxCutSolver``,
``QUBOSolver``, the data getters and parsers) imports a pybind11 module
``biqbin`` (``src/wrapper.cpp:283-291``) with these functions:

    run(prog_name, problem_instance_name, params_file, time_limit) -> dict
    set_heuristic(func), default_heuristic(P0_L, P_L, xfixed, sol_X, x)
    set_read_data(func), default_read_data(instance) -> adjacency
    get_rank()

This module provides the same functions, with the same arguments, result
dictionary and errors, on the GPU bounding path, so the reference's Python
code runs unchanged with ``biqbin`` resolved to this module (for example
``sys.modules["biqbin"] = parallel_biqbin_maxcut_b200.biqbin`` before it is
imported).  It also carries the input formats of that layer: the Rudy edge
list, the JSON sparse-COO adjacency and QUBO files, and the QUBO to Max-Cut
conversion (``biqbin_base.py:186-258``).

One process, one GPU: ``get_rank()`` is 0, and ``run`` bounds the nodes of
its best-first B&B either one at a time on the library's default engine
(when a Python heuristic is set, since it is called per node) or in batches
with the fused node kernel.
"""
from __future__ import annotations

import ctypes as C
import json
import time as _time

import numpy as np

from . import _lib

_heuristic = None
_read_data = None
_callback = None            # keeps the C callback object alive during run()

_HEUR_CFUNC = C.CFUNCTYPE(C.c_double, C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double), C.c_int,
                          C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int))


def set_heuristic(func) -> None:
    """Use ``func(P0_L, P_L, xfixed, sol_X, x) -> float`` as the heuristic of
    every node (src/wrapper.cpp:38-40, 205-227)."""
    global _heuristic
    _heuristic = func


def set_read_data(func) -> None:
    """Use ``func() -> adjacency`` to read the instance (src/wrapper.cpp:42-44, 240-255)."""
    global _read_data
    _read_data = func


def get_rank() -> int:
    return 0


def _check_array(a, dtype, ndim: int, name: str) -> None:
    # the checks of src/wrapper.cpp:60-96, with its messages
    if not isinstance(a, np.ndarray) or a.dtype != dtype:
        raise TypeError(f"{name} must have dtype {np.dtype(dtype).name}")
    if a.ndim != ndim:
        raise TypeError(f"{name} must have {ndim} dimensions, got {a.ndim}")
    if ndim == 2 and a.shape[0] != a.shape[1]:
        raise TypeError(f"{name} must be square (shape[0] == shape[1]), got shape {tuple(a.shape)}")
    if not a.flags.c_contiguous:
        raise TypeError(f"{name} must be row-major (C-contiguous).")
    if not a.flags.writeable:
        raise TypeError(f"{name} must be writable.")


def default_heuristic(P0_L: np.ndarray, P_L: np.ndarray, xfixed: np.ndarray, sol_X: np.ndarray,
                      x: np.ndarray) -> float:
    """runHeuristic_unpacked (src/heuristic.c:19-115) on the GPU; x receives the
    0/1 solution.  The library's global X must hold the node's X (it does
    while a node is being bounded)."""
    _check_array(P0_L, np.float64, 2, "P0_L")
    _check_array(P_L, np.float64, 2, "P_L")
    _check_array(xfixed, np.int32, 1, "xfixed")
    _check_array(sol_X, np.int32, 1, "node_sol_x")
    _check_array(x, np.int32, 1, "x")
    lib = _lib.load()
    return lib.runHeuristic_unpacked(_lib.dptr(P0_L), P0_L.shape[0], _lib.dptr(P_L), P_L.shape[0],
                                     _lib.iptr(xfixed), _lib.iptr(sol_X), _lib.iptr(x))


def default_read_data(instance: str) -> np.ndarray:
    """The Rudy edge-list reader (src/process_input.c:201-253): n x n adjacency."""
    lib = _lib.load()
    n = C.c_int()
    p = lib.readData(instance.encode(), C.byref(n))
    if not p:
        raise ValueError(f"cannot read instance {instance}")
    A = np.ctypeslib.as_array(p, shape=(n.value * n.value,)).copy().reshape(n.value, n.value)
    C.CDLL("libc.so.6").free(C.cast(p, C.c_void_p))
    return A


def _from_sparse(d: dict) -> np.ndarray:
    """Dense matrix of a JSON sparse-COO dict {shape, row, col, data}
    (biqbin_base.py:33-46: duplicates are summed)."""
    M = np.zeros(tuple(d["shape"]), dtype=np.float64)
    np.add.at(M, (np.asarray(d["row"], dtype=np.int64), np.asarray(d["col"], dtype=np.int64)),
              np.asarray(d["data"], dtype=np.float64))
    return M


def read_json_adjacency(path: str) -> np.ndarray:
    """Adjacency from a JSON file with key "adjacency" (biqbin_base.py:77-91);
    every weight must be an integer."""
    with open(path) as fh:
        A = _from_sparse(json.load(fh)["adjacency"])
    if not np.all(A == np.round(A)):
        raise ValueError("All values in the adjacency matrix need to be integers!")
    return A


def read_json_qubo(path: str) -> np.ndarray:
    """QUBO matrix from a JSON file with key "qubo" (biqbin_base.py:186-218)."""
    with open(path) as fh:
        return _from_sparse(json.load(fh)["qubo"])


def to_sparse(M) -> dict:
    """JSON-serialisable sparse-COO dict of a dense matrix (the reference's
    utils.to_sparse format)."""
    M = np.asarray(M, dtype=np.float64)
    r, c = np.nonzero(M)
    return {"shape": list(M.shape), "nnz": int(len(r)), "row": r.tolist(), "col": c.tolist(),
            "data": M[r, c].tolist()}


def qubo_to_maxcut(Q: np.ndarray, optimize_input: bool = False):
    """(adjacency, gcd): the (n+1)-vertex Max-Cut equivalent of min x'Qx
    (biqbin_base.py:230-258); with optimize_input the symmetrised QUBO is
    divided by the gcd of its entries."""
    from functools import reduce
    from math import gcd as _gcd
    qs = 0.5 * (Q.T + Q)
    if not np.all(qs == np.round(qs)):
        raise ValueError("All QUBO values need to be integers!")
    g = 1
    if optimize_input:
        vals = set(int(v) for v in qs.flatten())
        d = reduce(_gcd, vals)
        if d > 1:
            qs = qs / d
            g = d
    qe = -qs.sum(axis=1)
    qs = qs.copy()
    np.fill_diagonal(qs, 0.0)
    n = Q.shape[0]
    A = np.zeros((n + 1, n + 1))
    A[:n, :n] = qs
    A[:n, n] = qe
    A[n, :n] = qe
    return A, g


def maxcut_to_qubo_solution(maxcut_solution, n: int):
    """(qubo solution vertices, qubo x, maxcut x) from the 1-based cut
    vertices of the (n+1)-vertex Max-Cut (biqbin_base.py:260-283)."""
    sel = np.asarray(maxcut_solution, dtype=int) - 1
    s = np.ones(n + 1)
    xx = np.zeros(n + 1, dtype=int)
    xx[sel] = 1
    s[sel] = -1
    s *= -s[-1]
    y = (0.5 * (s + 1))[:-1]
    return (np.nonzero(y)[0] + 1).tolist(), y.astype(int).tolist(), xx.tolist()


def run(prog_name: str, problem_instance_name: str, params_file: str, time_limit: int = 0,
        solver: str = "auto") -> dict:
    """Solve the instance to optimality and return src/wrapper.cpp:123-150's
    result dictionary.  solver: "auto" (one node at a time on the default
    engine when a Python heuristic is set, since it is called per node, else
    the fused node kernel), "fused", "serial" or "engines" (16 nodes bounded
    at once).  heuristic_run_count counts the heuristic runs of every node
    (the Python function's calls when one is set; the reference counts those
    calls, src/wrapper.cpp:212).  A Python heuristic is called by the serial
    solver only."""
    global _callback
    lib = _lib.load()
    assert lib.bqb_init(-1) == 0, lib.bqb_last_error()
    try:
        if _read_data is not None:
            adj = np.asarray(_read_data())
            _check_array(adj, np.float64, 2, "adj")
        else:
            adj = default_read_data(problem_instance_name)
        p = _lib.Params()
        if lib.bqb_read_params(params_file.encode(), C.byref(p)) != 0:
            raise FileNotFoundError(f"cannot read parameters file {params_file}")
        p.time_limit = int(time_limit)
        mode = solver
        if mode == "auto":
            mode = "serial" if _heuristic is not None else "fused"
        if _heuristic is not None:
            heur = _heuristic

            def _cb(P0, N0, PL, n, xf, sx, x):
                N = N0 - 1
                P0_L = np.ctypeslib.as_array(P0, shape=(N0, N0))
                P_L = np.ctypeslib.as_array(PL, shape=(n, n))
                return float(heur(P0_L, P_L, np.ctypeslib.as_array(xf, shape=(N,)),
                                  np.ctypeslib.as_array(sx, shape=(N,)), np.ctypeslib.as_array(x, shape=(N,))))

            _callback = _HEUR_CFUNC(_cb)
            lib.bqb_set_heuristic_hook(C.cast(_callback, C.c_void_p))
        lib.bqb_heuristic_runs(1)
        lib.bqb_fused_stats_reset()
        res = _lib.SolveResult()
        A = np.ascontiguousarray(adj, dtype=np.float64)
        pp, rp = C.cast(C.pointer(p), C.c_void_p), C.cast(C.pointer(res), C.c_void_p)
        t0 = _time.perf_counter()
        if mode == "fused":
            rc = lib.bqb_solve_fused(_lib.dptr(A), A.shape[0], pp, 296, 4, rp)
        elif mode == "engines":
            rc = lib.bqb_solve_parallel(_lib.dptr(A), A.shape[0], pp, 16, rp)
        else:
            rc = lib.bqb_solve(_lib.dptr(A), A.shape[0], pp, rp)
        elapsed = _time.perf_counter() - t0
        if rc != 0:
            raise RuntimeError(f"solve failed: {lib.bqb_last_error().decode()}")
        fused_calls = (C.c_longlong * 11)()
        lib.bqb_fused_phase_calls(fused_calls)
        heur_runs = int(lib.bqb_heuristic_runs(0)) + int(fused_calls[2])
        nv = A.shape[0]
        sol = np.array([i + 1 for i in range(nv - 1) if res.solution[i] == 1], dtype=np.int32)
        return {
            "meta_data": {"time": elapsed, "time_limit_reached": bool(res.stopped),
                          "eval_bab_nodes": int(res.nodes),
                          "heuristic_run_count": heur_runs,
                          "num_workers_used": 1},
            "maxcut": {"computed_val": float(res.best_value), "solution": sol},
        }
    finally:
        # src/wrapper.cpp:50-54: the overrides are dropped after every run
        lib.bqb_set_heuristic_hook(None)
        _callback = None
        _clean()


def _clean() -> None:
    global _heuristic, _read_data
    _heuristic = None
    _read_data = None
