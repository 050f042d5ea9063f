"""The reference's Python module API (parallel_biqbin_maxcut_b200.biqbin):
input readers and the QUBO <-> Max-Cut conversion on CPU (pinned by the
reference's shipped QUBO test fixture when the reference is present), and
run() / set_heuristic / set_read_data end to end on the GPU against the
golden B&B optima."""
from __future__ import annotations

import itertools
import json
import os

import numpy as np
import pytest

from helpers import ref_path
from parallel_biqbin_maxcut_b200 import _lib, biqbin, instances

HERE = os.path.dirname(os.path.abspath(__file__))
REF_QUBOS = [ref_path("tests", "qubos", "40", "kcluster40_025_10_1.json"),
             ref_path("tests", "qubos", "80", "kcluster80_025_20_1.json")]


def brute_maxcut(A):
    """Max cut with the last vertex on side 0, and its 0/1 vector."""
    n = A.shape[0]
    best, bx = -np.inf, None
    for bits in itertools.product((0, 1), repeat=n - 1):
        x = np.array(bits + (0,))
        v = float(sum(A[i, j] for i in range(n) for j in range(i + 1, n) if x[i] != x[j]))
        if v > best:
            best, bx = v, x
    return best, bx


def brute_qubo_min(Q):
    n = Q.shape[0]
    return min(float(np.array(b) @ Q @ np.array(b)) for b in itertools.product((0, 1), repeat=n))


def test_qubo_to_maxcut_matches_generator_restatement():
    Q = instances.qubo_dense(12, 0.3, 7)
    A, g = biqbin.qubo_to_maxcut(Q)
    assert g == 1
    assert np.array_equal(A, instances.qubo_to_maxcut(Q))


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_qubo_maxcut_equivalence_small(seed):
    rng = np.random.default_rng(seed)
    n = 8
    Q = rng.integers(-5, 6, (n, n)).astype(float) * 2
    A, g = biqbin.qubo_to_maxcut(Q, optimize_input=True)
    cut, x = brute_maxcut(A)
    qmin = brute_qubo_min(Q)
    # the cut of the (n+1)-vertex graph is -min x'Qx / gcd
    assert cut * g == pytest.approx(-qmin)
    sel = [i + 1 for i in range(n + 1) if x[i] == 1]
    qsol, qx, mcx = biqbin.maxcut_to_qubo_solution(sel, n)
    assert float(np.array(qx) @ Q @ np.array(qx)) == pytest.approx(qmin)
    assert mcx == x.tolist() and qsol == [i + 1 for i in range(n) if qx[i] == 1]


def test_maxcut_solution_flip_side():
    # a cut that puts the last vertex on side 1 converts through the flip
    Q = np.array([[-3.0, 2.0], [2.0, -1.0]])
    A, _ = biqbin.qubo_to_maxcut(Q)
    qsol, qx, _ = biqbin.maxcut_to_qubo_solution([3], 2)   # {v3} vs {v1, v2}
    assert qx == [1, 1]
    qsol, qx, _ = biqbin.maxcut_to_qubo_solution([1], 2)
    assert qx == [1, 0]


def test_sparse_json_roundtrip_and_duplicates(tmp_path):
    Q = instances.qubo_dense(9, 0.4, 3)
    p = tmp_path / "q.json"
    p.write_text(json.dumps({"qubo": biqbin.to_sparse(Q)}))
    assert np.array_equal(biqbin.read_json_qubo(str(p)), Q)
    d = {"shape": [3, 3], "row": [0, 0, 1], "col": [1, 1, 2], "data": [1, 2, 5]}
    (tmp_path / "a.json").write_text(json.dumps({"adjacency": d}))
    A = biqbin.read_json_adjacency(str(tmp_path / "a.json"))
    assert A[0, 1] == 3 and A[1, 2] == 5 and A.sum() == 8
    d["data"] = [0.5, 1, 1]
    (tmp_path / "b.json").write_text(json.dumps({"adjacency": d}))
    with pytest.raises(ValueError):
        biqbin.read_json_adjacency(str(tmp_path / "b.json"))
    with pytest.raises(ValueError):
        biqbin.qubo_to_maxcut(np.array([[0.5, 0.0], [0.0, 1.0]]))


def test_default_heuristic_argument_checks():
    good = np.zeros((4, 4))
    iv = np.zeros(3, dtype=np.int32)
    with pytest.raises(TypeError, match="dtype"):
        biqbin.default_heuristic(good.astype(np.float32), good, iv, iv, iv)
    with pytest.raises(TypeError, match="square"):
        biqbin.default_heuristic(np.zeros((4, 3)), good, iv, iv, iv)
    with pytest.raises(TypeError, match="dimensions"):
        biqbin.default_heuristic(good, good, np.zeros((3, 1), dtype=np.int32), iv, iv)
    with pytest.raises(TypeError, match="C-contiguous"):
        biqbin.default_heuristic(np.asfortranarray(np.arange(16.0).reshape(4, 4)), good, iv, iv, iv)
    ro = iv.copy()
    ro.setflags(write=False)
    with pytest.raises(TypeError, match="writable"):
        biqbin.default_heuristic(good, good, iv, iv, ro)


def test_default_read_data_rudy(tmp_path):
    A = instances.gnp_int(12, 0.6, 7, seed=4)
    p = tmp_path / "g.rudy"
    instances.write_rudy(str(p), A)
    assert np.array_equal(biqbin.default_read_data(str(p)), A)
    with pytest.raises(ValueError):
        biqbin.default_read_data(str(tmp_path / "missing"))


@pytest.mark.parametrize("path", REF_QUBOS)
def test_reference_qubo_fixture_conversion(path):
    """The reference's shipped QUBO tests (tests/qubos/40 and 80) read by our
    JSON reader: the expected Max-Cut solution converts to the expected QUBO
    x, whose value x'Qx is the expected QUBO value."""
    if not os.path.exists(path):
        pytest.skip("reference test fixtures not present")
    Q = biqbin.read_json_qubo(path)
    with open(path + "-expected_output.json") as fh:
        exp = json.load(fh)
    n = Q.shape[0]
    qsol, qx, mcx = biqbin.maxcut_to_qubo_solution(exp["maxcut"]["solution"], n)
    assert qx == [int(v) for v in exp["qubo"]["x"]]
    assert mcx == [int(v) for v in exp["maxcut"]["x"]]
    assert float(np.array(qx) @ Q @ np.array(qx)) == pytest.approx(exp["qubo"]["computed_val"])
    A, g = biqbin.qubo_to_maxcut(Q)
    x = np.array(mcx)
    cut = float(sum(A[i, j] for i in range(n + 1) for j in range(i + 1, n + 1) if x[i] != x[j]))
    assert cut * g == pytest.approx(exp["maxcut"]["computed_val"])


def test_reference_qubo_fixture_through_reference_bab(tmp_path):
    """tests/qubos/40 converted by our QUBO -> Max-Cut conversion and solved
    by the reference build's own B&B: the expected Max-Cut value (its
    tests/test.sh compares this line)."""
    import re
    import subprocess
    from oracle import refbind
    path = REF_QUBOS[0]
    if not (os.path.exists(path) and refbind.available()):
        pytest.skip("reference fixtures or build absent")
    Q = biqbin.read_json_qubo(path)
    with open(path + "-expected_output.json") as fh:
        exp = json.load(fh)
    A, g = biqbin.qubo_to_maxcut(Q)
    inst, prm = tmp_path / "q.rudy", tmp_path / "params"
    instances.write_rudy(str(inst), A)
    with open(ref_path("params")) as fi:
        prm.write_text(fi.read())
    out = subprocess.run([refbind.REF_BAB, str(inst), str(prm)], capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, OPENBLAS_NUM_THREADS="1")).stdout
    best = float(re.search(r"Maximum value = (\S+)", out).group(1))
    assert best * g == pytest.approx(exp["maxcut"]["computed_val"])


@pytest.mark.skipif(not os.path.exists(ref_path("biqbin_base.py")), reason="reference Python layer not present")
def test_reference_python_layer_imports_this_module(tmp_path, monkeypatch):
    """The reference's biqbin_base.py imports its six functions from this
    module: its solvers install their overrides here, and its default data
    getter reads a Rudy file through our default_read_data."""
    import importlib
    import sys
    monkeypatch.setattr(sys, "dont_write_bytecode", True)   # nothing is written next to the reference
    monkeypatch.setitem(sys.modules, "biqbin", biqbin)
    monkeypatch.syspath_prepend(ref_path())
    monkeypatch.delitem(sys.modules, "biqbin_base", raising=False)
    base = importlib.import_module("biqbin_base")
    try:
        A = instances.gnp_int(10, 0.5, 5, seed=2)
        p = tmp_path / "g.rudy"
        instances.write_rudy(str(p), A)
        solver = base.MaxCutSolver(base.DataGetterMaxCutDefault(str(p)), "params")
        assert biqbin._heuristic is not None and biqbin._read_data is not None
        assert np.array_equal(biqbin._read_data(), A)
        assert solver.get_rank() == 0
        (tmp_path / "a.json").write_text(json.dumps({"adjacency": biqbin.to_sparse(A)}))
        assert np.array_equal(base.DataGetterAdjacencyJson(str(tmp_path / "a.json")).read_file(), A)
    finally:
        biqbin._clean()
        sys.modules.pop("biqbin_base", None)


# ---- GPU: run() end to end ------------------------------------------------

def _golden(kind, nv, seed):
    with open(os.path.join(HERE, "golden", "bab_optima.json")) as fh:
        for r in json.load(fh):
            if (r["kind"], r["nv"], r["seed"]) == (kind, nv, seed):
                return r
    raise KeyError((kind, nv, seed))


def _params_file(tmp_path):
    p = tmp_path / "params"
    instances.write_params(str(p), _lib.PARAMS_FILE)
    return str(p)


def _cut_value(A, solution):
    x = np.zeros(A.shape[0], dtype=int)
    x[np.asarray(solution, dtype=int) - 1] = 1
    return float(sum(A[i, j] for i in range(len(x)) for j in range(i + 1, len(x)) if x[i] != x[j]))


@pytest.mark.gpu
@pytest.mark.parametrize("solver", ["auto", "serial", "engines"])
def test_run_rudy_instance(tmp_path, solver):
    A = instances.gnp_unit(40, 0.5, 1)
    g = _golden("unit", 40, 1)
    p = tmp_path / "g.rudy"
    instances.write_rudy(str(p), A)
    r = biqbin.run("biqbin", str(p), _params_file(tmp_path), 0, solver=solver)
    assert r["maxcut"]["computed_val"] == g["max_value"]
    assert _cut_value(A, r["maxcut"]["solution"]) == g["max_value"]
    md = r["meta_data"]
    assert md["eval_bab_nodes"] >= 1 and md["heuristic_run_count"] >= 1
    assert md["time_limit_reached"] is False and md["num_workers_used"] == 1


@pytest.mark.gpu
def test_run_qubo_with_python_heuristic_and_reader(tmp_path):
    """QUBOSolver's flow: a read_data override returning the converted QUBO
    and a Python heuristic that calls default_heuristic, as biqbin_base.py's
    solvers install them."""
    Q = instances.qubo_dense(30, 0.1, 4)
    g = _golden("qubo", 30, 4)
    qp = tmp_path / "q.json"
    qp.write_text(json.dumps({"qubo": biqbin.to_sparse(Q)}))
    calls = []

    def heuristic(L0, L, xfixed, sol_X, x):
        calls.append(L.shape[0])
        assert L0.shape == (31, 31) and xfixed.shape == (30,) and x.dtype == np.int32
        return biqbin.default_heuristic(L0, L, xfixed, sol_X, x)

    biqbin.set_read_data(lambda: biqbin.qubo_to_maxcut(biqbin.read_json_qubo(str(qp)))[0])
    biqbin.set_heuristic(heuristic)
    r = biqbin.run("biqbin", str(qp), _params_file(tmp_path), 0)
    assert r["maxcut"]["computed_val"] == g["max_value"]
    assert r["meta_data"]["heuristic_run_count"] == len(calls) >= 1
    _, qx, _ = biqbin.maxcut_to_qubo_solution(r["maxcut"]["solution"], 30)
    assert float(np.array(qx) @ Q @ np.array(qx)) == pytest.approx(-g["max_value"])
    # the overrides are dropped after the run: the next run uses the file reader
    assert biqbin._heuristic is None and biqbin._read_data is None


def _one_opt_heuristic(A, seed=0, restarts=3):
    """A Python heuristic in the reference's contract that does not call the
    library: random completions of the fixed part improved by 1-opt on the
    adjacency (the last vertex stays on side 0)."""
    rng = np.random.default_rng(seed)
    nv = A.shape[0]

    def heuristic(L0, L, xfixed, sol_X, x):
        free = np.flatnonzero(xfixed == 0)
        best_v, best_x = -np.inf, None
        for _ in range(restarts):
            xx = np.zeros(nv, dtype=np.int64)
            xx[:-1] = np.where(xfixed == 1, sol_X, 0)
            xx[free] = rng.integers(0, 2, len(free))
            s = 2.0 * xx - 1.0
            while len(free):
                gain = s[free] * (A[free] @ s)   # cut change of flipping each free vertex
                j = int(np.argmax(gain))
                if gain[j] <= 1e-9:
                    break
                s[free[j]] = -s[free[j]]
            xx = (s > 0).astype(np.int64)
            v = float(np.sum(np.triu(A, 1) * (xx[:, None] != xx[None, :])))
            if v > best_v:
                best_v, best_x = v, xx
        x[:] = best_x[:-1]
        return best_v

    return heuristic


@pytest.mark.gpu
def test_python_heuristic_replaces_the_gpu_one(tmp_path):
    """A heuristic that never calls the library (1-opt in numpy) drives the
    B&B to the optimum; every node's heuristic is the Python one."""
    A = instances.gnp_pm1(40, 0.5, 3)
    g = _golden("pm1", 40, 3)
    p = tmp_path / "g.rudy"
    instances.write_rudy(str(p), A)
    heur = _one_opt_heuristic(A)
    n_calls = [0]

    def counted(*args):
        n_calls[0] += 1
        return heur(*args)

    biqbin.set_heuristic(counted)
    r = biqbin.run("biqbin", str(p), _params_file(tmp_path), 0)
    assert r["maxcut"]["computed_val"] == g["max_value"]
    assert _cut_value(A, r["maxcut"]["solution"]) == g["max_value"]
    assert n_calls[0] == r["meta_data"]["heuristic_run_count"] >= 1
