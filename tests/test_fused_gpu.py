"""Fused node bounding (bqb_bound_nodes_fused): one CTA bounds a whole node
on the device.

Parity: with the incumbent held at the optimum (the heuristic can then never
change it) and pentagonal / heptagonal separation off (the only other use of
random numbers), a node's bound does not depend on the random streams, and
the fused kernel runs the engine path's arithmetic (same IPM, lambda_eta,
bundle step and cut-operator code at the same thread count, the same
triangle list), so its bounds and fractional solutions must equal the serial
drop-in SDPbound (src/bounding.c) bit for bit.  The library is compiled
without contraction of multiplies and adds into FMAs (-fmad=false), so the
device bodies shared by the two kernels round identically in both.  With
the random streams in play every bound must still be an upper bound of the
node."""
import ctypes as C

import numpy as np
import pytest

from helpers import O, instances
from parallel_biqbin_maxcut_b200 import _lib

NV = 60


def _nodes(count, kmax, seed, nv=NV):
    out = (_lib.BabNode * count)()
    for q, (xf, sol) in enumerate(instances.random_fixings(nv, count, kmax, seed)):
        out[q].xfixed[: nv - 1] = [int(v) for v in xf]
        out[q].sol[: nv - 1] = [int(v) for v in sol]
        out[q].level = int(xf.sum())
    return out


def _copy(nodes):
    c = (_lib.BabNode * len(nodes))()
    C.memmove(c, nodes, C.sizeof(nodes))
    return c


def _serial(lib, nodes):
    SP = C.cast(C.c_void_p.in_dll(lib, "SP").value, C.POINTER(_lib.Problem))
    PP = C.cast(C.c_void_p.in_dll(lib, "PP").value, C.POINTER(_lib.Problem))
    return np.array([lib.Evaluate(C.byref(nodes[i]), SP, PP, 1) for i in range(len(nodes))])


@pytest.fixture(scope="module")
def solved(lib):
    A = instances.gnp_pm1(NV, 0.5, 11)
    r = _lib.solve(A, include_Pent=0, include_Hepta=0)
    assert lib.Bab_LBGet() == r["best_value"]
    return A, r


@pytest.mark.gpu
@pytest.mark.parametrize("kmax,seed", [(25, 31), (45, 32)])
def test_fused_bounds_equal_serial(lib, solved, kmax, seed):
    nodes = _nodes(40, kmax, seed)
    ser = _copy(nodes)
    want = _serial(lib, ser)
    f0 = lib.bqb_fused_fallbacks()
    got = np.zeros(len(nodes))
    assert lib.bqb_bound_nodes_fused(nodes, len(nodes), 1, _lib.dptr(got)) == 0
    assert lib.bqb_fused_fallbacks() == f0
    np.testing.assert_array_equal(got, want)
    for i in range(len(nodes)):
        assert list(nodes[i].fracsol[: NV - 1]) == list(ser[i].fracsol[: NV - 1])


@pytest.mark.gpu
def test_fused_bounds_with_kgon_separation(lib, solved):
    A, _ = solved
    _lib.set_params(lib, _lib.make_params())
    try:
        nodes = _nodes(24, 45, seed=33)
        b = np.zeros(len(nodes))
        assert lib.bqb_bound_nodes_fused(nodes, len(nodes), 1, _lib.dptr(b)) == 0
        SPL = O.build_SP_L(A)
        rng = np.random.default_rng(6)
        for i in range(len(nodes)):
            xf = np.array(nodes[i].xfixed[: NV - 1])
            sol = np.array(nodes[i].sol[: NV - 1])
            for _ in range(20):
                x = np.where(xf == 1, sol, rng.integers(0, 2, NV - 1))
                assert O.evaluateSolution(SPL, x) <= b[i] + 1e-6
    finally:
        _lib.set_params(lib, _lib.make_params(include_Pent=0, include_Hepta=0))


@pytest.mark.gpu
def test_fused_submit_collect_pipelined(lib, solved):
    """Eight batches in flight give the same bounds as one batch at a time
    (the incumbent is the optimum, so no batch can change another's)."""
    batches = [_nodes(20, 30, seed=40 + q) for q in range(8)]
    singles = []
    for b in batches:
        c = _copy(b)
        out = np.zeros(len(c))
        assert lib.bqb_bound_nodes_fused(c, len(c), 1, _lib.dptr(out)) == 0
        singles.append(out)
    outs = [np.zeros(len(b)) for b in batches]
    tickets = [lib.bqb_fused_submit(b, len(b), 1) for b in batches]
    assert all(t >= 0 for t in tickets)
    assert lib.bqb_fused_submit(batches[0], len(batches[0]), 1) == -1   # every pipe busy
    for t, b, o in zip(reversed(tickets), reversed(batches), reversed(outs)):
        assert lib.bqb_fused_collect(t, b, _lib.dptr(o)) == 0
    assert lib.bqb_fused_collect(tickets[0], batches[0], _lib.dptr(outs[0])) == 1   # already collected
    for o, s in zip(outs, singles):
        np.testing.assert_array_equal(o, s)


@pytest.mark.gpu
@pytest.mark.parametrize("depth", [8, 5])
def test_fused_rolling_window_fifo(lib, solved, depth):
    """A rolling window of `depth` submissions in flight, collected oldest
    first, for three times as many submissions as there are slots (the
    pattern of a benchmark that keeps the window full).  Submissions made
    while a launch runs are grouped into one launch; the launch record must
    not keep a submission slot once its own submission is collected, so no
    submission is ever refused.  Bounds equal one batch at a time."""
    nsub = 24
    batches = [_nodes(12, 30, seed=400 + q) for q in range(nsub)]
    singles = []
    for b in batches:
        c = _copy(b)
        out = np.zeros(len(c))
        assert lib.bqb_bound_nodes_fused(c, len(c), 1, _lib.dptr(out)) == 0
        singles.append(out)
    outs = [np.zeros(len(b)) for b in batches]
    lib.bqb_fused_stats_reset()
    window = []
    for q, b in enumerate(batches):
        if len(window) == depth:
            t, j = window.pop(0)
            assert lib.bqb_fused_collect(t, batches[j], _lib.dptr(outs[j])) == 0, lib.bqb_last_error()
        t = lib.bqb_fused_submit(b, len(b), 1)
        assert t >= 0, (q, lib.bqb_last_error())
        window.append((t, q))
    for t, j in window:
        assert lib.bqb_fused_collect(t, batches[j], _lib.dptr(outs[j])) == 0, lib.bqb_last_error()
    launches = lib.bqb_fused_launches()
    assert 1 <= launches < nsub        # submissions made during a launch were grouped
    for o, s in zip(outs, singles):
        np.testing.assert_array_equal(o, s)
    # nine uncollected submissions are refused, eight are accepted
    tickets = [lib.bqb_fused_submit(batches[q], len(batches[q]), 1) for q in range(8)]
    assert all(t >= 0 for t in tickets)
    assert lib.bqb_fused_submit(batches[8], len(batches[8]), 1) == -1
    for t, q in zip(tickets, range(8)):
        assert lib.bqb_fused_collect(t, batches[q], _lib.dptr(outs[q])) == 0


@pytest.mark.gpu
def test_pending_submissions_survive_a_problem_change(lib, solved):
    """Submissions made while a launch runs wait on the host; replacing the
    problem (process_adj_matrix) first launches them for the problem they
    were made for."""
    A, r = solved
    batches = [_nodes(24, 30, 60 + q) for q in range(3)]
    singles = []
    for b in batches:
        c = _copy(b)
        out = np.zeros(len(c))
        assert lib.bqb_bound_nodes_fused(c, len(c), 1, _lib.dptr(out)) == 0
        singles.append(out)
    tickets = [lib.bqb_fused_submit(b, len(b), 1) for b in batches]
    assert all(t >= 0 for t in tickets)
    B = instances.gnp_unit(NV, 0.5, 77)
    keep = np.ascontiguousarray(B, dtype=np.float64).copy()
    lib.process_adj_matrix(_lib.dptr(keep), NV)      # a different problem, same size
    outs = [np.zeros(len(b)) for b in batches]
    for t, b, o in zip(tickets, batches, outs):
        assert lib.bqb_fused_collect(t, b, _lib.dptr(o)) == 0
    for o, s in zip(outs, singles):
        np.testing.assert_array_equal(o, s)
    # the module's problem back for the tests that follow
    lib.process_adj_matrix(_lib.dptr(np.ascontiguousarray(A, dtype=np.float64).copy()), NV)


@pytest.mark.gpu
@pytest.mark.parametrize("kind,nv,seed", [("unit", 60, 2), ("pm1", 50, 4), ("qubo", 40, 6)])
def test_fused_solve_optimum(lib, kind, nv, seed):
    """B&B with fused batches reaches the serial solver's optimum."""
    if kind == "unit":
        A = instances.gnp_unit(nv, 0.5, seed)
    elif kind == "pm1":
        A = instances.gnp_pm1(nv, 0.5, seed)
    else:
        A = instances.qubo_to_maxcut(instances.qubo_dense(nv, 0.1, seed))
    serial = _lib.solve(A)
    fused = _lib.solve(A, fused_batch=64, fused_depth=4)
    assert fused["best_value"] == serial["best_value"]
    assert fused["root_bound"] == serial["root_bound"]
    assert O.evaluateSolution(O.build_SP_L(A), fused["x"]) == fused["best_value"]


@pytest.mark.gpu
def test_fused_solve_depth8_optimum(lib):
    """bqb_solve_fused with eight batches in flight reaches the optimum the
    reference's serial B&B printed (tests/golden/bab_optima.json)."""
    import json
    import os
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "bab_optima.json")) as fh:
        case = next(c for c in json.load(fh) if c["kind"] == "int10" and c["nv"] == 80)
    A = instances.gnp_int(case["nv"], 0.9, 10, case["seed"])
    r = _lib.solve(A, fused_batch=16, fused_depth=8)
    assert r["best_value"] == case["max_value"]
    assert O.evaluateSolution(O.build_SP_L(A), r["x"]) == r["best_value"]
