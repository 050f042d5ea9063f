"""Concurrent node bounding (bqb_bound_nodes) and the parallel B&B
(bqb_solve_parallel): several engines bound nodes at the same time, each on
its own stream with its own cut lists and random stream.

Parity: with the incumbent held at the optimum (the heuristic can then never
change it) and pentagonal / heptagonal separation off (the only other use of
random numbers), a node's bound does not depend on the random stream, so
concurrent bounds must equal the serial drop-in SDPbound (src/bounding.c)
bit for bit, whatever engine bounds which node.  The parallel B&B must reach
the reference's optimum (the serial reference build, when present)."""
import ctypes as C

import numpy as np
import pytest

from helpers import O, instances
from parallel_biqbin_maxcut_b200 import _lib

NV = 60


def _nodes(count, kmax, seed):
    out = (_lib.BabNode * count)()
    for q, (xf, sol) in enumerate(instances.random_fixings(NV, count, kmax, seed)):
        out[q].xfixed[: NV - 1] = [int(v) for v in xf]
        out[q].sol[: NV - 1] = [int(v) for v in sol]
        out[q].level = int(xf.sum())
    return out


def _copy(nodes):
    c = (_lib.BabNode * len(nodes))()
    C.memmove(c, nodes, C.sizeof(nodes))
    return c


@pytest.fixture(scope="module")
def solved(lib):
    """SP set up for a G(60, 0.5) +-1 instance, incumbent = its optimum."""
    A = instances.gnp_pm1(NV, 0.5, 11)
    r = _lib.solve(A, include_Pent=0, include_Hepta=0)
    assert lib.Bab_LBGet() == r["best_value"]
    return A, r


def _serial_bounds(lib, nodes):
    SP = C.cast(C.c_void_p.in_dll(lib, "SP").value, C.POINTER(_lib.Problem))
    PP = C.cast(C.c_void_p.in_dll(lib, "PP").value, C.POINTER(_lib.Problem))
    return np.array([lib.Evaluate(C.byref(nodes[i]), SP, PP, 1) for i in range(len(nodes))])


@pytest.mark.gpu
@pytest.mark.parametrize("threads", [1, 4, 16])
def test_concurrent_bounds_equal_serial(lib, solved, threads):
    nodes = _nodes(24, 25, seed=21)
    ser_nodes = _copy(nodes)
    serial = _serial_bounds(lib, ser_nodes)
    conc = np.zeros(len(nodes))
    assert lib.bqb_bound_nodes(nodes, len(nodes), 1, threads, None, _lib.dptr(conc)) == 0
    np.testing.assert_array_equal(conc, serial)
    for i in range(len(nodes)):
        assert list(nodes[i].fracsol[: NV - 1]) == list(ser_nodes[i].fracsol[: NV - 1])


@pytest.mark.gpu
def test_concurrent_bounds_device_matrices(lib, solved):
    """L_dev: the subproblem matrices createSubproblem builds, already in
    device memory, give the same bounds as building them on the host."""
    import torch
    SP = C.cast(C.c_void_p.in_dll(lib, "SP").value, C.POINTER(_lib.Problem))
    nodes = _nodes(12, 25, seed=22)
    mats = []
    for i in range(len(nodes)):
        buf = np.zeros(NV * NV)
        prob = _lib.Problem()
        prob.L = buf.ctypes.data_as(C.POINTER(C.c_double))
        lib.createSubproblem(C.byref(nodes[i]), SP, C.byref(prob))
        mats.append(torch.from_numpy(buf[: prob.n * prob.n].copy()).cuda())
    ptrs = (C.c_void_p * len(nodes))(*[m.data_ptr() for m in mats])
    torch.cuda.synchronize()
    ref = np.zeros(len(nodes))
    host_nodes = _copy(nodes)
    assert lib.bqb_bound_nodes(host_nodes, len(nodes), 1, 4, None, _lib.dptr(ref)) == 0
    dev = np.zeros(len(nodes))
    assert lib.bqb_bound_nodes(nodes, len(nodes), 1, 4, ptrs, _lib.dptr(dev)) == 0
    np.testing.assert_array_equal(dev, ref)


@pytest.mark.gpu
def test_concurrent_bounds_with_kgon_separation(lib, solved):
    """Random streams in play (pentagonal / heptagonal annealing): every
    bound is still an upper bound on the node's best cut."""
    A, r = solved
    _lib.set_params(lib, _lib.make_params())
    try:
        nodes = _nodes(16, 45, seed=23)
        b = np.zeros(len(nodes))
        assert lib.bqb_bound_nodes(nodes, len(nodes), 1, 8, None, _lib.dptr(b)) == 0
        SPL = O.build_SP_L(A)
        rng = np.random.default_rng(5)
        for i in range(len(nodes)):
            xf = np.array(nodes[i].xfixed[: NV - 1])
            sol = np.array(nodes[i].sol[: NV - 1])
            # a few feasible completions of the node: none may beat its bound
            for _ in range(20):
                x = np.where(xf == 1, sol, rng.integers(0, 2, NV - 1))
                assert O.evaluateSolution(SPL, x) <= b[i] + 1e-6
    finally:
        _lib.set_params(lib, _lib.make_params(include_Pent=0, include_Hepta=0))


@pytest.mark.gpu
@pytest.mark.parametrize("kind,nv,seed", [("unit", 60, 2), ("pm1", 50, 4), ("qubo", 40, 6)])
def test_parallel_solve_optimum(lib, kind, nv, seed):
    if kind == "unit":
        A = instances.gnp_unit(nv, 0.5, seed)
    elif kind == "pm1":
        A = instances.gnp_pm1(nv, 0.5, seed)
    else:
        A = instances.qubo_to_maxcut(instances.qubo_dense(nv, 0.1, seed))
    serial = _lib.solve(A)
    par = _lib.solve(A, threads=8)
    assert par["best_value"] == serial["best_value"]
    assert O.evaluateSolution(O.build_SP_L(A), par["x"]) == par["best_value"]
    # the parallel solver bounds its root on an engine, whose heuristic and
    # k-gonal separation draw from their own streams: the root bound is the
    # serial one's only up to those streams, and above the optimum
    assert par["root_bound"] >= par["best_value"]
    assert abs(par["root_bound"] - serial["root_bound"]) <= 1e-3 * abs(serial["root_bound"])


@pytest.mark.gpu
def test_root_effort_and_parent_start(lib):
    """Root effort (no early give-up at the root) and parent start (children
    begin from their parent's final cuts and multipliers) change only how
    fast the bound falls: the optimum is the serial solver's, the root bound
    with root effort is no larger than without it for the same random
    streams (the bundle's objective never rises, and the first rounds are
    the same), and children keep some parent starts."""
    A = instances.gnp_pm1(50, 0.5, 4)
    serial = _lib.solve(A)
    assert lib.bqb_seed_engines(2021) == 0
    plain = _lib.solve(A, threads=8)
    assert lib.bqb_seed_engines(2021) == 0
    effort = _lib.solve(A, threads=8, root_effort=True)
    assert effort["root_bound"] <= plain["root_bound"] + 1e-9 * abs(plain["root_bound"])
    st = (C.c_longlong * 2)()
    lib.bqb_warm_stats(st, 1)
    assert lib.bqb_seed_engines(2021) == 0
    ps = _lib.solve(A, threads=8, parent_start=True)
    lib.bqb_warm_stats(st, 1)
    lib.bqb_set_parent_start(0)
    for r in (plain, effort, ps):
        assert r["best_value"] == serial["best_value"]
        assert O.evaluateSolution(O.build_SP_L(A), r["x"]) == r["best_value"]
    if ps["nodes"] > 1:
        assert st[0] + st[1] > 0 and st[0] > 0, list(st)
