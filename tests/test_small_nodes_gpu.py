"""GPU: nodes with almost every variable fixed (subproblems of 1 to 9
vertices), bounded by the serial SDPbound, by engines and by the fused
kernel.

The reference's bounding is undefined on some of these nodes: with no
violated triangle inequality its bundle starts from a step size divided by
zero cuts and its BLAS calls reject the empty cut matrix
(src/bounding.c:122-131, src/bundle.c:63, 315), and k-gonal annealing on
fewer than k vertices reads past its permutation.  Such nodes are reached
when the heuristic is weak and the B&B dives.  Here every bound must be a
valid upper bound on the node's best completion (enumerated), and the
fractional solution must lie in [0, 1]."""
import ctypes as C
import itertools

import numpy as np
import pytest

from helpers import O, instances
from parallel_biqbin_maxcut_b200 import _lib

NV = 24


@pytest.fixture(scope="module")
def setup(lib):
    A = instances.gnp_pm1(NV, 0.5, 5)
    r = _lib.solve(A)
    return A, r


def _nodes(free_counts, seed):
    rng = np.random.default_rng(seed)
    out = (_lib.BabNode * len(free_counts))()
    for q, f in enumerate(free_counts):
        xf = np.ones(NV - 1, dtype=int)
        xf[rng.choice(NV - 1, f, replace=False)] = 0
        sol = rng.integers(0, 2, NV - 1) * xf
        out[q].xfixed[: NV - 1] = [int(v) for v in xf]
        out[q].sol[: NV - 1] = [int(v) for v in sol]
        out[q].level = int(xf.sum())
    return out


def _best_completion(SPL, xf, sol):
    free = np.flatnonzero(xf == 0)
    best = -np.inf
    for bits in itertools.product((0, 1), repeat=len(free)):
        x = np.where(xf == 1, sol, 0)
        x[free] = bits
        best = max(best, O.evaluateSolution(SPL, x))
    return best


def _check(nodes, bounds, SPL):
    for q in range(len(nodes)):
        xf = np.array(nodes[q].xfixed[: NV - 1])
        sol = np.array(nodes[q].sol[: NV - 1])
        assert np.isfinite(bounds[q])
        assert bounds[q] >= _best_completion(SPL, xf, sol) - 1e-6, q
        fs = np.array(nodes[q].fracsol[: NV - 1])
        assert np.all((fs >= -1e-9) & (fs <= 1 + 1e-9))


FREE = [0, 1, 2, 3, 4, 5, 6, 7, 8] * 2


@pytest.mark.gpu
@pytest.mark.parametrize("incumbent", ["optimum", "low"])
def test_small_nodes_serial_engines_fused(lib, setup, incumbent):
    A, r = setup
    SPL = O.build_SP_L(A)
    SP = C.cast(C.c_void_p.in_dll(lib, "SP").value, C.POINTER(_lib.Problem))
    PP = C.cast(C.c_void_p.in_dll(lib, "PP").value, C.POINTER(_lib.Problem))
    # "low": every node runs its bundle (no early pruning on the incumbent)
    lb = r["best_value"] if incumbent == "optimum" else -1e6

    nodes = _nodes(FREE, seed=3)
    lib.bqb_reset_incumbent(C.c_double(lb))
    serial = np.array([lib.Evaluate(C.byref(nodes[i]), SP, PP, 1) for i in range(len(nodes))])
    _check(nodes, serial, SPL)

    nodes = _nodes(FREE, seed=3)
    lib.bqb_reset_incumbent(C.c_double(lb))
    eng = np.zeros(len(nodes))
    assert lib.bqb_bound_nodes(nodes, len(nodes), 1, 4, None, _lib.dptr(eng)) == 0, lib.bqb_last_error()
    _check(nodes, eng, SPL)

    nodes = _nodes(FREE, seed=3)
    lib.bqb_reset_incumbent(C.c_double(lb))
    fused = np.zeros(len(nodes))
    assert lib.bqb_bound_nodes_fused(nodes, len(nodes), 1, _lib.dptr(fused)) == 0, lib.bqb_last_error()
    _check(nodes, fused, SPL)
    lib.bqb_reset_incumbent(C.c_double(r["best_value"]))
