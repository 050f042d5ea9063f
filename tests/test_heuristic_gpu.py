"""GPU parity: Goemans-Williamson rounding + 1-opt (src/heuristic.c).

Cut values and cuts are integers and must match bit-exactly: mc_1opt against
the oracle, and GW_heuristic / runHeuristic_unpacked against the reference
build from the same rand() state (both draw every random number from glibc
rand() in the same order; the test also checks the rand() state after the
call)."""
import ctypes as C

import numpy as np
import pytest

from helpers import O, instances
from parallel_biqbin_maxcut_b200 import _lib

libc = C.CDLL("libc.so.6")
libc.rand.restype = C.c_int


@pytest.mark.gpu
@pytest.mark.parametrize("nv,seed", [(10, 1), (60, 2), (101, 3), (343, 4)])
def test_mc_1opt_exact(lib, nv, seed):
    A = instances.torus3d(7, seed) if nv == 343 else instances.gnp_pm1(nv, 0.5, seed)
    L = O.create_subproblem(O.build_SP_L(A), np.zeros(nv - 1, int), np.zeros(nv - 1, int))
    n = L.shape[0]
    rng = np.random.default_rng(seed)
    Lc = _lib.colmajor(L)
    for _ in range(5):
        x0 = rng.choice(np.array([-1, 1], np.int32), n)
        xg = x0.copy()
        cost = lib.mc_1opt(_lib.iptr(xg), _lib.dptr(Lc), n)
        xo = x0.astype(np.int64).copy()
        cost_ref = O.mc_1opt(xo, L)
        assert cost == cost_ref
        assert np.array_equal(xg, xo)


def _node(N, k, seed):
    rng = np.random.default_rng(seed)
    xf = np.zeros(N, np.int32)
    sol = np.zeros(N, np.int32)
    idx = rng.choice(N, k, replace=False)
    xf[idx] = 1
    sol[idx] = rng.integers(0, 2, k)
    return xf, sol


@pytest.mark.gpu
@pytest.mark.parametrize("k,seed", [(0, 1), (10, 2), (35, 3)])
def test_gw_and_heuristic_match_reference(lib, lib_globals, ref, k, seed):
    SPL = ref.SP_L()
    N0 = SPL.shape[0]
    xf, sol = _node(N0 - 1, k, seed)
    L = O.create_subproblem(SPL, xf, sol)
    n = L.shape[0]
    Xm = O.ipm_mc_pk(L).X
    P0c = _lib.colmajor(SPL)
    Lc = _lib.colmajor(L)
    Xc = _lib.colmajor(Xm)
    Lf = np.linalg.cholesky(Xm)
    Zc = _lib.colmajor(Lf)
    refX = ref.gptr("X", C.c_double)
    refZ = ref.gptr("Z", C.c_double)
    for q in range(n * n):
        refX[q] = Xc[q]
        refZ[q] = Zc[q]
    lib_globals["X"][: n * n] = Xc
    lib_globals["Z"][: n * n] = Zc

    # one GW call on a fixed factor
    res = []
    for L_ in (ref.lib, lib):
        libc.srand(1000 + seed)
        x = np.zeros(N0 - 1, np.int32)
        v = L_.GW_heuristic(_lib.dptr(P0c), N0, _lib.dptr(Lc), n, _lib.iptr(xf), _lib.iptr(sol), _lib.iptr(x), N0)
        res.append((v, x.copy(), libc.rand()))
    assert res[0][0] == res[1][0]
    assert np.array_equal(res[0][1], res[1][1])
    assert res[0][2] == res[1][2]

    # the full heuristic (Cholesky of X, GW rounds, re-mixing)
    res = []
    for L_ in (ref.lib, lib):
        libc.srand(2000 + seed)
        x = np.zeros(N0 - 1, np.int32)
        v = L_.runHeuristic_unpacked(_lib.dptr(P0c), N0, _lib.dptr(Lc), n, _lib.iptr(xf), _lib.iptr(sol),
                                     _lib.iptr(x))
        res.append((v, x.copy(), libc.rand()))
    assert res[0][0] == res[1][0]
    assert np.array_equal(res[0][1], res[1][1])
    assert res[0][2] == res[1][2]


@pytest.mark.gpu
def test_heuristic_matches_oracle(lib, lib_globals):
    A = instances.gnp_unit(40, 0.5, 5)
    SPL = O.build_SP_L(A)
    N0 = SPL.shape[0]
    xf, sol = _node(N0 - 1, 6, 5)
    L = O.create_subproblem(SPL, xf, sol)
    n = L.shape[0]
    Xm = O.ipm_mc_pk(L).X
    lib_globals["X"][: n * n] = _lib.colmajor(Xm)
    P0c, Lc = _lib.colmajor(SPL), _lib.colmajor(L)
    libc.srand(77)
    x = np.zeros(N0 - 1, np.int32)
    v = lib.runHeuristic_unpacked(_lib.dptr(P0c), N0, _lib.dptr(Lc), n, _lib.iptr(xf), _lib.iptr(sol), _lib.iptr(x))
    after = libc.rand()
    libc.srand(77)
    xo = np.zeros(N0 - 1, np.int64)
    vo = O.runHeuristic_unpacked(SPL, L, xf, sol, xo, Xm)
    assert v == vo
    assert np.array_equal(x, xo)
    assert after == libc.rand()
    assert v == O.evaluateSolution(SPL, x)
