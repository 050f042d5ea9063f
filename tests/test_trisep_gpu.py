"""GPU parity: triangle separation (src/cutting_planes.c:20-214).

The separated list must be identical to the reference's for the same FP64 X
-- same cuts, same values, same slot order -- and the maximum violation
equal; checked against the oracle (which replays the streaming top-K) and
against the reference build itself."""
import ctypes as C

import numpy as np
import pytest

from helpers import O, instances, root_L
from oracle import refbind
from parallel_biqbin_maxcut_b200 import _lib


def gpu_sep(lib, Xm, T, viol):
    n = Xm.shape[0]
    p = _lib.make_params(TriIneq=T, violated_TriIneq=viol)
    _lib.set_params(lib, p)
    Xc = _lib.colmajor(Xm)
    lst = (_lib.TriIneq * max(T, 1))()
    size = C.c_int()
    mx = lib.getViolated_TriangleInequalities(_lib.dptr(Xc), n, lst, C.byref(size))
    out = [(lst[q].type, lst[q].i, lst[q].j, lst[q].k, lst[q].value) for q in range(size.value)]
    return out, mx


def ipm_X(A):
    return O.ipm_mc_pk(root_L(A)).X


@pytest.mark.gpu
@pytest.mark.parametrize("nv,seed,T", [(20, 1, 200), (61, 2, 610), (101, 3, 1010), (101, 4, 50),
                                       (150, 5, 1500)])
def test_trisep_identical_to_oracle(lib, nv, seed, T):
    Xm = ipm_X(instances.gnp_pm1(nv, 0.5, seed))
    got, mx = gpu_sep(lib, Xm, T, 0.05)
    want, mx_ref = O.getViolated_TriangleInequalities(Xm, T, 0.05)
    assert mx == mx_ref
    assert got == want


@pytest.mark.gpu
def test_trisep_ties_and_edges(lib):
    # all off-diagonal entries equal: every type-1 triple has the same value,
    # so the slot order depends only on the tie rule
    n = 30
    Xm = np.full((n, n), -0.6)
    np.fill_diagonal(Xm, 1.0)
    for T in (1, 7, 100, 5000):
        got, mx = gpu_sep(lib, Xm, T, 0.05)
        want, mx_ref = O.getViolated_TriangleInequalities(Xm, T, 0.05)
        assert mx == mx_ref and got == want
    # nothing violated
    got, mx = gpu_sep(lib, np.eye(n), 100, 0.05)
    assert got == [] and mx == O.getViolated_TriangleInequalities(np.eye(n), 100, 0.05)[1]
    # smallest sizes
    for n in (3, 4):
        Xm = ipm_X(instances.gnp_unit(n, 1.0, 1))
        assert gpu_sep(lib, Xm, 10, -5.0) == tuple(O.getViolated_TriangleInequalities(Xm, 10, -5.0))
    # TriIneq = 0: no list at all
    got, _ = gpu_sep(lib, ipm_X(instances.gnp_unit(20, 0.5, 2)), 0, 0.05)
    assert got == []


@pytest.mark.gpu
def test_trisep_large_torus(lib):
    """n = 343: ~107M triangle evaluations per separation."""
    Xm = ipm_X(instances.torus3d(7, 2))
    got, mx = gpu_sep(lib, Xm, 3430, 0.05)
    want, mx_ref = O.getViolated_TriangleInequalities(Xm, 3430, 0.05)
    assert mx == mx_ref
    assert got == want


@pytest.mark.gpu
def test_trisep_matches_reference_build(lib, ref):
    for nv, seed in ((41, 7), (90, 8)):
        Xm = ipm_X(instances.gnp_unit(nv, 0.5, seed))
        n = Xm.shape[0]
        T = 10 * nv
        ref.set_param("TriIneq", T)
        ref.set_param("violated_TriIneq", 0.05)
        lst = (refbind.TriIneq * T)()
        size = C.c_int()
        Xc = _lib.colmajor(Xm)
        mx_r = ref.lib.getViolated_TriangleInequalities(_lib.dptr(Xc), n, lst, C.byref(size))
        want = [(lst[q].type, lst[q].i, lst[q].j, lst[q].k, lst[q].value) for q in range(size.value)]
        got, mx = gpu_sep(lib, Xm, T, 0.05)
        assert mx == mx_r
        assert got == want


@pytest.mark.gpu
def test_update_triangles_purge_and_dedupe(lib, lib_globals):
    """updateTriangleInequalities: purge by y < 1e-5 keeping order, separate
    on the global X, append only new cuts (src/cutting_planes.c:132-214)."""
    Xm = ipm_X(instances.gnp_unit(50, 0.5, 11))
    n = Xm.shape[0]
    T = 500
    _lib.set_params(lib, _lib.make_params(TriIneq=T, violated_TriIneq=0.05))
    lst0, _ = O.getViolated_TriangleInequalities(Xm, T, 0.05)
    # existing cuts: half of the cuts that will be separated, plus two others
    existing = [c[:4] for c in lst0[::2]] + [(1, 5, 3, 1), (2, 9, 4, 0)]
    for q, (t, i, j, k) in enumerate(existing):
        c = lib_globals.cuts[q]
        c.type, c.i, c.j, c.k = t, i, j, k
    rng = np.random.default_rng(0)
    y = np.where(rng.random(len(existing)) < 0.3, 0.0, rng.random(len(existing)) + 1e-3)
    lib_globals["X"][: n * n] = _lib.colmajor(Xm)
    prob = _lib.Problem()
    prob.n = n
    prob.NIneq = len(existing)
    added, sub = C.c_int(), C.c_int()
    yy = np.ascontiguousarray(y)
    mx = lib.updateTriangleInequalities(prob, _lib.dptr(yy), C.byref(added), C.byref(sub))
    cuts = O.Cuts(tri=np.array([c[1:] for c in existing], np.int32),
                  tri_type=np.array([c[0] for c in existing], np.int32))
    tri, tt, yk, a_ref, s_ref, mx_ref = O.updateTriangleInequalities(cuts, y, Xm, T, 0.05)
    assert (added.value, sub.value) == (a_ref, s_ref)
    assert prob.NIneq == len(tt)
    got = [(lib_globals.cuts[q].type, lib_globals.cuts[q].i, lib_globals.cuts[q].j, lib_globals.cuts[q].k)
           for q in range(prob.NIneq)]
    assert got == [(int(t), int(a), int(b), int(c)) for t, (a, b, c) in zip(tt, tri)]
    assert mx == mx_ref
