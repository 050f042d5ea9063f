"""GPU parity: op_B (src/operators.c:51-132) and op_Bt (:140-481) through the
C ABI against the oracle, on triangle, pentagonal and heptagonal cuts.

Both kernels keep the reference's summation order (op_B: the bracket in
lexicographic pair order; op_Bt: contributions to one entry in cut order),
so the results are expected to be bit-identical; the test allows 1e-12."""
import numpy as np
import pytest

from helpers import O, make_problem, random_cuts, set_global_cuts
from parallel_biqbin_maxcut_b200 import _lib


def _sym(rng, n):
    A = rng.standard_normal((n, n))
    return A + A.T


@pytest.mark.gpu
@pytest.mark.parametrize("n,mt,mp,mh", [(10, 5, 0, 0), (60, 600, 40, 0), (100, 1000, 180, 200),
                                        (343, 3430, 0, 0), (20, 0, 0, 30)])
def test_opB_opBt_match_oracle(lib, n, mt, mp, mh):
    rng = np.random.default_rng(n + mt)
    cuts = random_cuts(n, mt, mp, mh, rng)
    keep = set_global_cuts(lib, cuts)
    Xm = _sym(rng, n)
    Xc = _lib.colmajor(Xm)
    prob = make_problem(Xc, n, cuts)
    m = cuts.m
    y = rng.standard_normal(m)
    y_gpu = y.copy()
    lib.op_B(prob, _lib.dptr(y_gpu), _lib.dptr(Xc))
    y_ref = O.op_B(cuts, y, Xm)
    np.testing.assert_allclose(y_gpu, y_ref, rtol=0, atol=1e-12)

    t = np.abs(rng.standard_normal(m))
    Xt = Xc.copy()
    lib.op_Bt(prob, _lib.dptr(Xt), _lib.dptr(t))
    X_ref = O.op_Bt(cuts, Xm, t)
    np.testing.assert_allclose(_lib.from_colmajor(Xt, n), X_ref, rtol=0, atol=1e-12)
    del keep


@pytest.mark.gpu
def test_opB_adjoint_identity(lib):
    """<B(X), t> == <X, B^T(t)> (size-independent property)."""
    n = 120
    rng = np.random.default_rng(5)
    cuts = random_cuts(n, 800, 100, 100, rng)
    keep = set_global_cuts(lib, cuts)
    Xm = _sym(rng, n)
    Xc = _lib.colmajor(Xm)
    prob = make_problem(Xc, n, cuts)
    y = np.zeros(cuts.m)
    lib.op_B(prob, _lib.dptr(y), _lib.dptr(Xc))      # y = -B(X)
    t = rng.random(cuts.m)
    Z0 = np.zeros(n * n)
    lib.op_Bt(prob, _lib.dptr(Z0), _lib.dptr(t))     # Z0 = -B^T(t)
    lhs = float(-y @ t)
    rhs = float(np.vdot(Xc, -Z0))
    assert abs(lhs - rhs) <= 1e-9 * max(1.0, abs(lhs))
    del keep


@pytest.mark.gpu
def test_fct_eval_matches_oracle(lib):
    from helpers import instances, root_L
    A = instances.gnp_unit(50, 0.5, 3)
    L = root_L(A)
    n = L.shape[0]
    rng = np.random.default_rng(3)
    cuts = random_cuts(n, 300, 20, 10, rng)
    keep = set_global_cuts(lib, cuts)
    Lc = _lib.colmajor(L)
    prob = make_problem(Lc, n, cuts)
    gam = 0.01 * rng.random(cuts.m)
    Xc = np.zeros(n * n)
    gv = np.zeros(cuts.m)
    fv = lib.fct_eval(prob, _lib.dptr(gam), _lib.dptr(Xc), _lib.dptr(gv))
    f_ref, X_ref, g_ref = O.fct_eval(L, cuts, gam)
    assert abs(fv - f_ref) <= 1e-6 * abs(f_ref)
    assert np.max(np.abs(_lib.from_colmajor(Xc, n) - X_ref)) <= 1e-6
    assert np.max(np.abs(gv - g_ref)) <= 1e-6
    del keep
