"""GPU parity: the bundle QP pieces (src/bundle.c:292-653).

solve_lambda: the same primal-dual IPM; the GPU solves its KKT system by a
Schur complement where the reference uses dsysv, so lambda agrees to
rounding (tolerance 1e-8 absolute; lambda lies in the unit simplex).
lambda_eta: same alternation and stopping rule (tolerance 1e-7)."""
import ctypes as C

import numpy as np
import pytest

from helpers import O
from parallel_biqbin_maxcut_b200 import _lib


def _qp_case(k, m, seed):
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((m, k))
    t = 0.05 + rng.random()
    Q = t * (G.T @ G)
    c = rng.standard_normal(k) * 3
    return G, t, Q, c


@pytest.mark.gpu
@pytest.mark.parametrize("k,seed", [(1, 0), (2, 1), (5, 2), (20, 3), (40, 4), (100, 5)])
def test_solve_lambda(lib, k, seed):
    G, t, Q, c = _qp_case(k, max(2 * k, 10), seed)
    lam = np.zeros(k)
    Qc = _lib.colmajor(Q)
    cc = c.copy()
    lib.solve_lambda(k, _lib.dptr(Qc), _lib.dptr(cc), _lib.dptr(lam))
    want = O.solve_lambda(Q, c)
    np.testing.assert_allclose(lam, want, rtol=0, atol=1e-8)
    assert abs(lam.sum() - 1.0) < 1e-6 and np.all(lam > 0)


@pytest.mark.gpu
@pytest.mark.parametrize("k,m,seed", [(1, 30, 0), (4, 200, 1), (12, 800, 2), (30, 3000, 3)])
def test_lambda_eta(lib, k, m, seed):
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((m, k)) * 0.3
    zeta = -rng.random(k) * 10
    gam = np.where(rng.random(m) < 0.5, 0.0, rng.random(m))
    t = 0.2
    prob = _lib.Problem()
    prob.NIneq = m
    prob.bundle = k
    Gc = np.ascontiguousarray(G.T).reshape(-1)   # column-major m x k
    dg, lam, eta = np.zeros(m), np.zeros(k), np.zeros(m)
    tt = C.c_double(t)
    z = zeta.copy()
    gg = gam.copy()
    lib.lambda_eta(prob, _lib.dptr(z), _lib.dptr(Gc), _lib.dptr(gg), _lib.dptr(dg), _lib.dptr(lam),
                   _lib.dptr(eta), C.byref(tt))
    dg_r, lam_r, eta_r, t_r = O.lambda_eta(zeta, G, gam, t)
    np.testing.assert_allclose(lam, lam_r, rtol=0, atol=1e-7)
    np.testing.assert_allclose(dg, dg_r, rtol=0, atol=1e-7 * max(1.0, np.abs(dg_r).max()))
    np.testing.assert_allclose(eta, eta_r, rtol=0, atol=1e-7 * max(1.0, np.abs(eta_r).max()))
    assert tt.value == t_r


@pytest.mark.gpu
def test_solve_lambda_matches_reference_build(lib, ref):
    for k, seed in ((3, 10), (15, 11), (35, 12)):
        G, t, Q, c = _qp_case(k, 3 * k, seed)
        Qc = _lib.colmajor(Q)
        lam_r = np.zeros(k)
        ref.lib.solve_lambda(k, _lib.dptr(Qc.copy()), _lib.dptr(c.copy()), _lib.dptr(lam_r))
        lam = np.zeros(k)
        lib.solve_lambda(k, _lib.dptr(Qc.copy()), _lib.dptr(c.copy()), _lib.dptr(lam))
        np.testing.assert_allclose(lam, lam_r, rtol=0, atol=1e-8)
