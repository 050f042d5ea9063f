"""FP64 certificates of the SDP bounds (csrc/certificate.cu).

The certificate is an upper bound on max <L, X> over the elliptope that holds
for any dual vector y: the sum of y plus n times a rigorous lower bound on
-lambda_min(Diag(y) - L).  Checked here: on the IPM's own y (both IPM forms,
n <= 128 in registers and n = 343 multi-CTA) the certificate exceeds the
IPM's bound by less than 1e-9 relative, needs no shift, and its eigenvalue
bound lies below numpy's lambda_min; with y lowered until Diag(y) - L is
indefinite it still bounds the oracle's primal value <L, X>; and with the
engines' certification on, every node of a B&B is certified within the
goal's 1e-6 relative (in fact 1e-9).  The certified bounds equal the
oracle's restatement (oracle/bqb_oracle.py sdp_certificate) on the same y."""
import ctypes as C

import numpy as np
import pytest

from helpers import O, instances, root_L
from parallel_biqbin_maxcut_b200 import _lib

REL = 1e-9   # certified bound over the IPM's bound, relative (the goal's bar is 1e-6)


def _dual(lib, L):
    n = L.shape[0]
    y = np.zeros(n)
    out = np.zeros(4)
    assert lib.bqb_ipm_dual(_lib.dptr(_lib.colmajor(L)), n, None, _lib.dptr(y), _lib.dptr(out)) == 0
    return y, out


def _cert(lib, L, y):
    out = np.zeros(4)
    assert lib.bqb_sdp_certificate(_lib.dptr(_lib.colmajor(L)), _lib.dptr(y), L.shape[0], _lib.dptr(out)) == 0
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("kind,nv,seed", [("pm1", 40, 1), ("pm1", 100, 2), ("unit", 129, 3), ("torus", 343, 1)])
def test_certificate_of_the_ipm_dual(lib, kind, nv, seed):
    if kind == "torus":
        A = instances.torus3d(7, seed)
    elif kind == "unit":
        A = instances.gnp_unit(nv, 0.5, seed)
    else:
        A = instances.gnp_pm1(nv, 0.5, seed)
    L = root_L(A)
    n = L.shape[0]
    y, out = _dual(lib, L)
    phi = out[0]
    assert int(out[2]) == 0
    assert abs(y.sum() - phi) <= 1e-12 * abs(phi)
    c = _cert(lib, L, y)
    assert int(c[3]) == 0 and c[2] <= 1e-10 * abs(phi)   # Diag(y) - L factors (as it is, in practice)
    assert c[0] >= phi and (c[0] - phi) <= REL * abs(phi), (c[0], phi)
    lam = np.linalg.eigvalsh(np.diag(y) - L).min()
    assert c[1] <= lam + 1e-12 * np.abs(L).max() * n
    # the oracle's certificate of the same y (LAPACK's factorisation)
    bo, lo, to = O.sdp_certificate(L, y)
    assert to == 0.0 and abs(c[0] - bo) <= 1e-12 * abs(bo), (c[0], bo)
    if n <= 129:   # the oracle's IPM: its phi agrees and its primal value is below the certificate
        r = O.ipm_mc_pk(L)
        assert abs(phi - r.phi) <= 1e-6 * abs(r.phi)
        assert c[0] >= float(np.sum(L * r.X)) - 1e-9 * abs(r.phi)


@pytest.mark.gpu
def test_certificate_of_an_infeasible_dual(lib):
    """y lowered by delta makes Diag(y) - L indefinite: the certificate needs
    a shift and adds n times the (bounded) negative eigenvalue, so it stays
    above the oracle's primal value and within a little of e'y + n * delta."""
    L = root_L(instances.gnp_pm1(60, 0.5, 7))
    n = L.shape[0]
    y, out = _dual(lib, L)
    lam0 = np.linalg.eigvalsh(np.diag(y) - L).min()
    delta = 0.5
    yl = y - (lam0 + delta)
    c = _cert(lib, L, yl)
    assert int(c[3]) == 0 and c[2] > 0.0
    lam = np.linalg.eigvalsh(np.diag(yl) - L).min()
    scale = 1e-12 * n * np.abs(np.diag(yl) - L).max()   # numpy's own eigenvalue error
    assert lam < 0 and c[1] <= lam + scale
    r = O.ipm_mc_pk(L)
    assert c[0] >= float(np.sum(L * r.X))
    exact = yl.sum() + n * -lam
    assert exact - n * scale <= c[0] <= exact + 1e-6 * abs(exact)
    bo, _, to = O.sdp_certificate(L, yl)
    assert to > 0.0 and abs(c[0] - bo) <= 1e-9 * abs(bo), (c[0], bo)


@pytest.mark.gpu
def test_engine_node_bounds_are_certified(lib):
    """With certification on, a B&B on 4 engines certifies every node it
    bounds: no failure, the certified bound exceeds the node's bound by at
    most 1e-9 relative, and the rerun IPM at the final multipliers returns
    the bundle's value."""
    A = instances.gnp_pm1(60, 0.5, 5)
    st = np.zeros(6)
    lib.bqb_certify_stats(_lib.dptr(st), 1)
    lib.bqb_certify_enable(1)
    try:
        r = _lib.solve(A, threads=4)
    finally:
        lib.bqb_certify_enable(0)
    lib.bqb_certify_stats(_lib.dptr(st), 1)
    nodes, max_rel, mean_rel, failed, shift, mismatch = st
    assert nodes >= r["nodes"] >= 1
    assert failed == 0 and shift <= 1e-10 * abs(r["root_bound"])
    assert 0.0 <= mean_rel <= max_rel <= REL, st
    assert mismatch <= 1e-12, st
