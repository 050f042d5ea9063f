"""The oracle's restatement of the FP64 certificate (no GPU): on the oracle
IPM's own dual vector the certified bound lies just above e'y and above the
primal value <L, X>; on a dual vector lowered until Diag(y) - L is
indefinite it needs a shift, stays a valid bound and is tight to
e'y + n (-lambda_min)."""
import numpy as np

from helpers import O, instances, root_L


def test_oracle_certificate_of_the_ipm_dual():
    L = root_L(instances.gnp_pm1(40, 0.5, 3))
    r = O.ipm_mc_pk(L)
    assert abs(r.y.sum() - r.phi) <= 1e-12 * abs(r.phi)
    b, lam, t = O.sdp_certificate(L, r.y)
    assert t == 0.0 and b >= r.phi and b - r.phi <= 1e-9 * abs(r.phi)
    assert lam <= np.linalg.eigvalsh(np.diag(r.y) - L).min() + 1e-12
    assert b >= float(np.sum(L * r.X))


def test_oracle_certificate_of_an_infeasible_dual():
    L = root_L(instances.gnp_unit(30, 0.5, 4))
    n = L.shape[0]
    r = O.ipm_mc_pk(L)
    lam0 = np.linalg.eigvalsh(np.diag(r.y) - L).min()
    yl = r.y - (lam0 + 0.25)
    b, lam, t = O.sdp_certificate(L, yl)
    true_min = np.linalg.eigvalsh(np.diag(yl) - L).min()
    assert t > 0.0 and lam <= true_min + 1e-12
    exact = yl.sum() + n * -true_min
    assert exact - 1e-9 <= b <= exact + 1e-6 * abs(exact)
    assert b >= float(np.sum(L * r.X))
