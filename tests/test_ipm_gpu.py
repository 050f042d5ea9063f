"""GPU parity: the basic SDP IPM (src/ipm_mc_pk.c:28-359) through the C ABI
against the oracle (and against the reference build when it is present).

Tolerance: phi within 1e-6 relative and X within 1e-6 absolute (X entries
lie in [-1, 1]); both paths are FP64 and take the same line-search steps, so
the observed gap is ~1e-12."""
import ctypes as C

import numpy as np
import pytest

from helpers import O, instances, root_L
from oracle import refbind
from parallel_biqbin_maxcut_b200 import _lib

RTOL_PHI = 1e-6
ATOL_X = 1e-6


def gpu_ipm(lib, L):
    n = L.shape[0]
    Lc = _lib.colmajor(L)
    Xc = np.zeros(n * n)
    phi = C.c_double()
    lib.ipm_mc_pk(_lib.dptr(Lc), n, _lib.dptr(Xc), C.byref(phi), 0)
    return _lib.from_colmajor(Xc, n), phi.value


CASES = [
    ("unit", 12, 1), ("unit", 40, 2), ("unit", 60, 3), ("pm1", 100, 4),
    ("int10", 80, 5), ("qubo", 100, 6),
]


def _adj(kind, nv, seed):
    if kind == "unit":
        return instances.gnp_unit(nv, 0.5, seed)
    if kind == "pm1":
        return instances.gnp_pm1(nv, 0.5, seed)
    if kind == "int10":
        return instances.gnp_int(nv, 0.9, 10, seed)
    return instances.qubo_to_maxcut(instances.qubo_dense(nv, 0.1, seed))


@pytest.mark.gpu
@pytest.mark.parametrize("kind,nv,seed", CASES)
def test_ipm_root_matches_oracle(lib, kind, nv, seed):
    L = root_L(_adj(kind, nv, seed))
    X, phi = gpu_ipm(lib, L)
    r = O.ipm_mc_pk(L)
    assert abs(phi - r.phi) <= RTOL_PHI * abs(r.phi), (phi, r.phi)
    assert np.max(np.abs(X - r.X)) <= ATOL_X
    assert np.allclose(np.diag(X), 1.0, atol=1e-9)
    assert np.array_equal(X, X.T)


@pytest.mark.gpu
def test_ipm_subproblems_match_oracle(lib):
    A = instances.gnp_pm1(100, 0.5, 7)
    SPL = O.build_SP_L(A)
    for xf, sol in instances.random_fixings(100, 6, 40, seed=8):
        L = O.create_subproblem(SPL, xf, sol)
        X, phi = gpu_ipm(lib, L)
        r = O.ipm_mc_pk(L)
        assert abs(phi - r.phi) <= RTOL_PHI * abs(r.phi)
        assert np.max(np.abs(X - r.X)) <= ATOL_X


@pytest.mark.gpu
def test_ipm_large_torus(lib):
    """n = 343 (7x7x7 torus, weights ~1e5): the global-memory path."""
    L = root_L(instances.torus3d(7, 1))
    X, phi = gpu_ipm(lib, L)
    r = O.ipm_mc_pk(L)
    assert abs(phi - r.phi) <= RTOL_PHI * abs(r.phi)
    assert np.max(np.abs(X - r.X)) <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("kind,nv,seed", [("pm1", 129, 21), ("unit", 160, 22), ("int10", 200, 23)])
def test_ipm_multi_cta_panel_edges(lib, kind, nv, seed):
    """n > 128 runs as 32-column panels: a last panel of one column (129),
    whole panels only (160), a ragged last panel (200)."""
    L = root_L(_adj(kind, nv, seed))
    X, phi = gpu_ipm(lib, L)
    r = O.ipm_mc_pk(L)
    assert abs(phi - r.phi) <= RTOL_PHI * abs(r.phi), (phi, r.phi)
    assert np.max(np.abs(X - r.X)) <= ATOL_X
    assert np.allclose(np.diag(X), 1.0, atol=1e-9)
    assert np.array_equal(X, X.T)


@pytest.mark.gpu
def test_ipm_torus_subproblems_match_oracle(lib):
    """Subproblems of the n = 343 torus (couplings ~1e5) after fixing up to
    40 vertices."""
    A = instances.torus3d(7, 1)
    SPL = O.build_SP_L(A)
    for xf, sol in instances.random_fixings(343, 2, 40, seed=24):
        L = O.create_subproblem(SPL, xf, sol)
        X, phi = gpu_ipm(lib, L)
        r = O.ipm_mc_pk(L)
        assert abs(phi - r.phi) <= RTOL_PHI * abs(r.phi)
        assert np.max(np.abs(X - r.X)) <= 1e-5


@pytest.mark.gpu
@pytest.mark.skipif(not refbind.available(), reason="reference build absent")
def test_ipm_matches_reference_build(lib):
    ref = refbind.RefLib()
    for nv, seed in ((30, 11), (70, 12)):
        L = root_L(instances.gnp_unit(nv, 0.5, seed))
        Xr, phir = ref.ipm(L)
        X, phi = gpu_ipm(lib, L)
        assert abs(phi - phir) <= RTOL_PHI * abs(phir)
        assert np.max(np.abs(X - Xr)) <= ATOL_X


@pytest.mark.gpu
def test_ipm_batch_mixed_sizes(lib):
    """One launch, problems of different n (the batched form)."""
    A = instances.gnp_pm1(100, 0.5, 9)
    SPL = O.build_SP_L(A)
    Ls = [O.create_subproblem(SPL, xf, sol) for xf, sol in instances.random_fixings(100, 16, 40, 10)]
    ns = np.array([L.shape[0] for L in Ls], np.int32)
    Lc = [_lib.colmajor(L) for L in Ls]
    Xc = [np.zeros(n * n) for n in ns]
    phi = np.zeros(len(Ls))
    it = np.zeros(len(Ls), np.int32)
    st = np.zeros(len(Ls), np.int32)
    pl = (C.c_void_p * len(Ls))(*[a.ctypes.data for a in Lc])
    px = (C.c_void_p * len(Ls))(*[a.ctypes.data for a in Xc])
    lib.bqb_ipm_batch(pl, px, _lib.iptr(ns), len(Ls), _lib.dptr(phi), _lib.iptr(it), _lib.iptr(st))
    assert np.all(st == 0)
    for L, x, p in zip(Ls, Xc, phi):
        r = O.ipm_mc_pk(L)
        assert abs(p - r.phi) <= RTOL_PHI * abs(r.phi)
        assert np.max(np.abs(_lib.from_colmajor(x, L.shape[0]) - r.X)) <= ATOL_X
