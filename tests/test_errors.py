"""Error paths, without any GPU fault.

The reference ends the process (MPI_Abort(..., 10)) on a failed Cholesky
factorisation or QP solve.  The library reports the same failures through
an abort hook (default: exit(10)): kernels never trap, they write a status
word that the host reads.  These tests make the failures happen with
inputs whose arithmetic fails (a non-positive-definite X for the
heuristic's factorisation, an indefinite QP matrix), check that
the hook sees code 10 with the reference's message, and that the device
context is still usable afterwards.  Argument errors of the C entry points
return codes without touching the GPU (CPU tests)."""
import ctypes as C

import numpy as np
import pytest

from helpers import O, instances
from parallel_biqbin_maxcut_b200 import _lib

HOOK = C.CFUNCTYPE(None, C.c_int)


@pytest.fixture
def hook(lib):
    codes = []
    cb = HOOK(lambda code: codes.append(code))
    lib.bqb_set_abort_hook.argtypes = [HOOK]
    lib.bqb_set_abort_hook(cb)
    try:
        yield codes
    finally:
        lib.bqb_set_abort_hook(C.cast(None, HOOK))


def test_argument_errors_return_codes():
    lib = _lib.load()
    assert lib.bqb_warm_train(None, None, 0, 1, 1, 1e-3, 0, None, None) == -1
    assert lib.bqb_warm_grad(None, None, None, 0, None, None) == -1
    assert lib.bqb_warm_predict(None, None, 0, None) == -1
    assert lib.bqb_fused_submit(None, 0, 1) == -4
    assert lib.bqb_fused_collect(123456789, None, None) == 1
    assert b"unknown or already collected ticket" in lib.bqb_last_error()


@pytest.mark.gpu
def test_heuristic_factorisation_failure_reaches_abort_hook(lib, lib_globals, hook):
    """runHeuristic_unpacked factors the global X (src/heuristic.c:68-74);
    X = -I is not positive definite."""
    A = instances.gnp_unit(20, 0.5, 3)
    SPL = O.build_SP_L(A)
    L = O.create_subproblem(SPL, np.zeros(19, int), np.zeros(19, int))
    n = L.shape[0]
    lib_globals["X"][: n * n] = _lib.colmajor(-np.eye(n))
    z = np.zeros(19, np.int32)
    x = np.zeros(19, np.int32)
    lib.runHeuristic_unpacked(_lib.dptr(_lib.colmajor(SPL)), SPL.shape[0], _lib.dptr(_lib.colmajor(L)), n,
                              _lib.iptr(z), _lib.iptr(z.copy()), _lib.iptr(x))
    assert hook and hook[0] == 10
    assert b"Cholesky" in lib.bqb_last_error()
    # the context is usable: a regular IPM call afterwards is exact
    phi = C.c_double()
    lib.ipm_mc_pk(_lib.dptr(_lib.colmajor(L)), n, _lib.dptr(np.zeros(n * n)), C.byref(phi), 0)
    r = O.ipm_mc_pk(L)
    assert abs(phi.value - r.phi) <= 1e-6 * abs(r.phi)


@pytest.mark.gpu
def test_qp_failure_reaches_abort_hook(lib, hook):
    k = 5
    Q = -100.0 * np.eye(k)   # indefinite: the first KKT pivot is negative
    lam = np.zeros(k)
    lib.solve_lambda(k, _lib.dptr(_lib.colmajor(Q)), _lib.dptr(np.ones(k)), _lib.dptr(lam))
    assert hook == [10]
    assert b"solve_lambda" in lib.bqb_last_error()
