"""The allocation-free IPM entry point (bqb_ipm_noalloc).

Callers that may not allocate device memory while they run (for instance a
solver embedded in an application whose memory manager owns the GPU) pass
their own device inputs and outputs; the IPM's scratch comes from a fixed
array in the library's static device memory.  This test calls that entry
point through the C ABI several times in a row, on problems of different
sizes (a small one after the largest, and the same one twice), and compares
each result with the regular entry point (ipm_mc_pk), within the tolerance of
the other IPM tests, and a repeated call with the first bit for bit; it also checks that an oversized problem is
rejected with a message.  It runs last so that a failure here leaves every
other test already run, and it passes both alone and after the others."""
import ctypes as C

import numpy as np
import pytest

from helpers import instances, root_L
from parallel_biqbin_maxcut_b200 import _lib

RTOL_PHI = 1e-6
ATOL_X = 1e-6


def _regular(lib, L):
    n = L.shape[0]
    Xc = np.zeros(n * n)
    phi = C.c_double()
    lib.ipm_mc_pk(_lib.dptr(_lib.colmajor(L)), n, _lib.dptr(Xc), C.byref(phi), 0)
    return _lib.from_colmajor(Xc, n), phi.value


def _noalloc(lib, L):
    import torch
    f = lib.bqb_ipm_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    n = L.shape[0]
    dL = torch.from_numpy(_lib.colmajor(L)).to("cuda")
    dX = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    dout = torch.zeros(4, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = f(dL.data_ptr(), dX.data_ptr(), n, dout.data_ptr(), None)
    assert rc == 0, lib.bqb_last_error()
    torch.cuda.synchronize()
    return _lib.from_colmajor(dX.cpu().numpy(), n), dout.cpu().numpy()


@pytest.mark.gpu
def test_noalloc_matches_regular_entry_point_twice(lib):
    problems = [root_L(instances.gnp_unit(61, 0.5, 21)),                           # n = 61
                root_L(instances.qubo_to_maxcut(instances.qubo_dense(100, 0.1, 22))),  # n = 101
                root_L(instances.gnp_pm1(128, 0.5, 23))]                             # n = 128 (limit)
    # increasing sizes, then a small problem after the largest left its
    # contents in the shared scratch, then the same problem again
    first = {}
    for q in (0, 1, 2, 0, 0):
        L = problems[q]
        X, out = _noalloc(lib, L)
        X_ref, phi_ref = _regular(lib, L)
        assert int(out[2]) == 0
        assert abs(out[0] - phi_ref) <= RTOL_PHI * abs(phi_ref), (out[0], phi_ref)
        assert np.max(np.abs(X - X_ref)) <= ATOL_X
        if q in first:   # a repeated call gives bit-identical results
            assert np.array_equal(X, first[q][0]) and np.array_equal(out, first[q][1])
        else:
            first[q] = (X, out)


@pytest.mark.gpu
def test_noalloc_rejects_sizes_beyond_the_limit(lib):
    f = lib.bqb_ipm_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    dummy = C.c_double()
    assert f(C.addressof(dummy), C.addressof(dummy), 129, C.addressof(dummy), None) == 1
    assert b"outside 1..128" in lib.bqb_last_error()
    assert f(C.addressof(dummy), C.addressof(dummy), 0, C.addressof(dummy), None) == 1
