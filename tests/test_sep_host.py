"""Host-side separation (CPU): the pentagonal / heptagonal simulated-annealing
separation restated in host_sep.cpp against the reference build, from the
same rand() state: identical cuts, values and rand() state afterwards.
These routines run on the host in both implementations; no GPU call is made.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import O, instances, root_L
from oracle import refbind
from parallel_biqbin_maxcut_b200 import _lib

libc = C.CDLL("libc.so.6")
libc.rand.restype = C.c_int

pytestmark = pytest.mark.skipif(not (refbind.available() and __import__("os").path.exists(_lib.LIB_PATH)),
                                reason="reference build or library absent")


@pytest.fixture(scope="module")
def both():
    ref = refbind.RefLib()
    mine = C.CDLL(_lib.LIB_PATH)
    for L_ in (ref.lib, mine):
        L_.qap_simulated_annealing.restype = C.c_double
        L_.qap_simulated_annealing.argtypes = [C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_double), C.c_int,
                                              C.POINTER(C.c_int)]
    return ref, mine


def _X(nv, seed):
    return O.ipm_mc_pk(root_L(instances.gnp_unit(nv, 0.5, seed))).X


@pytest.mark.parametrize("k,nv,seed", [(5, 30, 1), (5, 60, 2), (7, 30, 3), (7, 60, 4)])
def test_qap_simulated_annealing_identical(both, k, nv, seed):
    ref, mine = both
    Xc = _lib.colmajor(_X(nv, seed))
    n = nv
    for typ in range(1, (4 if k == 7 else 3) + 1):
        e = np.array([-1 if a < typ - 1 else 1 for a in range(k)])
        Hm = np.ascontiguousarray(np.outer(e, e).reshape(-1), dtype=np.int32)
        out = []
        for L_ in (ref.lib, mine):
            libc.srand(seed * 100 + typ)
            p = np.zeros(k, np.int32)
            v = L_.qap_simulated_annealing(_lib.iptr(Hm), k, _lib.dptr(Xc), n, _lib.iptr(p))
            out.append((v, tuple(p), libc.rand()))
        assert out[0] == out[1]
