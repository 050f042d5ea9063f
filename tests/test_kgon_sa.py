"""k-gonal separation by annealing chains.

CPU: the oracle's C restatement of one chain (oracle/kgon_sa_chain.c),
built with the reference's flags and drawing from rand(), returns the
reference build's qap_simulated_annealing value, permutation and rand()
state (src/qap_simulated_annealing.c) -- this pins the restatement.

GPU: the chains of bqb_kgon_sa (one warp per chain evaluating its moves
speculatively, SplitMix64 streams) equal the oracle's one-move-at-a-time
chains with the same streams bit for bit: the same best values,
permutations and round-limit flag, with X in shared memory (n <= 127) and
in global memory (n = 200, 343)."""
import ctypes as C

import numpy as np
import pytest

from helpers import O, instances, root_L
from oracle import portbind, refbind
from parallel_biqbin_maxcut_b200 import _lib

libc = C.CDLL("libc.so.6")
libc.rand.restype = C.c_int

port = pytest.mark.skipif(not portbind.available(), reason="oracle port not built (make -C oracle port)")


def _X(nv, seed):
    return _lib.colmajor(O.ipm_mc_pk(root_L(instances.gnp_unit(nv, 0.5, seed))).X)


@port
@pytest.mark.skipif(not refbind.available(), reason="reference build absent")
@pytest.mark.parametrize("k,nv,seed", [(5, 30, 1), (5, 60, 2), (7, 30, 3), (7, 60, 4)])
def test_oracle_chain_pinned_to_reference(k, nv, seed):
    ref = refbind.RefLib()
    L = ref.lib
    L.qap_simulated_annealing.restype = C.c_double
    L.qap_simulated_annealing.argtypes = [C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_double), C.c_int,
                                          C.POINTER(C.c_int)]
    X = _X(nv, seed)
    for typ in range(1, (4 if k == 7 else 3) + 1):
        e = np.array([-1 if a < typ - 1 else 1 for a in range(k)])
        H = np.ascontiguousarray(np.outer(e, e).reshape(-1), dtype=np.int32)
        for s in range(3):
            libc.srand(seed * 1000 + typ * 10 + s)
            p = np.zeros(k, np.int32)
            v = L.qap_simulated_annealing(_lib.iptr(H), k, _lib.dptr(X), nv, _lib.iptr(p))
            want = (v, tuple(p), libc.rand())
            libc.srand(seed * 1000 + typ * 10 + s)
            w, q = portbind.qap_sa_glibc(X, nv, k, typ)
            assert (w, tuple(q), libc.rand()) == want


@port
def test_oracle_chain_values_are_inequality_values():
    """Each chain's best value is <(P X P^T)(1:k, 1:k), H> of its permutation."""
    nv = 40
    X = _X(nv, 7)
    Xm = X.reshape(nv, nv, order="F")
    for k, types in ((5, 3), (7, 4)):
        cost, perm, _ = portbind.kgon_sa(X, nv, k, types, 24, seed=99)
        for c in range(24):
            typ = c % types + 1
            e = np.array([-1 if a < typ - 1 else 1 for a in range(k)])
            p = perm[c, :k]
            assert len(set(p.tolist())) == k
            val = float(np.sum(np.outer(e, e) * Xm[np.ix_(p, p)]))
            assert abs(val - cost[c]) < 1e-8


@pytest.mark.gpu
@port
@pytest.mark.parametrize("k,types,nv,seed", [(5, 3, 30, 1), (7, 4, 30, 2), (5, 3, 100, 3), (7, 4, 100, 4),
                                             (5, 3, 64, 5), (7, 4, 127, 6), (5, 3, 200, 7), (7, 4, 343, 8)])
def test_gpu_chains_equal_oracle(lib, k, types, nv, seed):
    X = _X(nv, seed)
    chains = 60 * types if nv <= 64 else 50 * types
    cost = np.zeros(chains)
    perm = np.zeros(chains * 7, np.int32)
    sd = 0x1234_5678_0000_0000 + seed
    rc = lib.bqb_kgon_sa(_lib.dptr(X), nv, k, types, chains, sd, _lib.dptr(cost), _lib.iptr(perm))
    oc, op, capped = portbind.kgon_sa(X, nv, k, types, chains, sd)
    assert rc == int(capped)
    np.testing.assert_array_equal(cost, oc)
    np.testing.assert_array_equal(perm.reshape(chains, 7), op)


@pytest.mark.gpu
def test_gpu_chains_argument_checks(lib):
    X = np.eye(4).ravel()
    cost = np.zeros(4)
    perm = np.zeros(28, np.int32)
    assert lib.bqb_kgon_sa(_lib.dptr(X), 4, 5, 3, 4, 1, _lib.dptr(cost), _lib.iptr(perm)) == 2
    assert lib.bqb_kgon_sa(_lib.dptr(X), 4, 6, 3, 4, 1, _lib.dptr(cost), _lib.iptr(perm)) == 2
