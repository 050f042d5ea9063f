"""ctypes binding of the oracle's C restatements (oracle/_port, built by
``make -C oracle port``).  TEST INFRASTRUCTURE ONLY: tests, smoke() and the
benchmark's CPU baseline use it as the checker; the product never does."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_port", "libbqb_oracle_c.so")
PORT_FM_SO = os.path.join(HERE, "_port", "libbqb_oracle_c_fm.so")
SA_MAX_ROUNDS = 80

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_libs = {}


def available() -> bool:
    return os.path.exists(PORT_SO) and os.path.exists(PORT_FM_SO)


def _load(path: str):
    if path not in _libs:
        L = C.CDLL(path)
        L.oracle_kgon_sa.restype = C.c_int
        L.oracle_kgon_sa.argtypes = [_D, C.c_int, C.c_int, C.c_int, C.c_int, C.c_ulonglong, C.c_int, _D, _I]
        L.oracle_qap_sa_glibc.restype = C.c_double
        L.oracle_qap_sa_glibc.argtypes = [_D, C.c_int, C.c_int, C.c_int, _I]
        _libs[path] = L
    return _libs[path]


def kgon_sa(Xc: np.ndarray, n: int, k: int, types: int, chains: int, seed: int,
            max_rounds: int = SA_MAX_ROUNDS):
    """All chains of one GPU separation call, sequentially on the CPU.
    Xc: column-major n*n float64.  Returns (cost[chains], perm[chains, 7], capped)."""
    L = _load(PORT_SO)
    X = np.ascontiguousarray(Xc, dtype=np.float64)
    cost = np.zeros(chains)
    perm = np.zeros(chains * 7, np.int32)
    capped = L.oracle_kgon_sa(X.ctypes.data_as(_D), n, k, types, chains, seed, max_rounds,
                              cost.ctypes.data_as(_D), perm.ctypes.data_as(_I))
    return cost, perm.reshape(chains, 7), bool(capped)


def qap_sa_glibc(Xc: np.ndarray, n: int, k: int, typ: int, fastmath: bool = True):
    """One chain drawing from rand() (seed with srand first); with the
    reference's flags when ``fastmath``.  Returns (value, perm[k])."""
    L = _load(PORT_FM_SO if fastmath else PORT_SO)
    X = np.ascontiguousarray(Xc, dtype=np.float64)
    p = np.zeros(k, np.int32)
    v = L.oracle_qap_sa_glibc(X.ctypes.data_as(_D), n, k, typ, p.ctypes.data_as(_I))
    return v, p
