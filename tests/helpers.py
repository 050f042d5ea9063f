"""Shared helpers for the parity tests: instances, random cut lists, and
writing cut lists into a library's reference-layout globals."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from oracle import bqb_oracle as O
from parallel_biqbin_maxcut_b200 import _lib, instances

# Where the reference's sources and test fixtures lie (only tests that pin
# against them read it; they skip when it is absent).
REFERENCE_ROOT = os.environ.get("BQB_REFERENCE", "/root/reference")


def ref_path(*parts: str) -> str:
    return os.path.join(REFERENCE_ROOT, *parts)


def root_L(A: np.ndarray) -> np.ndarray:
    """PP->L of the root node (nothing fixed) for adjacency A."""
    SPL = O.build_SP_L(A)
    N = A.shape[0] - 1
    return O.create_subproblem(SPL, np.zeros(N, int), np.zeros(N, int))


def random_cuts(n: int, mt: int, mp: int, mh: int, rng) -> O.Cuts:
    tri = np.array([np.sort(rng.choice(n, 3, replace=False))[::-1] for _ in range(mt)],
                   dtype=np.int32).reshape(-1, 3)
    pent = np.array([rng.choice(n, 5, replace=False) for _ in range(mp)], dtype=np.int32).reshape(-1, 5)
    hept = np.array([rng.choice(n, 7, replace=False) for _ in range(mh)], dtype=np.int32).reshape(-1, 7)
    return O.Cuts(tri=tri, tri_type=rng.integers(1, 5, mt).astype(np.int32),
                  pent=pent, pent_type=rng.integers(1, 4, mp).astype(np.int32),
                  hept=hept, hept_type=rng.integers(1, 5, mh).astype(np.int32))


def cut_arrays(cuts: O.Cuts, mod=_lib):
    """Reference-layout arrays (Triangle/Pentagonal/Heptagonal_Inequality)."""
    mt, mp, mh = len(cuts.tri_type), len(cuts.pent_type), len(cuts.hept_type)
    T = (mod.TriIneq * max(mt, 1))()
    P = (mod.PentIneq * max(mp, 1))()
    H = (mod.HeptIneq * max(mh, 1))()
    for c in range(mt):
        T[c].i, T[c].j, T[c].k = (int(v) for v in cuts.tri[c])
        T[c].type = int(cuts.tri_type[c])
    for c in range(mp):
        P[c].type = int(cuts.pent_type[c])
        for a in range(5):
            P[c].permutation[a] = int(cuts.pent[c, a])
    for c in range(mh):
        H[c].type = int(cuts.hept_type[c])
        for a in range(7):
            H[c].permutation[a] = int(cuts.hept[c, a])
    return T, P, H


def set_global_cuts(cdll, cuts: O.Cuts, mod=_lib):
    """Point the library's Cuts/Pent_Cuts/Hepta_Cuts globals at fresh arrays
    holding ``cuts``; returns the arrays (keep them alive)."""
    T, P, H = cut_arrays(cuts, mod)
    C.c_void_p.in_dll(cdll, "Cuts").value = C.addressof(T)
    C.c_void_p.in_dll(cdll, "Pent_Cuts").value = C.addressof(P)
    C.c_void_p.in_dll(cdll, "Hepta_Cuts").value = C.addressof(H)
    return T, P, H


def make_problem(L_colmajor: np.ndarray, n: int, cuts: O.Cuts, mod=_lib):
    p = mod.Problem()
    p.L = L_colmajor.ctypes.data_as(C.POINTER(C.c_double))
    p.n = n
    p.NIneq = len(cuts.tri_type)
    p.NPentIneq = len(cuts.pent_type)
    p.NHeptaIneq = len(cuts.hept_type)
    p.bundle = 0
    return p


__all__ = ["REFERENCE_ROOT", "ref_path", "root_L", "random_cuts", "cut_arrays", "set_global_cuts", "make_problem", "instances", "O"]
