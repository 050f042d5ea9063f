"""Seeded synthetic Max-Cut / QUBO instances for the benchmark configurations.

None of these is a public benchmark item: they are generated from numpy's
``default_rng(seed)`` (PCG64) with the shapes, sizes and weight distributions
of the configurations the bounding path is measured on.

* C1  ``gnp_unit(60, 0.5, seed)``       G(n, p), every edge weight 1
* C2  ``gnp_pm1(100, 0.5, seed)``       G(n, p), weights uniform in {-1, +1};
      ``random_fixings`` draws the 512 subproblems (k in [0, 40] fixed)
* C3  ``qubo_dense(100, 0.1, seed)``    upper-triangular integer Q; converted
      with ``qubo_to_maxcut`` exactly as the reference's ``_qubo2maxcut``
      (biqbin_base.py:230-258), which requires (Q + Q')/2 integral, so the
      off-diagonal entries are drawn from the even integers in [-100, 100]
* C4  ``torus3d(7, seed)``              7x7x7 periodic grid, J ~ N(0,1)*1e5,
      rounded to integers
* C5  ``gnp_int(150, 0.9, 10, seed)``   G(n, p), weights uniform integers in
      [-10, 10], zero weights dropped

Adjacency matrices are dense symmetric float64 arrays with zero diagonal,
vertex order as written; the solver fixes the LAST vertex to 0
(src/process_input.c:276-278).
"""
from __future__ import annotations

import numpy as np


def _sym(upper: np.ndarray) -> np.ndarray:
    a = np.triu(upper, 1)
    return a + a.T


def gnp_unit(n: int = 60, p: float = 0.5, seed: int = 1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return _sym((rng.random((n, n)) < p).astype(np.float64))


def gnp_pm1(n: int = 100, p: float = 0.5, seed: int = 1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    keep = rng.random((n, n)) < p
    w = rng.choice(np.array([-1.0, 1.0]), size=(n, n))
    return _sym(np.where(keep, w, 0.0))


def gnp_int(n: int = 150, p: float = 0.9, wmax: int = 10, seed: int = 1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    keep = rng.random((n, n)) < p
    w = rng.integers(-wmax, wmax + 1, size=(n, n)).astype(np.float64)
    return _sym(np.where(keep, w, 0.0))


def torus3d(L: int = 7, seed: int = 1, scale: float = 1e5) -> np.ndarray:
    rng = np.random.default_rng(seed)
    n = L ** 3
    A = np.zeros((n, n))

    def idx(x, y, z):
        return (x % L) * L * L + (y % L) * L + (z % L)

    for x in range(L):
        for y in range(L):
            for z in range(L):
                i = idx(x, y, z)
                for j in (idx(x + 1, y, z), idx(x, y + 1, z), idx(x, y, z + 1)):
                    w = float(np.rint(rng.standard_normal() * scale))
                    A[i, j] = A[j, i] = w
    return A


def qubo_dense(n: int = 100, density: float = 0.1, seed: int = 1) -> np.ndarray:
    """Upper-triangular integer Q: diagonal uniform in [-100, 100], off-diagonal
    uniform over the even integers in [-100, 100]; each entry kept with
    probability ``density``."""
    rng = np.random.default_rng(seed)
    keep = rng.random((n, n)) < density
    off = 2 * rng.integers(-50, 51, size=(n, n))
    dia = rng.integers(-100, 101, size=n)
    Q = np.triu(np.where(keep, off, 0), 1).astype(np.float64)
    Q[np.diag_indices(n)] = np.where(np.diag(keep), dia, 0)
    return Q


def qubo_to_maxcut(Q: np.ndarray) -> np.ndarray:
    """Adjacency of the (n+1)-vertex Max-Cut equivalent of min x'Qx, as
    biqbin_base.py:230-258 builds it (raises if (Q+Q')/2 is not integral)."""
    qs = 0.5 * (Q.T + Q)
    if not np.all(qs == np.round(qs)):
        raise ValueError("All QUBO values need to be integers!")
    qe = -qs.sum(axis=1)
    qs = qs.copy()
    np.fill_diagonal(qs, 0.0)
    n = Q.shape[0]
    A = np.zeros((n + 1, n + 1))
    A[:n, :n] = qs
    A[:n, n] = qe
    A[n, :n] = qe
    return A


def root_matrix(A: np.ndarray) -> np.ndarray:
    """The root node's matrix PP->L of an adjacency matrix A (nv x nv): the
    Laplacian over the first nv - 1 vertices bordered by its row sums, the
    last vertex fixed to 0, scaled by 1/4 (src/process_input.c:289-333,
    src/evaluate.c:38-115 with nothing fixed).  nv x nv, row-major."""
    nv = A.shape[0]
    lap = np.diag(A.sum(axis=1)) - A
    L = np.zeros((nv, nv))
    L[:nv - 1, :nv - 1] = lap[:nv - 1, :nv - 1]
    rs = L[:nv - 1, :nv - 1].sum(axis=1)
    L[:nv - 1, nv - 1] = rs
    L[nv - 1, :nv - 1] = rs
    L[nv - 1, nv - 1] = rs.sum()
    return 0.25 * L


def random_fixings(nv: int, count: int, kmax: int, seed: int):
    """``count`` (xfixed, sol) pairs over the nv-1 branchable vertices: k
    uniform in [0, kmax] vertices fixed, values uniform in {0, 1}."""
    rng = np.random.default_rng(seed)
    N = nv - 1
    out = []
    for _ in range(count):
        k = int(rng.integers(0, kmax + 1))
        xf = np.zeros(N, np.int32)
        sol = np.zeros(N, np.int32)
        idx = rng.choice(N, size=k, replace=False)
        xf[idx] = 1
        sol[idx] = rng.integers(0, 2, size=k)
        out.append((xf, sol))
    return out


def write_rudy(path: str, A: np.ndarray) -> None:
    """Rudy edge list: 'n m' then 'i j w' (1-based), the format
    src/process_input.c:201-253 reads."""
    n = A.shape[0]
    iu, ju = np.nonzero(np.triu(A, 1))
    with open(path, "w") as fh:
        fh.write(f"{n} {len(iu)}\n")
        for i, j in zip(iu, ju):
            fh.write(f"{i + 1} {j + 1} {int(A[i, j])}\n")


def write_params(path: str, values: dict) -> None:
    with open(path, "w") as fh:
        for k, v in values.items():
            fh.write(f"{k} = {v}\n")
