"""CPU restatement of BiqBin's per-node bounding path (numpy) -- the oracle.

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import this module, and only as the
checker: the GPU product never routes through it.

Every function restates one reference routine and cites it as
``src/<file>.c:<lines>`` (paths relative to the BiqBin repository).  The
arithmetic follows the reference's order where that order decides a discrete
outcome (comparisons, tie-breaks, streaming top-K replacement); dense linear
algebra uses LAPACK through numpy/scipy, as the reference uses OpenBLAS.

Parity pin: ``tests/test_oracle_golden.py`` checks this module against
golden vectors in ``tests/golden/`` that ``tests/golden/make_golden.py``
produced by calling the reference's own C code (built unmodified into
``oracle/_ref/libbqb_ref.so`` by ``oracle/Makefile``), and the reference build
itself reproduces the optimal values and solution lines of the reference's
``tests/rudy/*-expected_output`` fixtures.

Matrices are square numpy arrays.  The reference stores them column-major
with ld = n; all matrices on this path are symmetric, so ``X[i, j]`` here is
``X[i + j*n]`` there.
"""
from __future__ import annotations

import ctypes
import heapq
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg as sla

BIG_NUMBER = 1e9  # src/biqbin.h:35


# --------------------------------------------------------------------------
# glibc rand(): the reference draws every random number from it
# (src/heuristic.c:39,103,143; src/qap_simulated_annealing.c:68,102,103,139)
# --------------------------------------------------------------------------
_libc = ctypes.CDLL("libc.so.6")
_libc.rand.restype = ctypes.c_int
_libc.srand.argtypes = [ctypes.c_uint]
RAND_MAX = 2147483647


def srand(seed: int) -> None:
    _libc.srand(seed)


def rand() -> int:
    return _libc.rand()


# --------------------------------------------------------------------------
# Cut lists
# --------------------------------------------------------------------------
# Sign vectors e of each cut kind/type.  A cut is B_c(X) <= 1 with
#   B_c(X) = -scale * sum_{a<b} e_a e_b X[p_a, p_b]
# Triangle types 1-4 (src/operators.c:64-77, src/cutting_planes.c:24-36),
# pentagonal types 1-3 (H1..H3 of src/cutting_planes.c:239-244,
# src/operators.c:90-100) and heptagonal types 1-4 (src/cutting_planes.c:
# 431-438, src/operators.c:116-129).
TRI_SIGNS = {1: (1, 1, 1), 2: (1, 1, -1), 3: (1, -1, 1), 4: (-1, 1, 1)}
PENT_SIGNS = {1: (1, 1, 1, 1, 1), 2: (-1, 1, 1, 1, 1), 3: (-1, -1, 1, 1, 1)}
HEPT_SIGNS = {1: (1,) * 7, 2: (-1,) + (1,) * 6, 3: (-1, -1) + (1,) * 5,
              4: (-1, -1, -1) + (1,) * 4}
SCALE = {3: 1.0, 5: 0.5, 7: 1.0 / 3.0}


@dataclass
class Cuts:
    """The reference's three global cut arrays (src/global_var.h:37-47).

    ``tri``: (m_t, 3) int rows (i, j, k); ``tri_type``: (m_t,) in 1..4.
    ``pent``: (m_p, 5) permutations; ``pent_type`` in 1..3.
    ``hept``: (m_h, 7) permutations; ``hept_type`` in 1..4.
    Dual vectors are laid out [tri | pent | hept] (src/bounding.c:268-275).
    """
    tri: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))
    tri_type: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    pent: np.ndarray = field(default_factory=lambda: np.zeros((0, 5), np.int32))
    pent_type: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    hept: np.ndarray = field(default_factory=lambda: np.zeros((0, 7), np.int32))
    hept_type: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))

    @property
    def m(self) -> int:
        return len(self.tri_type) + len(self.pent_type) + len(self.hept_type)

    def groups(self):
        yield 3, self.tri, self.tri_type, TRI_SIGNS
        yield 5, self.pent, self.pent_type, PENT_SIGNS
        yield 7, self.hept, self.hept_type, HEPT_SIGNS


def _pair_terms(k: int, signs_of_type, idx: np.ndarray, types: np.ndarray):
    """Yield (a, b, coef) per lexicographic pair a<b: coef[c] = -e_a e_b."""
    e = np.array([signs_of_type[int(t)] for t in types], dtype=np.float64).reshape(-1, k)
    for a in range(k):
        for b in range(a + 1, k):
            yield idx[:, a], idx[:, b], -(e[:, a] * e[:, b])


def op_B(cuts: Cuts, y: np.ndarray, X: np.ndarray) -> np.ndarray:
    """y -= B(X) (src/operators.c:51-132).

    The bracket of each cut is summed over pairs in lexicographic order of
    the stored index tuple, then scaled by 1, 1/2 or 1/3, as written there.
    """
    y = np.array(y, dtype=np.float64, copy=True)
    off = 0
    for k, idx, types, signs in cuts.groups():
        mk = len(types)
        if mk == 0:
            continue
        acc = None
        for a, b, coef in _pair_terms(k, signs, idx, types):
            term = coef * X[a, b]
            acc = term if acc is None else acc + term
        if k == 3:
            y[off:off + mk] -= acc
        else:
            y[off:off + mk] -= SCALE[k] * acc
        off += mk
    return y


def op_Bt(cuts: Cuts, X: np.ndarray, t: np.ndarray) -> np.ndarray:
    """X -= B^T(t), symmetric scatter (src/operators.c:140-481).

    Each cut adds +-temp to both (p_a, p_b) and (p_b, p_a) with
    temp = t/2, t/4, t/6 (src/operators.c:154,202,292).  Contributions to
    one entry are applied in cut order (tri, then pent, then hept).
    """
    X = np.array(X, dtype=np.float64, copy=True)
    off = 0
    for k, idx, types, signs in cuts.groups():
        mk = len(types)
        if mk == 0:
            continue
        temp = (0.5 * SCALE[k]) * t[off:off + mk] if k != 3 else 0.5 * t[off:off + mk]
        if k == 7:
            temp = (1.0 / 6.0) * t[off:off + mk]
        e = np.array([signs[int(tt)] for tt in types], dtype=np.float64).reshape(-1, k)
        for c in range(mk):
            for a in range(k):
                for b in range(a + 1, k):
                    v = e[c, a] * e[c, b] * temp[c]
                    pa, pb = idx[c, a], idx[c, b]
                    X[pa, pb] += v
                    X[pb, pa] += v
        off += mk
    return X


# --------------------------------------------------------------------------
# Basic SDP: primal-dual predictor-corrector IPM (src/ipm_mc_pk.c:28-359)
# --------------------------------------------------------------------------
def _is_pd(A: np.ndarray) -> bool:
    try:
        np.linalg.cholesky(A)
        return True
    except np.linalg.LinAlgError:
        return False


@dataclass
class IpmResult:
    X: np.ndarray
    phi: float
    iters: int
    alphas: list
    y: np.ndarray = None   # the dual vector of the last iterate (phi = its sum)


def sdp_certificate(L: np.ndarray, y: np.ndarray):
    """FP64 certificate of a basic SDP bound from any dual vector y: returns
    (bound, lambda_lb, shift).  No reference counterpart (the reference's
    bound is its IPM's e'y); this restates the library's certificate
    (csrc/certificate.cu) for its tests.  For any y, max <L, X> over
    diag(X) = e, X psd is at most e'y + n max(0, -lambda_min(Diag(y) - L));
    a completed floating-point Cholesky factorisation of A = Diag(y) - L + tI
    gives lambda_min(A) >= -g/(1-g) trace(A), g = (n+1)u/(1-(n+1)u) (Higham,
    Accuracy and Stability of Numerical Algorithms, Theorem 10.3).  The shift
    t is 0, else found by doubling from trace * 2^-40 and 40 bisections; the
    errors of forming the diagonal and of summing y are added as there.
    LAPACK's factorisation stands in for the kernel's (the bound holds for
    any completed one)."""
    L = np.asarray(L, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    n = len(y)
    u = 2.0 ** -53

    def gam(k):
        return k * u / (1.0 - k * u)

    z = y - np.diag(L)
    sy, say, tr, mz = float(y.sum()), float(np.abs(y).sum()), float(np.abs(z).sum()), float(np.abs(z).max())
    slack = 1.0 + 4.0 * n * u

    def passes(t):
        A = -L.copy()
        A[np.diag_indices(n)] = z + t
        try:
            np.linalg.cholesky(A)
            return True
        except np.linalg.LinAlgError:
            return False

    t = 0.0
    ok = passes(0.0)
    if not ok:
        lo, t = 0.0, max(tr, 1.0) * 2.0 ** -40
        for _ in range(64):
            ok = passes(t)
            if ok:
                break
            lo, t = t, 2.0 * t
        if ok:
            for _ in range(40):
                mid = 0.5 * (lo + t)
                if not (lo < mid < t):
                    break
                if passes(mid):
                    t = mid
                else:
                    lo = mid
    if not ok:
        return float("inf"), float("-inf"), t
    g = gam(n + 1)
    lam = -(g / (1.0 - g) * (tr + n * t) * slack + t + 2.0 * u * (mz + t)) * slack
    corr = n * -lam if lam < 0 else 0.0
    v = sy + gam(n) * say * slack + corr
    return v + abs(v) * 2.0 ** -50, lam, t


def ipm_mc_pk(L: np.ndarray, max_iter: int = 500) -> IpmResult:
    """max <L,X> s.t. diag(X) = e, X psd; returns X, phi = e'y.

    Start y = 1.1 + column sums of |L|, X = I, Z = Diag(y) - L
    (src/ipm_mc_pk.c:65-99); loop while |phi - psi| > 1e-2 (:124-126).
    """
    L = np.asarray(L, dtype=np.float64)
    n = L.shape[0]
    e = np.ones(n)
    y = np.abs(L).sum(axis=0) + 1.1
    X = np.eye(n)
    Z = np.diag(y) - L
    phi = float(y.sum())
    psi = float(np.vdot(L, X))
    mu = float(np.vdot(Z, X)) / (2.0 * n)
    gap = abs(phi - psi)
    it = 0
    alphas = []
    while gap > 1e-2:
        it += 1
        if it > max_iter:
            raise RuntimeError("ipm_mc_pk: iteration limit")
        Zi = np.linalg.inv(Z)                     # :129-150 (dpotrf + dpotri)
        Zi = 0.5 * (Zi + Zi.T)
        M = Zi * X                                # :157-158
        cf = sla.cho_factor(M, lower=False)       # :166 dposv
        dy1 = sla.cho_solve(cf, -e)
        tmp = -(dy1[:, None] * X)                 # :181-184  -Diag(dy1) X
        dX1 = Zi @ tmp - X                        # :189-193
        dX1 = 0.5 * (dX1 + dX1.T)                 # :196-199
        dy = mu * np.diag(Zi) - (Zi * dX1) @ dy1  # :208-216
        dy2 = sla.cho_solve(cf, dy)               # :220-225
        tmp = -(dy2[:, None] * X) - (dy1[:, None] * dX1)   # :238-251
        dX = Zi @ tmp + mu * Zi                   # :257-260
        dy = dy1 + dy2                            # :265
        dX = dX1 + dX                             # :266
        dX = 0.5 * (dX + dX.T)                    # :269-272
        ap = 1.0                                  # :281-293 primal line search
        while not _is_pd(X + ap * dX):
            ap *= 0.8
        if ap < 1.0:
            ap *= 0.95
        ad = 1.0                                  # :297-309 dual line search
        while not _is_pd(Z + np.diag(ad * dy)):
            ad *= 0.8
        if ad < 1.0:
            ad *= 0.95
        X = X + ap * dX                           # :313-315
        y = y + ad * dy
        Z = Z + np.diag(ad * dy)
        mu = float(np.vdot(Z, X)) / (2.0 * n)     # :318
        if ap + ad > 1.6:                         # :321-324
            mu *= 0.5
        if ap + ad > 1.9:
            mu *= 0.2
        phi = float(y.sum())
        psi = float(np.vdot(L, X))
        gap = abs(phi - psi)
        alphas.append((ap, ad))
    return IpmResult(X=X, phi=phi, iters=it, alphas=alphas, y=y.copy())


def fct_eval(L: np.ndarray, cuts: Cuts, gamma: np.ndarray):
    """Dual function value and subgradient (src/bundle.c:242-275):
    L0 = L - B^T(gamma); X = IPM(L0); f = phi + sum(gamma); g = 1 - B(X)."""
    m = cuts.m
    L0 = op_Bt(cuts, L, gamma[:m]) if m > 0 else np.array(L, copy=True)
    r = ipm_mc_pk(L0)
    f = r.phi
    g = np.zeros(0)
    if m > 0:
        f += float(np.sum(gamma[:m]))
        g = op_B(cuts, np.ones(m), r.X)
    return f, r.X, g


# --------------------------------------------------------------------------
# Triangle separation (src/cutting_planes.c:20-214)
# --------------------------------------------------------------------------
def triangle_values(X: np.ndarray):
    """All 4*C(n,3) values in the reference's scan order (type, i, j, k),
    i > j > k (src/cutting_planes.c:58-64): value = B_c(X) - 1.
    Returns (types, ii, jj, kk, values) as flat arrays in scan order."""
    n = X.shape[0]
    ii, jj, kk = [], [], []
    for i in range(n):
        for j in range(i):
            kk.append(np.arange(j, dtype=np.int32))
            ii.append(np.full(j, i, np.int32))
            jj.append(np.full(j, j, np.int32))
    if n < 3:
        z = np.zeros(0, np.int32)
        return z, z, z, z, np.zeros(0)
    ii = np.concatenate(ii); jj = np.concatenate(jj); kk = np.concatenate(kk)
    a = X[ii, jj]; b = X[ii, kk]; c = X[jj, kk]
    # The reference is built with -ffast-math (its Makefile:17); gcc then
    # evaluates each four-term sum in a reassociated order.  These orders
    # reproduce the reference build's values bit for bit (checked against
    # oracle/_ref on every triple of several X by tests/test_oracle_golden.py).
    vals = [(-a - 1.0) + (-b - c), (-a - 1.0) + (b + c), (a - b) + (c - 1.0), (a - c) + (b - 1.0)]
    T = len(ii)
    types = np.repeat(np.arange(1, 5, dtype=np.int32), T)
    return types, np.tile(ii, 4), np.tile(jj, 4), np.tile(kk, 4), np.concatenate(vals)


def getViolated_TriangleInequalities(X: np.ndarray, tri_ineq: int, violated: float):
    """Streaming top-K of src/cutting_planes.c:48-127, replayed exactly.

    The first ``tri_ineq`` violated cuts (value > violated) fill the list in
    scan order; afterwards a cut with value > current minimum replaces the
    slot of the first-found minimum (strict <, lowest slot among ties), and
    the minimum is recomputed.  A heap keyed on (value, slot) reproduces
    "first-found minimum" exactly.
    Returns (list of (type, i, j, k, value) in slot order, maxAll).
    """
    types, ii, jj, kk, vals = triangle_values(X)
    max_all = float(vals.max()) if len(vals) else -BIG_NUMBER
    sel = np.nonzero(vals > violated)[0]
    lst = []
    heap = []
    for s in sel:
        v = float(vals[s])
        rec = (int(types[s]), int(ii[s]), int(jj[s]), int(kk[s]), v)
        if len(lst) < tri_ineq:
            heapq.heappush(heap, (v, len(lst)))
            lst.append(rec)
        elif v > heap[0][0]:
            _, slot = heapq.heappop(heap)
            lst[slot] = rec
            heapq.heappush(heap, (v, slot))
    return lst, max_all


def updateTriangleInequalities(cuts: Cuts, y: np.ndarray, X: np.ndarray, tri_ineq: int,
                               violated: float, max_added: int = 50000):
    """Purge cuts with y < 1e-5 (keeping order), separate on X, append the
    separated cuts not already present (src/cutting_planes.c:132-214).
    Returns (new tri array, new types, kept y, added, subtracted, maxAll)."""
    m_t = len(cuts.tri_type)
    keep = np.nonzero(y[:m_t] >= 1e-5)[0] if m_t else np.zeros(0, np.int64)
    # note: the reference tests `y < 1e-5` to drop; NaN would be kept
    tri = cuts.tri[keep]
    ttype = cuts.tri_type[keep]
    ykept = y[:m_t][keep]
    subtracted = m_t - len(keep)
    lst, max_all = getViolated_TriangleInequalities(X, tri_ineq, violated)
    existing = {(int(t), int(a), int(b), int(c)) for t, (a, b, c) in zip(ttype, tri)}
    new_rows, new_types = [], []
    count = len(keep)
    for (t, i, j, k, v) in lst:
        if count == max_added:
            break
        if (t, i, j, k) in existing:
            continue
        new_rows.append((i, j, k)); new_types.append(t)
        count += 1
    added = len(new_rows)
    if added:
        tri = np.concatenate([tri, np.array(new_rows, np.int32)])
        ttype = np.concatenate([ttype, np.array(new_types, np.int32)])
        ykept = np.concatenate([ykept, np.zeros(added)])
    return tri.astype(np.int32), ttype.astype(np.int32), ykept, added, subtracted, max_all


# --------------------------------------------------------------------------
# Heuristic (src/heuristic.c, src/bab_functions.c:96-107)
# --------------------------------------------------------------------------
def evaluateSolution(SP_L: np.ndarray, sol: np.ndarray) -> float:
    """sum_ij SP->L[i,j] s_i s_j over the first BabPbSize rows/cols
    (src/bab_functions.c:96-107)."""
    N = SP_L.shape[0] - 1
    s = np.asarray(sol[:N], dtype=np.float64)
    return float(s @ SP_L[:N, :N] @ s)


def mc_1opt(x: np.ndarray, P_L: np.ndarray) -> float:
    """Greedy best-flip local search in +-1 form (src/heuristic.c:195-296).
    Modifies x in place; returns x'Lx.  Ties: first index (strict >)."""
    N = len(x)
    xf = x.astype(np.float64)
    Lx = P_L @ xf
    d = np.diag(P_L).copy()
    cost = float(xf @ Lx)
    delta = d - xf * Lx
    index = int(np.argmax(delta))
    best = float(delta[index])
    while best > 0.001:
        col = P_L[:, index]
        I = np.abs(col) > 0.001
        if x[index] > 0:
            Lx[I] -= 2 * col[I]
        else:
            Lx[I] += 2 * col[I]
        x[index] = -x[index]
        xf[index] = -xf[index]
        cost += 4 * best
        delta = d - xf * Lx
        index = int(np.argmax(delta))
        best = float(delta[index])
    return cost


def GW_heuristic(P0_L, P_L, xfixed, sol_X, x, num, Zfac, V=None):
    """Random-hyperplane rounding + 1-opt (src/heuristic.c:119-186).

    Zfac: lower Cholesky factor (n x n) of the current Z.  V (num x n): the
    hyperplanes; when None they are drawn from rand() in the reference's
    order (count-major, then i; src/heuristic.c:142-143).  x is updated in
    place with the best lifted 0/1 solution (strictly better replaces,
    src/heuristic.c:304-318); returns the best value of this call.
    """
    N = P_L.shape[0]
    P0_N = P0_L.shape[0]
    best = -BIG_NUMBER
    free_idx = np.nonzero(np.asarray(xfixed[:P0_N - 1]) == 0)[0]
    for count in range(num):
        if V is None:
            v = np.array([rand() / RAND_MAX - 0.5 for _ in range(N)])
        else:
            v = V[count]
        sca = Zfac @ v
        tx = np.where(sca < 0, -1, 1).astype(np.int64)
        mc_1opt(tx, P_L)
        sol = np.array(sol_X[:P0_N - 1], dtype=np.int64).copy()
        sol[free_idx] = (tx[:len(free_idx)] + 1) // 2
        val = evaluateSolution(P0_L, sol)
        if best < val:
            best = val
            x[:P0_N - 1] = sol
    return best


def runHeuristic_unpacked(P0_L, P_L, xfixed, sol_X, x, Xmat):
    """Alternating GW rounding / convex re-mixing (src/heuristic.c:19-115).
    Consumes rand() exactly as the reference.  Returns the last GW value."""
    n = P_L.shape[0]
    P0_N = P0_L.shape[0]
    N = P0_N - 1
    xh = np.array([2 * (rand() % 2) - 1 for _ in range(n)], dtype=np.float64)
    temp = np.zeros(N, np.int64)
    idx = 0
    for i in range(N):
        if xfixed[i]:
            temp[i] = sol_X[i]
        else:
            temp[i] = int((xh[idx] + 1) / 2.0)
            idx += 1
    fh = evaluateSolution(P0_L, temp)
    done = 0
    Zm = np.array(Xmat, copy=True)
    heur_val = None
    while done < 2:
        done += 1
        Lf = np.linalg.cholesky(Zm)
        heur_val = GW_heuristic(P0_L, P_L, xfixed, sol_X, x, P0_N, Lf)
        if heur_val > fh:
            done = 0
            fh = heur_val
            idx = 0
            for i in range(N):
                if not xfixed[i]:
                    xh[idx] = 2 * x[i] - 1
                    idx += 1
            xh[n - 1] = -1.0
        c = 0.3 + 0.6 * (rand() / RAND_MAX)
        Zm = (1.0 - c) * Xmat + c * np.outer(xh, xh)
    return heur_val


# --------------------------------------------------------------------------
# Bundle QP (src/bundle.c:292-653)
# --------------------------------------------------------------------------
def solve_lambda(Q: np.ndarray, c: np.ndarray) -> np.ndarray:
    """min <lambda,c> + 1/2 <lambda,Q lambda> over the unit simplex by a
    primal-dual IPM (src/bundle.c:390-653): <= 31 iterations, |gap| > 1e-5."""
    k = len(c)
    lam = np.full(k, 1.0 / k)
    Qlam = Q @ lam
    tmp = Qlam + c
    mintmp = min(float(tmp.min()), BIG_NUMBER)
    if mintmp > 1:
        y = 0.0
        z = tmp.copy()
    else:
        y = mintmp - 1.0
        z = tmp - y
    mu = 0.5 * float(z @ lam) / k
    res_p = 1.0 - lam.sum()
    temp = float(lam @ Qlam)
    gap = (float(lam @ c) + 0.5 * temp) - (y - 0.5 * temp)
    cnt = 0
    while abs(gap) > 1e-5:
        cnt += 1
        M = np.zeros((k + 1, k + 1))
        M[:k, :k] = -Q - np.diag(z / lam)
        M[:k, k] = 1.0
        M[k, :k] = 1.0
        rhs = np.concatenate([c - y + Qlam, [res_p]])
        dw = np.linalg.solve(M, rhs)
        dlam, dy = dw[:k], dw[k]
        dz = 1.0 / lam * (mu - lam * z - z * dlam)
        ap = max(float(np.max(-dlam / lam)), -BIG_NUMBER)
        ad = max(float(np.max(-dz / z)), -BIG_NUMBER)
        ap = min(0.99 / ap, 1.0) if ap > 0 else 1.0
        ad = min(0.99 / ad, 1.0) if ad > 0 else 1.0
        y += ad * dy
        lam = lam + ap * dlam
        z = z + ad * dz
        res_p = 1 - lam.sum()
        Qlam = Q @ lam
        mu = 0.4 * float(lam @ z) / k
        if ap + ad > 1.8:
            mu *= 0.2
        temp = float(lam @ Qlam)
        gap = (float(lam @ c) + 0.5 * temp) - (y - 0.5 * temp)
        if cnt > 30:
            break
    return lam


def lambda_eta(zeta, G, gamma, t):
    """Alternate the lambda-QP and the eta projection (src/bundle.c:292-373).
    G: (m, k).  Returns (dgamma, lambda, eta, t)."""
    m, k = G.shape
    eta = np.zeros(m)
    Q = t * (G.T @ G)
    dir_prev = 0.0
    cnt = 0
    while True:
        cnt += 1
        c = zeta - t * (G.T @ eta)
        lam = solve_lambda(Q, c)
        tmp = G @ lam
        eta = np.maximum(-gamma / t + tmp, 0.0)
        dgamma = t * (eta - tmp)
        dir_curr = float(np.linalg.norm(dgamma))
        done = abs(dir_curr - dir_prev) / (1.0 + dir_curr) < 1e-5
        if cnt >= 50:
            done = True
            t *= 0.95
        dir_prev = dir_curr
        if done:
            return dgamma, lam, eta, t


MAX_BUNDLE = 400   # MaxBundle, src/biqbin.h:42


def bundle_inner(L: np.ndarray, X: np.ndarray) -> float:
    """<L, X> over the upper triangle, off-diagonal terms doubled, column by
    column (src/bundle.c:150-160, src/bounding.c:143-152)."""
    n = L.shape[0]
    temp = 0.0
    for i in range(n):
        temp += L[i, i] * X[i, i] + float(np.sum(2.0 * L[i + 1:, i] * X[i + 1:, i]))
    return temp


@dataclass
class Bundle:
    """The bundle: F[k] = <L, X_i>, G (m x k) subgradients, Xb the k primal
    matrices, in the reference's slot order (src/bundle.c:14-17)."""
    F: np.ndarray
    G: np.ndarray
    Xb: list

    @property
    def k(self) -> int:
        return len(self.F)


def bundle_method(L: np.ndarray, cuts: Cuts, gamma: np.ndarray, f: float, X: np.ndarray, bundle: Bundle,
                  t: float, bdl_iter: int):
    """bdl_iter proximal bundle iterations (src/bundle.c:9-239).  Returns
    (gamma, f, X, bundle, t); the inputs are not modified.

    Per iteration: zeta = -F - G'gamma; (dgamma, lambda) from lambda_eta;
    f_test = fct_eval(gamma + dgamma); del = f - (F + G'gamma_test)'lambda;
    a serious step (f - f_test > 0.05 del) moves gamma, sets X = Xb lambda,
    t *= 1.01, drops the elements with lambda < 0.01 max(lambda) and appends
    the new one; a null step keeps gamma and X, t /= 1.01, purges the first
    k - 1 elements the same way and keeps the last one after the new one."""
    gamma = np.array(gamma, dtype=np.float64, copy=True)
    X = np.array(X, dtype=np.float64, copy=True)
    F = np.array(bundle.F, dtype=np.float64, copy=True)
    G = np.array(bundle.G, dtype=np.float64, copy=True)
    Xb = [np.array(x, dtype=np.float64, copy=True) for x in bundle.Xb]
    for _ in range(bdl_iter):
        k = len(F)
        zeta = -F - G.T @ gamma                                  # :54-61
        dgamma, lam, _eta, t = lambda_eta(zeta, G, gamma, t)     # :64
        gamma_test = gamma + dgamma                              # :67-68
        f_test, X_test, g = fct_eval(L, cuts, gamma_test)        # :71
        dl = f - float((F + G.T @ gamma_test) @ lam)             # :74-81
        lmax = float(np.max(lam))                                # :84-86
        F_new = bundle_inner(L, X_test)
        if f - f_test > 0.05 * dl:                               # :91 serious step
            gamma = gamma_test
            f = f_test
            X = sum(lam[i] * Xb[i] for i in range(k))            # :106-108
            t *= 1.01
            keep = [i for i in range(k) if not lam[i] < 0.01 * lmax]
            if len(keep) == MAX_BUNDLE:
                raise RuntimeError("Bundle size too large")
            F = np.concatenate([F[keep], [F_new]])
            G = np.concatenate([G[:, keep], g[:, None]], axis=1)
            Xb = [Xb[i] for i in keep] + [X_test]
        else:                                                    # :169 null step
            t /= 1.01
            keep = [i for i in range(k - 1) if not lam[i] < 0.01 * lmax]
            if len(keep) + 1 == MAX_BUNDLE:
                raise RuntimeError("Bundle size too large")
            F = np.concatenate([F[keep], [F_new, F[k - 1]]])
            G = np.concatenate([G[:, keep], g[:, None], G[:, k - 1:k]], axis=1)
            Xb = [Xb[i] for i in keep] + [X_test, Xb[k - 1]]
    return gamma, f, X, Bundle(F, G, Xb), t


MAX_KGON_ADDED = 50000   # MaxPentIneqAdded, MaxHeptaIneqAdded, src/biqbin.h:38-39


def getViolated_KgonalInequalities(X: np.ndarray, k: int, trials: int, cap: int):
    """Pentagonal (k = 5, types 1-3) or heptagonal (k = 7, types 1-4)
    separation (src/cutting_planes.c:223-301 and its heptagonal twin): for
    each trial and type one annealing chain (the C restatement in
    oracle/kgon_sa_chain.c, drawing from rand() with the reference's flags);
    values below 1 fill a list of at most `cap`, beyond which a more violated
    one replaces the tracked least violated entry.  Returns (list of
    (type, permutation, value), the smallest chain value).

    The reference's re-scan after a replacement starts from BIG_NUMBER and
    looks for a larger value, so it never moves the tracked entry again;
    this is kept."""
    from . import portbind
    types = 3 if k == 5 else 4
    n = X.shape[0]
    Xc = np.ascontiguousarray(np.asarray(X, dtype=np.float64).T).reshape(-1)
    lst = []
    least_idx, least_val, min_all = 0, -BIG_NUMBER, BIG_NUMBER
    for _ in range(trials):
        for typ in range(1, types + 1):
            v, perm = portbind.qap_sa_glibc(Xc, n, k, typ)
            min_all = v if v < min_all else min_all
            if v < 1.0:
                if len(lst) < cap:
                    lst.append((typ, tuple(int(a) for a in perm), v))
                    if len(lst) == 1 or v > least_val:
                        least_val, least_idx = v, len(lst) - 1
                elif v < least_val:
                    lst[least_idx] = (typ, tuple(int(a) for a in perm), v)
                    least_val = BIG_NUMBER
                    for q, entry in enumerate(lst):
                        if entry[2] > least_val:
                            least_val, least_idx = entry[2], q
    return lst, min_all


def updateKgonalInequalities(perm: np.ndarray, types: np.ndarray, y: np.ndarray, X: np.ndarray, k: int,
                             trials: int, cap: int):
    """Purge the k-gonal cuts whose multiplier is below 1e-5 (keeping
    order), separate, append the separated cuts that are not among the kept
    ones (src/cutting_planes.c:307-404 and its heptagonal twin).  Returns
    (perm, types, y of the new list, added, subtracted, smallest value)."""
    m_old = len(types)
    keep = [i for i in range(m_old) if not y[i] < 1e-5]
    perm = np.asarray(perm, dtype=np.int32).reshape(-1, k)[keep]
    types = np.asarray(types, dtype=np.int32)[keep]
    ykept = np.asarray(y[:m_old], dtype=np.float64)[keep]
    lst, min_all = getViolated_KgonalInequalities(X, k, trials, cap)
    existing = {(int(t), tuple(int(a) for a in p)) for t, p in zip(types, perm)}
    new_perm, new_types = [], []
    count = len(keep)
    for t, p, _v in lst:
        if count == MAX_KGON_ADDED:
            break
        if (t, p) in existing:
            continue
        new_perm.append(p)
        new_types.append(t)
        count += 1
    added = len(new_types)
    if added:
        perm = np.concatenate([perm, np.array(new_perm, np.int32)])
        types = np.concatenate([types, np.array(new_types, np.int32)])
        ykept = np.concatenate([ykept, np.zeros(added)])
    return perm, types, ykept, added, m_old - len(keep), min_all


@dataclass
class BoundResult:
    """What SDPbound leaves behind: the bound it returns, the incumbent
    value and cut (Bab_LBGet / BabSol after its updateSolution calls), the
    node's fracsol, and diff (set at the root, rank 0)."""
    bound: float
    lb: float
    best_x: np.ndarray
    fracsol: np.ndarray
    diff: float
    outer_iterations: int
    prune: bool
    giveup: bool
    kgon_rounds: int = 0   # pentagonal / heptagonal separation calls


def _fracsol(X, xfixed, sol, N):
    """Fixed variables keep their value, free ones 0.5 (X[n-1, i] + 1)
    (src/bounding.c:76-87, 246-257)."""
    n = X.shape[0]
    out = np.zeros(N)
    idx = 0
    for i in range(N):
        if xfixed[i]:
            out[i] = float(sol[i])
        else:
            out[i] = 0.5 * (X[n - 1, idx] + 1.0)
            idx += 1
    return out


def SDPbound(SP_L: np.ndarray, xfixed, sol, lb: float, best_x, prm: dict, rank: int = 1,
             diff: float = 0.0) -> BoundResult:
    """The node bound (src/bounding.c:24-342).

    prm holds the reference's parameters (init_bundle_iter, max_bundle_iter,
    triag_iter, pent_iter, hept_iter, max_outer_iter, extra_iter,
    violated_TriIneq, TriIneq after adjust_TriIneq, use_diff, include_Pent,
    include_Hepta, PentIneq, HeptaIneq, Pent_Trials, Hepta_Trials).  lb /
    best_x: the incumbent (Bab_LBGet / BabSol) before the call; diff: the
    global diff.  The heuristic and the k-gonal annealing draw from rand()
    in the reference's order, so call srand() first to reproduce a run.

    The cut lists keep the multipliers their last update stored (the
    reference's Cuts[i].y, Pent_Cuts[i].y, Hepta_Cuts[i].y); after each
    separation round the dual vector is rebuilt from them, so a k-gonal kind
    that was not separated in a round gets back the multipliers of its last
    separation (src/bounding.c:261-271)."""
    N = SP_L.shape[0] - 1
    xfixed = np.asarray(xfixed[:N])
    sol = np.asarray(sol[:N])
    best_x = np.array(best_x[:N], dtype=np.int64, copy=True)
    L = create_subproblem(SP_L, xfixed, sol)
    fixedvalue = fixed_value(SP_L, xfixed, sol)                  # :60
    cuts = Cuts()
    r = ipm_mc_pk(L)                                             # :73
    X, f = r.X, r.phi
    basic_bound = f + fixedvalue
    fracsol = _fracsol(X, xfixed, sol, N)

    def heuristic(Xcur, lb, best_x):                             # :90-103, :182-195
        x = np.where(xfixed != 0, sol, 0).astype(np.int64)
        runHeuristic_unpacked(SP_L, L, xfixed, sol, x, Xcur)
        val = evaluateSolution(SP_L, x)
        if val > lb:                                             # Bab_LBUpd, src/heap.c:185-193
            return val, x.copy()
        return lb, best_x

    lb, best_x = heuristic(X, lb, best_x)
    bound = f + fixedvalue
    if bound < lb + 1.0:                                         # :109
        return BoundResult(bound, lb, best_x, fracsol, diff, 0, True, False)
    if prm["use_diff"] and rank != 0 and bound > lb + diff + 1.0:   # :115
        return BoundResult(bound, lb, best_x, fracsol, diff, 0, False, True)

    tri, ttype, ytri, _, _, viol3 = updateTriangleInequalities(cuts, np.zeros(0), X, int(prm["TriIneq"]),
                                                                float(prm["violated_TriIneq"]))   # :120
    cuts = Cuts(tri=tri, tri_type=ttype)
    ypent, yhept = np.zeros(0), np.zeros(0)
    gamma = ytri.copy()
    viol5 = 0.0
    m = cuts.m
    t = 0.5 * (bound - lb) / (m * viol3 * viol3)                 # :133
    g = op_B(cuts, np.ones(m), X)                                # :138-139
    bundle = Bundle(F=np.array([bundle_inner(L, X)]), G=g[:, None].copy(), Xb=[X.copy()])

    bdl_iter = int(prm["init_bundle_iter"])
    count = 0
    kgon_rounds = 0
    prune = giveup = False
    while True:
        count += 1                                               # :168-172
        oldf = f
        gamma, f, X, bundle, t = bundle_method(L, cuts, gamma, f, X, bundle, t, bdl_iter)
        bound = f + fixedvalue
        prune = bound < lb + 1.0
        if not prune:
            lb, best_x = heuristic(X, lb, best_x)
            prune = bound < lb + 1.0
        gap = bound - lb
        if count == prm["triag_iter"] + prm["pent_iter"] + prm["hept_iter"]:     # :201-205
            if gap - 1.0 > (oldf - f) * (prm["max_outer_iter"] - count):
                giveup = True
        if count == prm["max_outer_iter"]:                       # :208-211
            if gap - 1.0 > (oldf - f) * prm["extra_iter"]:
                giveup = True
        if count == prm["max_outer_iter"] + prm["extra_iter"]:   # :214-215
            giveup = True
        if not prune and not giveup:                             # :219-230
            triag, penta = len(cuts.tri_type), len(cuts.pent_type)
            tri, ttype, ytri, _, _, viol3 = updateTriangleInequalities(cuts, gamma, X, int(prm["TriIneq"]),
                                                                        float(prm["violated_TriIneq"]))
            pent, ptype, hept, htype = cuts.pent, cuts.pent_type, cuts.hept, cuts.hept_type
            if prm.get("include_Pent", 0) and (count > prm["triag_iter"] or viol3 < 0.2):
                pent, ptype, ypent, _, _, viol5 = updateKgonalInequalities(
                    pent, ptype, gamma[triag:], X, 5, int(prm["Pent_Trials"]), int(prm["PentIneq"]))
                kgon_rounds += 1
            if prm.get("include_Hepta", 0) and ((count > prm["triag_iter"] + prm["pent_iter"])
                                                or (viol3 < 0.2 and (1 - viol5 < 0.4))):
                hept, htype, yhept, _, _, _ = updateKgonalInequalities(
                    hept, htype, gamma[triag + penta:], X, 7, int(prm["Hepta_Trials"]), int(prm["HeptaIneq"]))
                kgon_rounds += 1
            cuts = Cuts(tri=tri, tri_type=ttype, pent=np.asarray(pent, np.int32).reshape(-1, 5),
                        pent_type=np.asarray(ptype, np.int32), hept=np.asarray(hept, np.int32).reshape(-1, 7),
                        hept_type=np.asarray(htype, np.int32))
        done = prune or giveup
        fracsol = _fracsol(X, xfixed, sol, N)                    # :246-257
        if not done:                                             # :260-315
            gamma = np.concatenate([ytri, ypent, yhept])
            m = cuts.m
            _, X_test, g = fct_eval(L, cuts, gamma)
            k = bundle.k
            G = np.column_stack([op_B(cuts, np.ones(m), bundle.Xb[i]) for i in range(k)] + [g])
            if k == MAX_BUNDLE:
                raise RuntimeError("Bundle size too large")
            bundle = Bundle(F=np.concatenate([bundle.F, [bundle_inner(L, X_test)]]), G=G,
                            Xb=bundle.Xb + [X_test])
            t *= 1.05
        bdl_iter += count % 2                                    # :320-321
        bdl_iter = min(bdl_iter, int(prm["max_bundle_iter"]))
        if done:
            break
    bound = f + fixedvalue
    if rank == 0:
        diff = basic_bound - bound                               # :328-329
    return BoundResult(bound, lb, best_x, fracsol, diff, count, prune, giveup, kgon_rounds)


# --------------------------------------------------------------------------
# Instance construction (src/process_input.c:259-344, src/evaluate.c:38-138)
# --------------------------------------------------------------------------
def build_SP_L(adj: np.ndarray) -> np.ndarray:
    """SP->L = [Lap, Lap e; (Lap e)', e'Lap e] over the first nv-1 vertices
    (src/process_input.c:289-333); the last vertex is fixed to 0."""
    nv = adj.shape[0]
    lap = np.diag(adj.sum(axis=1)) - adj
    L = np.zeros((nv, nv))
    L[:nv - 1, :nv - 1] = lap[:nv - 1, :nv - 1]
    rs = L[:nv - 1, :nv - 1].sum(axis=1)
    L[:nv - 1, nv - 1] = rs
    L[nv - 1, :nv - 1] = rs
    L[nv - 1, nv - 1] = rs.sum()
    return L


def create_subproblem(SP_L: np.ndarray, xfixed: np.ndarray, sol: np.ndarray) -> np.ndarray:
    """PP->L for a node (src/evaluate.c:38-115), scaled by 1/4."""
    N = SP_L.shape[0] - 1
    free = [i for i in range(N) if not xfixed[i]]
    nf = len(free)
    n = nf + 1
    L = np.zeros((n, n))
    A = SP_L[:N, :N]
    L[:nf, :nf] = A[np.ix_(free, free)]
    L[:nf, nf] = L[:nf, :nf].sum(axis=1)
    L[nf, :nf] = L[:nf, nf]
    ones = [i for i in range(N) if xfixed[i] and sol[i] == 1]
    fixed_row = A[np.ix_(ones, free)].sum(axis=0) if ones else np.zeros(nf)
    for i in range(nf):
        L[i, i] += 2 * fixed_row[i]
        L[nf, i] += 2 * fixed_row[i]
        L[i, nf] += 2 * fixed_row[i]
    L[nf, nf] = L[:nf, nf].sum()
    return 0.25 * L


def fixed_value(SP_L: np.ndarray, xfixed, sol) -> float:
    """getFixedValue (src/evaluate.c:123-138)."""
    N = SP_L.shape[0] - 1
    f = np.array([1.0 if (xfixed[i] and sol[i]) else 0.0 for i in range(N)])
    return float(f @ SP_L[:N, :N] @ f)
