"""Learned warm start of the bundle multipliers.

CPU: the network oracle's analytic gradient against central differences.
GPU: the library's training kernels (loss and gradient) and its BF16
inference kernel against the oracle; training lowers the loss; the
recorder yields training pairs; warm-started bounds are valid upper bounds
(checked by enumeration) and the warm start is off by default."""
import ctypes as C
import itertools

import numpy as np
import pytest

from oracle import warm_oracle as W
from parallel_biqbin_maxcut_b200 import _lib, warm


def _data(N, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((N, W.F)).astype(np.float32)
    y = np.abs(rng.standard_normal(N)).astype(np.float32)
    return X, y


def test_oracle_gradient_matches_central_differences():
    X, y = _data(40, 1)
    p = warm.init_params(3, lib=_FakeDims()).astype(np.float64)
    p[-1] = 0.3
    loss, g = W.loss_and_grad(p, X, y)
    idx = list(range(0, W.NPARAM, 37)) + [W.NPARAM - 1]
    num = W.numeric_grad(p, X, y, idx)
    np.testing.assert_allclose(g[idx], num, rtol=1e-5, atol=1e-8)
    assert loss > 0


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0], np.float32)
    r = W.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0078125)
    assert abs(r[3] + 3.140625) < 1e-6 and r[4] == 0.0


class _FakeDims:
    """Stands in for the library in warm.init_params on CPU (the network's
    sizes come from the oracle)."""

    def bqb_warm_dims(self, d):
        d[0], d[1], d[2] = W.F, W.H, W.NPARAM


@pytest.mark.gpu
def test_dims_match_oracle(lib):
    assert warm.dims(lib) == (W.F, W.H, W.NPARAM)


@pytest.mark.gpu
def test_gpu_gradient_matches_oracle(lib):
    X, y = _data(700, 2)
    p = warm.init_params(5, lib)
    p[-1] = 0.2
    g = np.zeros(W.NPARAM, np.float32)
    loss = C.c_float()
    assert lib.bqb_warm_grad(_lib.fptr(p), _lib.fptr(X), _lib.fptr(y), len(y), _lib.fptr(g), C.byref(loss)) == 0
    l_ref, g_ref = W.loss_and_grad(p, X, y)
    assert abs(loss.value - l_ref) <= 1e-5 * l_ref
    # float32 sums over 700 rows: relative to the gradient's scale
    np.testing.assert_allclose(g, g_ref, rtol=0, atol=2e-5 * np.abs(g_ref).max())


@pytest.mark.gpu
def test_bf16_inference_matches_oracle(lib):
    X, _ = _data(333, 4)
    p = warm.init_params(6, lib)
    out = np.zeros(len(X))
    assert lib.bqb_warm_predict(_lib.fptr(p), _lib.fptr(X), len(X), _lib.dptr(out)) == 0
    ref, _ = W.forward(W.bf16(p), X)
    np.testing.assert_allclose(out, ref, rtol=1e-4, atol=1e-5)
    assert np.all(out >= 0)


@pytest.mark.gpu
def test_training_lowers_loss(lib):
    X, _ = _data(6000, 7)
    teacher = warm.init_params(11, lib)
    y, _ = W.forward(teacher, X)
    y = y.astype(np.float32)
    p0 = warm.init_params(12, lib)
    l0, _ = W.loss_and_grad(p0, X, y)
    p, losses = warm.train(lib, X, y, steps=600, batch=512, lr=3e-3, seed=1, params=p0, standardize=False)
    l1, _ = W.loss_and_grad(p, X, y)
    assert l1 < 0.2 * l0, (l0, l1)
    assert losses[-20:].mean() < losses[:20].mean()


def _best_completion(A, xf, sol):
    nv = A.shape[0]
    free = np.flatnonzero(xf == 0)
    best = -np.inf
    for bits in itertools.product((0, 1), repeat=len(free)):
        x = np.zeros(nv, dtype=int)
        x[:-1] = np.where(xf == 1, sol, 0)
        x[free] = bits
        best = max(best, float(np.sum(np.triu(A, 1) * (x[:, None] != x[None, :]))))
    return best


@pytest.mark.gpu
def test_record_train_and_warm_bounds_are_valid(lib):
    """End to end on a small instance of the warm-start family: record
    pairs, train, bound held-out nodes with and without the warm start.
    Every bound must be an upper bound of the node's best cut."""
    feats, targets = warm.record_pairs(lib, [(40, 101), (40, 102)], nodes_per_instance=24, kmax=20, threads=8)
    assert len(targets) > 0 and feats.shape == (len(targets), W.F)
    assert np.all(targets >= 0) and np.all(np.isfinite(feats))
    p, _ = warm.train(lib, feats, targets, steps=300, batch=256, lr=3e-3, seed=2)
    A = warm.c5_instance(40, 103)
    inst = warm.Instance(lib, A)
    rng = np.random.default_rng(9)
    nodes = (_lib.BabNode * 8)()
    for q in range(8):
        xf = np.ones(39, dtype=int)
        xf[rng.choice(39, 8 + q % 3, replace=False)] = 0   # 8..10 free vertices
        sol = rng.integers(0, 2, 39) * xf
        nodes[q].xfixed[:39] = [int(v) for v in xf]
        nodes[q].sol[:39] = [int(v) for v in sol]
    res = warm.compare(lib, inst, nodes, p, threads=4)
    for q in range(8):
        xf, sol = np.array(nodes[q].xfixed[:39]), np.array(nodes[q].sol[:39])
        best = _best_completion(A, xf, sol)
        assert res["bounds_plain"][q] >= best - 1e-6
        assert res["bounds_warm"][q] >= best - 1e-6
    # off by default again, and the counters saw every node that reached the bundle
    st = (C.c_longlong * 2)()
    lib.bqb_warm_stats(st, 0)
    assert res["warm"]["kept"] + res["warm"]["rejected"] <= 8


@pytest.mark.gpu
def test_shipped_model_against_plain_bundle(lib):
    """What the trained network gains: full B&B on a held-out instance of
    its family, plain bundle and warm-started bundle.  The optimum must be
    identical and proposals must be used; the times, node counts and IPM
    calls of both runs are printed (run with -s) for the record."""
    p, meta = warm.load_model(warm.MODEL_C5)
    assert len(p) == W.NPARAM
    A = warm.c5_instance(60, 911)
    out = {}
    for mode in ("plain", "warm"):
        warm.use_model(lib, p if mode == "warm" else None)
        st = (C.c_longlong * 2)()
        lib.bqb_warm_stats(st, 1)
        r = _lib.solve(A, threads=16, time_limit=120)
        lib.bqb_warm_stats(st, 1)
        out[mode] = dict(opt=r["best_value"], nodes=r["nodes"], seconds=round(r["seconds"], 3), kept=int(st[0]),
                         rejected=int(st[1]), stopped=r["stopped"])
    warm.use_model(lib, None)
    print(out)
    assert not out["plain"]["stopped"] and not out["warm"]["stopped"]
    assert out["warm"]["opt"] == out["plain"]["opt"]
    assert out["plain"]["kept"] == 0 and out["warm"]["kept"] >= 1


@pytest.mark.gpu
def test_fused_kernel_warm_start(lib):
    """The fused node kernel runs the same proposal (features, BF16
    network, one IPM, fallback): B&B optimum unchanged, proposals counted,
    and its bounds on enumerable nodes are valid upper bounds."""
    p, _ = warm.load_model(warm.MODEL_C5)
    A = warm.c5_instance(60, 911)
    plain = _lib.solve(A, fused_batch=64, fused_depth=2)
    st = (C.c_longlong * 2)()
    warm.use_model(lib, p)
    try:
        lib.bqb_warm_stats(st, 1)
        r = _lib.solve(A, fused_batch=64, fused_depth=2)
        lib.bqb_warm_stats(st, 1)
        assert r["best_value"] == plain["best_value"]
        assert st[0] + st[1] >= 1
        B = warm.c5_instance(40, 104)
        inst = warm.Instance(lib, B)
        rng = np.random.default_rng(10)
        nodes = (_lib.BabNode * 8)()
        for q in range(8):
            xf = np.ones(39, dtype=int)
            xf[rng.choice(39, 8 + q % 3, replace=False)] = 0
            nodes[q].xfixed[:39] = [int(v) for v in xf]
            nodes[q].sol[:39] = [int(v) for v in rng.integers(0, 2, 39) * xf]
        lib.bqb_reset_incumbent(C.c_double(-1e9))   # every node runs its bundle
        b = np.zeros(8)
        assert lib.bqb_bound_nodes_fused(nodes, 8, 1, _lib.dptr(b)) == 0, lib.bqb_last_error()
        for q in range(8):
            xf, sol = np.array(nodes[q].xfixed[:39]), np.array(nodes[q].sol[:39])
            assert b[q] >= _best_completion(B, xf, sol) - 1e-6
    finally:
        warm.use_model(lib, None)


def test_standardization_folds_into_the_first_layer():
    rng = np.random.default_rng(4)
    X = (rng.standard_normal((50, W.F)) * 3 + 2).astype(np.float32)
    mu, sd = X.mean(axis=0, dtype=np.float64), X.std(axis=0, dtype=np.float64)
    p = warm.init_params(8, lib=_FakeDims())
    q = warm.fold_standardization(p, mu, sd, W.F, W.H)
    a, _ = W.forward(p, (X - mu) / sd)
    b, _ = W.forward(q, X)
    np.testing.assert_allclose(b, a, rtol=1e-5, atol=1e-6)


def test_shipped_model_file():
    p, meta = warm.load_model(warm.MODEL_C5)
    assert p.dtype == np.float32 and len(p) == W.NPARAM and np.all(np.isfinite(p))
    assert meta["train_instances"] and "command" in meta
    g, _ = W.forward(p, np.zeros((3, W.F), np.float32))
    assert np.all(g >= 0)


@pytest.mark.gpu
def test_gpu_features_match_oracle(lib):
    from helpers import O, instances
    A = instances.gnp_int(30, 0.9, 10, 5)
    L = O.create_subproblem(O.build_SP_L(A), np.zeros(29, int), np.zeros(29, int))
    n = L.shape[0]
    rng = np.random.default_rng(3)
    Xm = rng.uniform(-1, 1, (n, n))
    Xm = 0.5 * (Xm + Xm.T)
    np.fill_diagonal(Xm, 1.0)
    cuts = []
    for _ in range(40):
        i, j, k = sorted(rng.choice(n, 3, replace=False), reverse=True)
        cuts.append((int(rng.integers(1, 5)), int(i), int(j), int(k)))
    values = rng.uniform(0.05, 0.9, len(cuts))
    out = np.zeros((len(cuts), W.F), np.float32)
    ci = np.ascontiguousarray(np.array(cuts, dtype=np.int32).ravel())
    assert lib.bqb_warm_features(_lib.dptr(_lib.colmajor(Xm)), _lib.dptr(_lib.colmajor(L)), n, _lib.iptr(ci),
                                 _lib.dptr(values), len(cuts), 0.9, 12.5, None, _lib.fptr(out)) == 0
    ref = W.features(Xm, L, cuts, values, 0.9, 12.5)
    np.testing.assert_allclose(out, ref, rtol=1e-6, atol=1e-6)
    # with the parent's multipliers: half the cuts were in the parent's list
    pg = np.where(np.arange(len(cuts)) % 2 == 0, rng.uniform(0, 3, len(cuts)), -1.0)
    assert lib.bqb_warm_features(_lib.dptr(_lib.colmajor(Xm)), _lib.dptr(_lib.colmajor(L)), n, _lib.iptr(ci),
                                 _lib.dptr(values), len(cuts), 0.9, 12.5, pg.ctypes.data,
                                 _lib.fptr(out)) == 0
    np.testing.assert_allclose(out, W.features(Xm, L, cuts, values, 0.9, 12.5, pg), rtol=1e-6, atol=1e-6)
    bad = ci.copy()
    bad[1] = n   # index out of range: rejected before any device work
    assert lib.bqb_warm_features(_lib.dptr(_lib.colmajor(Xm)), _lib.dptr(_lib.colmajor(L)), n, _lib.iptr(bad),
                                 _lib.dptr(values), len(cuts), 0.9, 12.5, None, _lib.fptr(out)) == -1


@pytest.mark.gpu
def test_parent_cuts_reach_children(lib):
    """B&B with the recorder on: every child node sees its parent's final
    cuts, so some recorded first-list cuts carry the parent's multiplier
    (feature 13 = 1), and the parent cuts the child's own separation did not
    find join the list as candidates (their violation is evaluated at the
    child's X).  Targets are the multipliers the cuts end with (>= 0).
    The instance's tree has dozens of nodes (39 in the reference's serial
    B&B), so children that run the cutting-plane loop exist whatever the
    engines' random streams do."""
    assert lib.bqb_seed_engines(2021) == 0
    feats, targets = warm.record_pairs_bab(lib, [(80, 913)], threads=4, time_limit=60)
    assert len(targets) > 0 and feats.shape == (len(targets), W.F)
    assert np.all(np.isfinite(feats)) and np.all(targets >= 0)
    with_parent = feats[:, 13] > 0.5
    assert with_parent.any() and (~with_parent).any()
    assert np.all(feats[with_parent, 12] >= 0) and np.all(feats[~with_parent, 12] == 0)


@pytest.mark.gpu
def test_parent_informed_bab_reaches_reference_optimum(lib):
    """The parallel B&B with the shipped model on (proposals and a shortlist
    built from each child's parent cuts) reaches the optimum the reference's
    serial B&B printed (tests/golden/bab_optima.json); every bound it uses
    is a bound at some gamma >= 0, so the optimum cannot change."""
    import json
    import os
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "bab_optima.json")) as fh:
        case = next(c for c in json.load(fh) if c["kind"] == "int10" and c["nv"] == 80)
    A = warm.c5_instance(case["nv"], case["seed"])
    p, _ = warm.load_model(warm.MODEL_C5)
    warm.use_model(lib, p)
    try:
        r = _lib.solve(A, threads=8)
    finally:
        warm.use_model(lib, None)
    assert r["best_value"] == case["max_value"]
