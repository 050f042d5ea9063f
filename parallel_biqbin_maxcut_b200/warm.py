"""Learned warm start of the bundle multipliers (host side).

SDPbound starts its bundle at gamma = 0 after the first triangle separation
(src/bounding.c:121-131).  The library can start it instead from multipliers
proposed by a small network (csrc/warm.h): the proposal is evaluated once and
kept only when its dual value is below the plain start's, so every bound
stays valid and the plain bundle still runs to its own stopping rules.

This module generates training pairs with the plain method (random
subproblems of seeded instances bounded by engines with the recorder on),
trains the network on the GPU with the library's own kernels, saves and
loads models, and compares warm-started and plain bounding on held-out
nodes (IPM calls per node, time, bounds).
"""
from __future__ import annotations

import ctypes as C
import json
import os
import time

import numpy as np

from . import _lib, instances


def dims(lib=None):
    lib = lib or _lib.load()
    d = (C.c_int * 3)()
    lib.bqb_warm_dims(d)
    return tuple(d)


_BOUND_BUFFERS = None


class Instance:
    """A Max-Cut instance set up in the library (SP, globals, incumbent from
    the root node), ready for bqb_bound_nodes."""

    def __init__(self, lib, A, **param_overrides):
        self.lib = lib
        self.A = np.ascontiguousarray(A, dtype=np.float64)
        self.nv = self.A.shape[0]
        _lib.set_params(lib, _lib.make_params(**param_overrides))
        lib.process_adj_matrix(_lib.dptr(self.A.copy()), self.nv)
        self.glob = _lib.GlobalArrays(lib, self.nv)
        self.babsol = (C.c_int * _lib.NMAX)()
        C.c_void_p.in_dll(lib, "BabSol").value = C.addressof(self.babsol)
        # the library's globals now point into these buffers: keep them alive
        # until the next Instance re-points them
        global _BOUND_BUFFERS
        _BOUND_BUFFERS = (self.glob, self.babsol)
        SP = C.cast(C.c_void_p.in_dll(lib, "SP").value, C.POINTER(_lib.Problem))
        PP = C.cast(C.c_void_p.in_dll(lib, "PP").value, C.POINTER(_lib.Problem))
        C.CDLL("libc.so.6").srand(2020)
        # a fresh incumbent (a cut of value 0 always exists), so the root's
        # heuristic records its cut in babsol
        lib.bqb_reset_incumbent(C.c_double(0.0))
        root = _lib.BabNode()
        self.root_bound = lib.Evaluate(C.byref(root), SP, PP, 0)
        self.lb = lib.Bab_LBGet()

    def nodes(self, count, kmax, seed):
        arr = (_lib.BabNode * count)()
        for q, (xf, sol) in enumerate(instances.random_fixings(self.nv, count, kmax, seed)):
            arr[q].xfixed[: self.nv - 1] = [int(v) for v in xf]
            arr[q].sol[: self.nv - 1] = [int(v) for v in sol]
            arr[q].level = int(xf.sum())
        return arr

    def nodes_near(self, count, kmax, seed, flip=0.1):
        """Subproblems of the kind a B&B meets: k ~ U[0, kmax] vertices fixed
        to the incumbent cut's sides, each side flipped with probability
        `flip`."""
        rng = np.random.default_rng(seed)
        N = self.nv - 1
        best = np.array(self.babsol[:N], dtype=np.int64)
        arr = (_lib.BabNode * count)()
        for q in range(count):
            k = int(rng.integers(0, kmax + 1))
            idx = rng.choice(N, size=k, replace=False)
            xf = np.zeros(N, np.int64)
            xf[idx] = 1
            sol = np.zeros(N, np.int64)
            sol[idx] = best[idx] ^ (rng.random(k) < flip)
            arr[q].xfixed[:N] = [int(v) for v in xf]
            arr[q].sol[:N] = [int(v) for v in sol]
            arr[q].level = k
        return arr

    def bound(self, nodes, threads=16):
        """Bound copies of `nodes` from the root incumbent; returns bounds,
        IPM calls and seconds."""
        lib = self.lib
        arr = (_lib.BabNode * len(nodes))()
        C.memmove(arr, nodes, C.sizeof(nodes))
        lib.bqb_reset_incumbent(C.c_double(self.lb))
        out = np.zeros(len(nodes))
        lib.bqb_stats_reset()
        lib.bqb_stats_enable(1)
        t0 = time.perf_counter()
        rc = lib.bqb_bound_nodes(arr, len(nodes), 1, threads, None, _lib.dptr(out))
        sec = time.perf_counter() - t0
        st = (C.c_double * 6)()   # bqb_ipm_stats writes six values
        lib.bqb_ipm_stats(st)
        lib.bqb_stats_enable(0)
        assert rc == 0, lib.bqb_last_error()
        return out, int(st[1]), sec


def c5_instance(n, seed):
    """The learned-warm-start family: G(n, 0.9), integer weights in [-10, 10]."""
    return instances.gnp_int(n, 0.9, 10, seed)


def record_pairs(lib, sizes_seeds, nodes_per_instance=48, kmax=30, threads=16, node_seed=0):
    """Training pairs from the plain method: for each (n, seed), bound
    random subproblems with the recorder on.  Returns (features, targets)."""
    lib.bqb_warm_enable(0)
    lib.bqb_warm_dataset_clear()
    lib.bqb_warm_record(1)
    try:
        for q, (n, seed) in enumerate(sizes_seeds):
            inst = Instance(lib, c5_instance(n, seed))
            inst.bound(inst.nodes_near(nodes_per_instance, kmax, node_seed + q), threads)
    finally:
        lib.bqb_warm_record(0)
    F = dims(lib)[0]
    count = lib.bqb_warm_dataset(None, None, 0)
    feats = np.zeros((count, F), np.float32)
    targets = np.zeros(count, np.float32)
    lib.bqb_warm_dataset(_lib.fptr(feats), _lib.fptr(targets), count)
    return feats, targets


def record_pairs_bab(lib, sizes_seeds, threads=16, time_limit=60):
    """Training pairs from B&B trees solved by the plain method (no model),
    so that every child node sees its parent's final cuts: its features
    carry the parent's multipliers, and the parent's cuts its own
    separation did not find join its first list (targets then say which of
    them the bundle keeps).  Each instance runs to optimality or
    `time_limit` seconds.  Returns (features, targets)."""
    lib.bqb_warm_enable(0)
    lib.bqb_warm_dataset_clear()
    lib.bqb_warm_record(1)
    try:
        for n, seed in sizes_seeds:
            _lib.solve(c5_instance(n, seed), threads=threads, time_limit=time_limit)
    finally:
        lib.bqb_warm_record(0)
    F = dims(lib)[0]
    count = lib.bqb_warm_dataset(None, None, 0)
    feats = np.zeros((count, F), np.float32)
    targets = np.zeros(count, np.float32)
    lib.bqb_warm_dataset(_lib.fptr(feats), _lib.fptr(targets), count)
    return feats, targets


def evaluate_bab(lib, A, params, threads=16, time_limit=300):
    """The same B&B plain and warm-started (parent-informed proposals and
    shortlist), in the order plain, warm: seconds, nodes, bundle iterations
    per node, IPM calls per node, proposals kept / rejected, the optimum (or
    the incumbent at the time limit) and whether it stopped early."""
    out = {}
    for name, p in (("plain", None), ("warm", params)):
        use_model(lib, p)
        st = (C.c_longlong * 2)()
        lib.bqb_warm_stats(st, 1)
        lib.bqb_bundle_iterations(1)
        lib.bqb_stats_reset()
        lib.bqb_stats_enable(1)
        t0 = time.perf_counter()
        r = _lib.solve(A, threads=threads, time_limit=time_limit)
        sec = time.perf_counter() - t0
        ipm = (C.c_double * 6)()
        lib.bqb_ipm_stats(ipm)
        lib.bqb_stats_enable(0)
        bi = lib.bqb_bundle_iterations(1)
        lib.bqb_warm_stats(st, 1)
        out[name] = {"seconds": sec, "nodes": r["nodes"], "optimum": r["best_value"], "stopped": r["stopped"],
                     "root_bound": r["root_bound"], "bundle_iterations_per_node": bi / max(r["nodes"], 1),
                     "ipm_calls_per_node": float(ipm[1]) / max(r["nodes"], 1),
                     "proposals_kept": int(st[0]), "proposals_rejected": int(st[1])}
    use_model(lib, None)
    return out


def init_params(seed=0, lib=None):
    """He-normal weights, zero biases (the output bias starts at -2, so the
    first proposals are small multipliers)."""
    F, H, P = dims(lib)
    rng = np.random.default_rng(seed)
    p = np.zeros(P, np.float32)
    o = 0
    p[o:o + F * H] = rng.standard_normal(F * H) * np.sqrt(2.0 / F)
    o += F * H + H
    p[o:o + H * H] = rng.standard_normal(H * H) * np.sqrt(2.0 / H)
    o += H * H + H
    p[o:o + H] = rng.standard_normal(H) * np.sqrt(1.0 / H)
    p[-1] = -2.0
    return p


def train(lib, feats, targets, steps=3000, batch=2048, lr=1e-3, seed=0, params=None, standardize=True):
    """Train on the GPU (bqb_warm_train); returns (params, minibatch losses).
    With `standardize`, the network trains on features scaled to zero mean
    and unit variance, and the scaling is folded into the first layer of
    the returned parameters (which then take raw features)."""
    F, H, _ = dims(lib)
    p = init_params(seed, lib) if params is None else np.array(params, np.float32)
    feats = np.ascontiguousarray(feats, np.float32)
    mu = np.zeros(F)
    sd = np.ones(F)
    if standardize:
        mu = feats.mean(axis=0, dtype=np.float64)
        sd = feats.std(axis=0, dtype=np.float64)
        sd[sd < 1e-6] = 1.0
        feats = np.ascontiguousarray(((feats - mu) / sd).astype(np.float32))
    losses = np.zeros(steps, np.float32)
    targets = np.ascontiguousarray(targets, np.float32)
    rc = lib.bqb_warm_train(_lib.fptr(feats), _lib.fptr(targets), len(targets), steps, batch, lr, seed,
                            _lib.fptr(p), _lib.fptr(losses))
    assert rc == 0
    if standardize:
        p = fold_standardization(p, mu, sd, F, H)
    return p, losses


def fold_standardization(p, mu, sd, F, H):
    """Parameters that take raw features x from parameters trained on
    (x - mu) / sd: W1' = W1 / sd (by row), b1' = b1 - (mu / sd) W1."""
    p = np.array(p, np.float32)
    W1 = p[:F * H].reshape(F, H).astype(np.float64)
    b1 = p[F * H:F * H + H].astype(np.float64)
    p[F * H:F * H + H] = (b1 - (np.asarray(mu) / np.asarray(sd)) @ W1).astype(np.float32)
    p[:F * H] = (W1 / np.asarray(sd)[:, None]).astype(np.float32).ravel()
    return p


def save_model(path, params, meta=None):
    with open(path, "w") as fh:
        json.dump({"dims": list(dims()), "params": [float(v) for v in params], "meta": meta or {}}, fh)


def load_model(path):
    with open(path) as fh:
        d = json.load(fh)
    return np.array(d["params"], np.float32), d.get("meta", {})


def use_model(lib, params):
    """Load `params` into the library and switch the warm start on (None:
    off)."""
    if params is None:
        lib.bqb_warm_enable(0)
        lib.bqb_warm_set_model(None)
        return
    p = np.ascontiguousarray(params, np.float32)
    assert lib.bqb_warm_set_model(_lib.fptr(p)) == 0
    lib.bqb_warm_enable(1)


def compare(lib, inst, nodes, params, threads=16):
    """Plain and warm-started bounds of the same nodes from the same
    incumbent: per-node IPM calls, seconds, bounds, proposals kept."""
    use_model(lib, None)
    b0, ipm0, s0 = inst.bound(nodes, threads)
    use_model(lib, params)
    st = (C.c_longlong * 2)()
    lib.bqb_warm_stats(st, 1)
    b1, ipm1, s1 = inst.bound(nodes, threads)
    lib.bqb_warm_stats(st, 1)
    use_model(lib, None)
    m = len(nodes)
    return {"nodes": m, "plain": {"ipm_per_node": ipm0 / m, "seconds": s0, "mean_bound": float(b0.mean())},
            "warm": {"ipm_per_node": ipm1 / m, "seconds": s1, "mean_bound": float(b1.mean()),
                     "kept": int(st[0]), "rejected": int(st[1])},
            "bounds_plain": b0, "bounds_warm": b1}


# the shipped model, trained on TRAIN_C5 (its recipe is in the file's meta)
MODEL_C5 = os.path.join(os.path.dirname(__file__), "warm_model_c5.json")
TRAIN_C5 = [(80, 1), (80, 2), (100, 3), (100, 4), (120, 5), (120, 6), (150, 7), (150, 8)]


# held-out instances of the same family (seeds disjoint from TRAIN_C5's)
EVAL_C5 = [(100, 903), (100, 904), (150, 901)]


def main(argv):
    """python -m parallel_biqbin_maxcut_b200.warm train <out.json>: record
    pairs from B&B trees of the training instances (each child with its
    parent's final cuts) and train (the shipped model's recipe; recording
    order across engines is not deterministic, so a new model is close to,
    not identical with, the shipped one).
    python -m parallel_biqbin_maxcut_b200.warm evaluate <model.json> <out.json> [seconds]:
    plain against warm-started B&B on the held-out instances (each run to
    optimality or the time limit, 120 s by default)."""
    if len(argv) < 2 or argv[0] not in ("train", "evaluate"):
        print(main.__doc__)
        return 2
    lib = _lib.load()
    assert lib.bqb_init(0) == 0, lib.bqb_last_error()
    if argv[0] == "evaluate":
        p, _ = load_model(argv[1])
        limit = int(argv[3]) if len(argv) > 3 else 120
        res = {f"G({n},0.9) seed {sd}": evaluate_bab(lib, c5_instance(n, sd), p, time_limit=limit)
               for n, sd in EVAL_C5}
        with open(argv[2], "w") as fh:
            json.dump(res, fh, indent=1)
        print(json.dumps(res, indent=1))
        return 0
    feats, targets = record_pairs_bab(lib, TRAIN_C5, threads=16, time_limit=60)
    p, losses = train(lib, feats, targets, steps=6000, batch=4096, lr=1e-3, seed=0)
    save_model(argv[1], p, {"family": "G(n, 0.9), integer weights uniform in [-10, 10] (warm.c5_instance)",
                            "train_instances": TRAIN_C5,
                            "nodes": "every node of plain B&B trees (16 engines, 60 s per instance), each child "
                                     "with its parent's final cuts (record_pairs_bab)",
                            "pairs": int(len(targets)), "parent_pairs": int((feats[:, 13] > 0).sum()),
                            "training": "bqb_warm_train, Adam lr 1e-3, 6000 steps, batch 4096, seed 0, "
                                        "standardized features folded into layer 1",
                            "final_minibatch_mse": float(losses[-200:].mean()),
                            "target_variance": float(targets.var()),
                            "command": "python -m parallel_biqbin_maxcut_b200.warm train "
                                       "parallel_biqbin_maxcut_b200/warm_model_c5.json"})
    print(f"{len(targets)} pairs ({int((feats[:, 13] > 0).sum())} with a parent multiplier), final minibatch "
          f"MSE {losses[-200:].mean():.5f} (target variance {targets.var():.5f})")
    return 0


if __name__ == "__main__":
    import sys
    sys.exit(main(sys.argv[1:]))
