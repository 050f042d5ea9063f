"""Generate the golden fixtures in tests/golden/ from the reference's own C
code (oracle/_ref, built from the reference sources by oracle/Makefile).

Run in a container that has the reference sources:
    make -C oracle ref && python tests/golden/make_golden.py

Every input is seeded synthetic data (parallel_biqbin_maxcut_b200.instances);
every output is what the reference build returns for it.  The fixtures pin
the CPU oracle (oracle/bqb_oracle.py) and the host-side separation code
without needing the reference at test time.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import bqb_oracle as O  # noqa: E402
from oracle import refbind  # noqa: E402
from parallel_biqbin_maxcut_b200 import _lib, instances  # noqa: E402

libc = C.CDLL("libc.so.6")
libc.rand.restype = C.c_int


def colmajor(A):
    return np.ascontiguousarray(np.asarray(A, dtype=np.float64).T).reshape(-1)


def from_col(v, n):
    return np.asarray(v[: n * n]).reshape(n, n).T.copy()


def main():
    ref = refbind.RefLib()
    A0 = instances.gnp_unit(31, 0.5, 101)
    ref.setup(A0, {"init_bundle_iter": 5, "violated_TriIneq": 0.05})
    SPL = ref.SP_L()
    N0 = SPL.shape[0]
    out = {}

    # 1. IPM on two subproblems
    rng = np.random.default_rng(5)
    for tag, (xf, sol) in (("root", (np.zeros(N0 - 1, np.int32), np.zeros(N0 - 1, np.int32))),
                           ("sub", instances.random_fixings(N0, 1, 8, seed=6)[0])):
        L = O.create_subproblem(SPL, xf, sol)
        X, phi = ref.ipm(L)
        out[f"ipm_{tag}_L"] = L
        out[f"ipm_{tag}_X"] = X
        out[f"ipm_{tag}_phi"] = np.array([phi])

    # 2. op_B / op_Bt with triangle, pentagonal and heptagonal cuts
    n = 20
    cuts = O.Cuts(
        tri=np.array([np.sort(rng.choice(n, 3, replace=False))[::-1] for _ in range(40)], np.int32),
        tri_type=rng.integers(1, 5, 40).astype(np.int32),
        pent=np.array([rng.choice(n, 5, replace=False) for _ in range(12)], np.int32),
        pent_type=rng.integers(1, 4, 12).astype(np.int32),
        hept=np.array([rng.choice(n, 7, replace=False) for _ in range(9)], np.int32),
        hept_type=rng.integers(1, 5, 9).astype(np.int32))
    Cp = ref.gptr("Cuts", refbind.TriIneq)
    Pp = ref.gptr("Pent_Cuts", refbind.PentIneq)
    Hp = ref.gptr("Hepta_Cuts", refbind.HeptIneq)
    for c in range(40):
        Cp[c].i, Cp[c].j, Cp[c].k = (int(v) for v in cuts.tri[c])
        Cp[c].type = int(cuts.tri_type[c])
    for c in range(12):
        Pp[c].type = int(cuts.pent_type[c])
        for a in range(5):
            Pp[c].permutation[a] = int(cuts.pent[c, a])
    for c in range(9):
        Hp[c].type = int(cuts.hept_type[c])
        for a in range(7):
            Hp[c].permutation[a] = int(cuts.hept[c, a])
    Xs = rng.standard_normal((n, n))
    Xs = Xs + Xs.T
    Xc = colmajor(Xs)
    prob = refbind.Problem()
    prob.L = Xc.ctypes.data_as(C.POINTER(C.c_double))
    prob.n, prob.NIneq, prob.NPentIneq, prob.NHeptaIneq = n, 40, 12, 9
    y = rng.standard_normal(cuts.m)
    yo = y.copy()
    ref.lib.op_B(C.byref(prob), refbind.dptr(yo), refbind.dptr(Xc))
    t = np.abs(rng.standard_normal(cuts.m))
    Xo = Xc.copy()
    ref.lib.op_Bt(C.byref(prob), refbind.dptr(Xo), refbind.dptr(t))
    for k, v in (("tri", cuts.tri), ("tri_type", cuts.tri_type), ("pent", cuts.pent),
                 ("pent_type", cuts.pent_type), ("hept", cuts.hept), ("hept_type", cuts.hept_type)):
        out[f"cuts_{k}"] = v
    out.update(cuts_X=Xs, cuts_y=y, cuts_yout=yo, cuts_t=t, cuts_Xout=from_col(Xo, n))

    # 3. triangle separation: the full value table (thr -10, list = all
    #    triples in scan order) and a streaming top-K case
    for tag, (nv, seed, T, thr) in (("all", (12, 7, 10 ** 6, -10.0)), ("topk", (30, 8, 60, 0.05))):
        Xm = O.ipm_mc_pk(O.create_subproblem(O.build_SP_L(instances.gnp_unit(nv, 0.5, seed)),
                                             np.zeros(nv - 1, int), np.zeros(nv - 1, int))).X
        ref.set_param("TriIneq", min(T, 4 * nv ** 3))
        ref.set_param("violated_TriIneq", thr)
        cap = min(T, 4 * nv ** 3)
        lst = (refbind.TriIneq * cap)()
        size = C.c_int()
        mx = ref.lib.getViolated_TriangleInequalities(refbind.dptr(colmajor(Xm)), nv, lst, C.byref(size))
        out[f"tri_{tag}_X"] = Xm
        out[f"tri_{tag}_param"] = np.array([cap, thr])
        out[f"tri_{tag}_list"] = np.array([(lst[q].type, lst[q].i, lst[q].j, lst[q].k) for q in range(size.value)],
                                          np.int32).reshape(-1, 4)
        out[f"tri_{tag}_values"] = np.array([lst[q].value for q in range(size.value)])
        out[f"tri_{tag}_max"] = np.array([mx])

    # 4. heuristic on a subproblem of SP, from a fixed rand() state
    xf, sol = instances.random_fixings(N0, 1, 6, seed=9)[0]
    L = O.create_subproblem(SPL, xf, sol)
    nsub = L.shape[0]
    Xm = O.ipm_mc_pk(L).X
    refX = ref.gptr("X", C.c_double)
    Xc = colmajor(Xm)
    for q in range(nsub * nsub):
        refX[q] = Xc[q]
    libc.srand(4242)
    x = np.zeros(N0 - 1, np.int32)
    v = ref.lib.runHeuristic_unpacked(refbind.dptr(colmajor(SPL)), N0, refbind.dptr(colmajor(L)), nsub,
                                      refbind.iptr(xf), refbind.iptr(sol), refbind.iptr(x))
    out.update(heur_SPL=SPL, heur_L=L, heur_X=Xm, heur_xfixed=xf, heur_sol=sol, heur_seed=np.array([4242]),
               heur_value=np.array([v]), heur_x=x, heur_rand_after=np.array([libc.rand()]))

    # 5. mc_1opt
    x0 = rng.choice(np.array([-1, 1], np.int32), nsub)
    xo = x0.copy()
    cost = ref.lib.mc_1opt(refbind.iptr(xo), refbind.dptr(colmajor(L)), nsub)
    out.update(opt_L=L, opt_x0=x0, opt_x=xo, opt_cost=np.array([cost]))

    # 6. solve_lambda and lambda_eta
    G = rng.standard_normal((60, 7)) * 0.3
    tq = 0.3
    Q = tq * (G.T @ G)
    c = rng.standard_normal(7) * 3
    lam = np.zeros(7)
    ref.lib.solve_lambda(7, refbind.dptr(colmajor(Q)), refbind.dptr(c.copy()), refbind.dptr(lam))
    out.update(qp_Q=Q, qp_c=c, qp_lambda=lam)
    zeta = -rng.random(7) * 10
    gam = np.where(rng.random(60) < 0.5, 0.0, rng.random(60))
    prob = refbind.Problem()
    prob.NIneq, prob.bundle = 60, 7
    dg, lm, et = np.zeros(60), np.zeros(7), np.zeros(60)
    tt = C.c_double(tq)
    Gc = colmajor(G)   # m x k, column-major
    ref.lib.lambda_eta(C.byref(prob), refbind.dptr(zeta.copy()), refbind.dptr(Gc), refbind.dptr(gam.copy()),
                       refbind.dptr(dg), refbind.dptr(lm), refbind.dptr(et), C.byref(tt))
    out.update(le_G=G, le_zeta=zeta, le_gamma=gam, le_t=np.array([tq]), le_dgamma=dg, le_lambda=lm, le_eta=et,
               le_tout=np.array([tt.value]))

    # 7. simulated annealing (pentagonal H2) from a fixed rand() state
    ref.lib.qap_simulated_annealing.restype = C.c_double
    ref.lib.qap_simulated_annealing.argtypes = [C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_double), C.c_int,
                                               C.POINTER(C.c_int)]
    e = np.array([-1, 1, 1, 1, 1])
    Hm = np.ascontiguousarray(np.outer(e, e).reshape(-1), dtype=np.int32)
    libc.srand(77)
    p = np.zeros(5, np.int32)
    sa_v = ref.lib.qap_simulated_annealing(refbind.iptr(Hm), 5, refbind.dptr(colmajor(Xm)), nsub, refbind.iptr(p))
    out.update(sa_X=Xm, sa_H=Hm, sa_seed=np.array([77]), sa_value=np.array([sa_v]), sa_perm=p,
               sa_rand_after=np.array([libc.rand()]))

    np.savez_compressed(os.path.join(HERE, "components.npz"), **out)

    # 9. bundle_method on the root of SP; 10. SDPbound (its own process: the
    #    reference's globals are sized once per process)
    bundle_golden(ref, SPL)
    subprocess.run([sys.executable, os.path.abspath(__file__), "--sdpbound"], check=True)

    # 8. end-to-end optimal values of the reference's serial B&B
    e2e = []
    with tempfile.TemporaryDirectory() as td:
        # the last four: the QUBO configuration at n = 100 (Max-Cut on 101
        # vertices) and two held-out instances of the learned warm start's
        # family, G(n, 0.9) with integer weights in [-10, 10]
        # and the 7 x 7 x 7 torus (n = 343, couplings N(0,1) x 1e5; about 5
        # minutes of the reference's serial B&B)
        for kind, nv, seed in (("unit", 40, 1), ("unit", 60, 2), ("pm1", 40, 3), ("qubo", 30, 4),
                               ("qubo", 100, 1), ("qubo", 100, 2), ("int10", 60, 911), ("int10", 80, 913),
                               ("torus", 343, 1)):
            if kind == "torus":
                A = instances.torus3d(7, seed)
            elif kind == "unit":
                A = instances.gnp_unit(nv, 0.5, seed)
            elif kind == "pm1":
                A = instances.gnp_pm1(nv, 0.5, seed)
            elif kind == "int10":
                A = instances.gnp_int(nv, 0.9, 10, seed)
            else:
                A = instances.qubo_to_maxcut(instances.qubo_dense(nv, 0.1, seed))
            inst, prm = os.path.join(td, "g.rudy"), os.path.join(td, "params")
            instances.write_rudy(inst, A)
            instances.write_params(prm, _lib.PARAMS_FILE)
            txt = subprocess.run([refbind.REF_BAB, inst, prm], capture_output=True, text=True,
                                 env=dict(os.environ, OPENBLAS_NUM_THREADS="1")).stdout
            e2e.append({"kind": kind, "nv": nv, "seed": seed,
                        "max_value": float(re.search(r"Maximum value = (\S+)", txt).group(1)),
                        "nodes": int(re.search(r"Nodes = (\d+)", txt).group(1)),
                        "root_bound": float(re.search(r"Root node bound = (\S+)", txt).group(1))})
    with open(os.path.join(HERE, "bab_optima.json"), "w") as fh:
        json.dump(e2e, fh, indent=1)
    print("wrote components.npz, bundle.npz, sdpbound.npz and bab_optima.json in", HERE)


def bundle_golden(ref, SPL):
    """The root of SP after the first triangle separation, the bundle set up
    as SDPbound does (src/bounding.c:120-157), then three calls of
    bundle_method with 4 iterations each, the third with t x 200 (null
    steps); the state after each call goes to bundle.npz."""
    N0 = SPL.shape[0]
    L = O.create_subproblem(SPL, np.zeros(N0 - 1, np.int32), np.zeros(N0 - 1, np.int32))
    n = L.shape[0]
    ref.set_param("TriIneq", 3 * n)
    ref.set_param("violated_TriIneq", 0.05)
    PP = C.POINTER(refbind.Problem).in_dll(ref.lib, "PP")
    pp = PP.contents
    Lc = colmajor(L)
    for q in range(n * n):
        pp.L[q] = Lc[q]
    pp.n, pp.NIneq, pp.NPentIneq, pp.NHeptaIneq = n, 0, 0, 0
    Xr, phi = ref.ipm(L)
    gX = ref.gptr("X", C.c_double)
    Xc = colmajor(Xr)
    for q in range(n * n):
        gX[q] = Xc[q]
    gamma = ref.gptr("dual_gamma", C.c_double)
    added, subtracted = C.c_int(), C.c_int()
    viol3 = ref.lib.updateTriangleInequalities(PP, gamma, C.byref(added), C.byref(subtracted))
    m = pp.NIneq
    cuts = ref.gptr("Cuts", refbind.TriIneq)
    tri = np.array([(cuts[c].i, cuts[c].j, cuts[c].k) for c in range(m)], np.int32).reshape(-1, 3)
    tri_type = np.array([cuts[c].type for c in range(m)], np.int32)
    for c in range(m):
        gamma[c] = cuts[c].y
    g = np.ones(m)
    ref.lib.op_B(PP, refbind.dptr(g), refbind.dptr(Xc))
    F0 = O.bundle_inner(L, Xr)
    gF, gG, gXb = ref.gptr("F", C.c_double), ref.gptr("G", C.c_double), ref.gptr("X_bundle", C.c_double)
    gF[0] = F0
    for c in range(m):
        gG[c] = g[c]
    for q in range(n * n):
        gXb[q] = Xc[q]
    pp.bundle = 1
    C.c_double.in_dll(ref.lib, "f").value = phi
    t = C.c_double(0.5 * 2.0 / (m * viol3 * viol3))   # a gap of 2 to the incumbent
    out = dict(L=L, tri=tri, tri_type=tri_type, gamma0=np.array([gamma[c] for c in range(m)]), f0=np.array([phi]),
               X0=Xr, F0=np.array([F0]), G0=g[:, None].copy(), t0=np.array([t.value]))
    for call in (1, 2, 3):
        if call == 3:
            t.value *= 200.0   # steps far too long: null steps
        ref.lib.bundle_method(PP, C.byref(t), 4)
        k = pp.bundle
        out[f"b{call}_f"] = np.array([C.c_double.in_dll(ref.lib, "f").value])
        out[f"b{call}_gamma"] = np.array([gamma[c] for c in range(m)])
        out[f"b{call}_X"] = from_col([gX[q] for q in range(n * n)], n)
        out[f"b{call}_F"] = np.array([gF[i] for i in range(k)])
        out[f"b{call}_G"] = np.array([gG[q] for q in range(m * k)]).reshape(k, m).T.copy()
        out[f"b{call}_t"] = np.array([t.value])
    np.savez_compressed(os.path.join(HERE, "bundle.npz"), **out)


SDP_PARAMS = {"init_bundle_iter": 5, "max_bundle_iter": 15, "triag_iter": 5, "pent_iter": 5, "hept_iter": 5,
              "max_outer_iter": 20, "extra_iter": 10, "violated_TriIneq": 0.05, "use_diff": 1,
              "include_Pent": 0, "include_Hepta": 0, "PentIneq": 5000, "HeptaIneq": 5000,
              "Pent_Trials": 60, "Hepta_Trials": 50}


def sdpbound_golden():
    """SDPbound (src/bounding.c:24-342) as Evaluate runs it, on G(50, 0.9)
    with integer weights in [-10, 10] (seed 4), each call from a fixed
    rand() state and from the incumbent the calls before left.  Triangle
    cuts only: the root at rank 0 with max_outer_iter = 7 and extra_iter = 0
    (it gives up after 7 outer iterations), the root with the default limits
    (it gives up at outer iteration 15 and sets diff), four subproblems at
    rank 1, the last with diff forced to 0.5 (the use_diff give-up).  With
    pentagonal and heptagonal cuts: the root capped at 7 and at 12 outer
    iterations (heptagonal separation starts after 10), two subproblems.
    Then the pentagonal and heptagonal updates alone on the root's X, three
    rounds each.  Inputs and results go to sdpbound.npz."""
    ref = refbind.RefLib()
    prm = dict(SDP_PARAMS)
    ref.setup(instances.gnp_int(50, 0.9, 10, 4), prm)
    SPL = ref.SP_L()
    N0 = SPL.shape[0]
    N = N0 - 1
    prm["TriIneq"] = ref.param("TriIneq")   # adjust_TriIneq: 10 SP->n
    PP = C.POINTER(refbind.Problem).in_dll(ref.lib, "PP")
    SP = C.POINTER(refbind.Problem).in_dll(ref.lib, "SP")
    babsol = C.POINTER(C.c_int).in_dll(ref.lib, "BabSol")
    root = (np.zeros(N, np.int32), np.zeros(N, np.int32))
    mo, ex = prm["max_outer_iter"], prm["extra_iter"]
    # (xfixed, sol, rank, max_outer_iter, extra_iter, k-gonal cuts, diff forced before the call)
    cases = [root + (0, 7, 0, 0, None), root + (0, mo, ex, 0, None)]
    fix = instances.random_fixings(N0, 6, 6, seed=31)
    cases += [(xf, sol, 1, mo, ex, 0, None) for xf, sol in fix[:3]]
    cases += [fix[3] + (1, mo, ex, 0, 0.5)]
    # pentagonal and heptagonal cuts on (the reference's defaults)
    cases += [root + (0, 7, 0, 1, None), root + (0, 12, 0, 1, None)]
    cases += [(xf, sol, 1, mo, ex, 1, None) for xf, sol in fix[4:]]
    out = {"SPL": SPL, "params": np.array([prm[k] for k in sorted(prm)]),
           "param_names": np.array(sorted(prm))}
    for q, (xf, sol, rank, max_outer, extra, kgon, force_diff) in enumerate(cases):
        ref.set_param("max_outer_iter", max_outer)
        ref.set_param("extra_iter", extra)
        ref.set_param("include_Pent", kgon)
        ref.set_param("include_Hepta", kgon)
        out[f"c{q}_limits"] = np.array([max_outer, extra, kgon])
        node = refbind.BabNode()
        node.xfixed[:N] = [int(v) for v in xf]
        node.sol[:N] = [int(v) for v in sol]
        out[f"c{q}_xfixed"], out[f"c{q}_sol"], out[f"c{q}_rank"] = xf, sol, np.array([rank])
        if force_diff is not None:
            ref.lib.bqbref_set_diff(force_diff)
        out[f"c{q}_lb_in"] = np.array([ref.lib.Bab_LBGet()])
        out[f"c{q}_best_in"] = np.array([babsol[i] for i in range(N)], np.int32)
        out[f"c{q}_diff_in"] = np.array([ref.lib.bqbref_get_diff()])
        libc.srand(500 + q)
        ref.lib.createSubproblem(C.byref(node), SP, PP)
        bound = ref.lib.SDPbound(C.byref(node), SP, PP, rank)
        out[f"c{q}_bound"] = np.array([bound])
        out[f"c{q}_lb_out"] = np.array([ref.lib.Bab_LBGet()])
        out[f"c{q}_best_out"] = np.array([babsol[i] for i in range(N)], np.int32)
        out[f"c{q}_fracsol"] = np.array(node.fracsol[:N])
        out[f"c{q}_diff_out"] = np.array([ref.lib.bqbref_get_diff()])
        out[f"c{q}_rand_after"] = np.array([libc.rand()])
    out["ncases"] = np.array([len(cases)])

    # the k-gonal updates alone (src/cutting_planes.c:223-602) on one X:
    # three rounds per kind, each purging every third cut first
    L = O.create_subproblem(SPL, np.zeros(N, np.int32), np.zeros(N, np.int32))
    n = L.shape[0]
    X = O.ipm_mc_pk(L).X
    pp = PP.contents
    pp.n, pp.NIneq, pp.NPentIneq, pp.NHeptaIneq = n, 0, 0, 0
    gX = ref.gptr("X", C.c_double)
    Xc = colmajor(X)
    for q in range(n * n):
        gX[q] = Xc[q]
    out["kg_X"] = X
    for k, fn, name, cls in ((5, "updatePentagonalInequalities", "Pent_Cuts", refbind.PentIneq),
                             (7, "updateHeptagonalInequalities", "Hepta_Cuts", refbind.HeptIneq)):
        for rnd in range(3):
            m = pp.NPentIneq if k == 5 else pp.NHeptaIneq
            y = np.where(np.arange(m) % 3 == 0, 0.0, 0.5)
            added, subtracted = C.c_int(), C.c_int()
            libc.srand(900 + rnd)
            v = getattr(ref.lib, fn)(PP, refbind.dptr(y.copy()), C.byref(added), C.byref(subtracted), 0)
            cuts = ref.gptr(name, cls)
            m2 = pp.NPentIneq if k == 5 else pp.NHeptaIneq
            tag = f"kg{k}_{rnd}"
            out[f"{tag}_y"] = y
            out[f"{tag}_perm"] = np.array([[cuts[c].permutation[j] for j in range(k)] for c in range(m2)],
                                          np.int32).reshape(-1, k)
            out[f"{tag}_type"] = np.array([cuts[c].type for c in range(m2)], np.int32)
            out[f"{tag}_yout"] = np.array([cuts[c].y for c in range(m2)])
            out[f"{tag}_counts"] = np.array([added.value, subtracted.value])
            out[f"{tag}_value"] = np.array([v])
            out[f"{tag}_rand_after"] = np.array([libc.rand()])
    np.savez_compressed(os.path.join(HERE, "sdpbound.npz"), **out)


if __name__ == "__main__":
    if sys.argv[1:] == ["--sdpbound"]:
        sdpbound_golden()
    else:
        main()
