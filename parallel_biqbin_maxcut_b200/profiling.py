"""Summaries of Nsight Compute output for the profiles/ notes.

    python -m parallel_biqbin_maxcut_b200.profiling launches <launches.csv>
        per-kernel launch count, total time and share from a
        `ncu --metrics gpu__time_duration.sum --csv --log-file ...` list
    python -m parallel_biqbin_maxcut_b200.profiling raw <report.csv>
        selected counters from `ncu -i report.ncu-rep --page raw --csv`
    python -m parallel_biqbin_maxcut_b200.profiling ipm <n> <repeats>
        bound the root of a G(n, 0.5) +-1 instance (IPM kernel case)
    python -m parallel_biqbin_maxcut_b200.profiling ipm_torus <side> <repeats>
        the same for the side^3-vertex 3D torus (side 7: n = 343, the
        multi-CTA IPM case)
    python -m parallel_biqbin_maxcut_b200.profiling fused <n> <count> <kmax>
        bound `count` subproblems with the fused node kernel (nodek case)
"""
from __future__ import annotations

import collections
import csv
import re
import sys

UNIT = {"ns": 1e-3, "nsecond": 1e-3, "us": 1.0, "usecond": 1.0, "ms": 1e3, "msecond": 1e3, "s": 1e6, "second": 1e6}


def kernel_short_name(full: str) -> str:
    name = full.split("(")[0]
    name = re.sub(r"<.*>$", "", name) if not name.endswith(">::") else name
    return name.replace("bqb::", "").replace("<unnamed>::", "").strip()


def summarize_launches(path: str) -> str:
    rows = list(csv.reader(open(path)))
    hdr = next(i for i, r in enumerate(rows) if "Kernel Name" in r)
    h = rows[hdr]
    ki, vi, ui = h.index("Kernel Name"), h.index("Metric Value"), h.index("Metric Unit")
    agg = collections.defaultdict(lambda: [0, 0.0])
    for r in rows[hdr + 1:]:
        if len(r) <= vi or not r[vi]:
            continue
        us = float(r[vi].replace(",", "")) * UNIT.get(r[ui], 1.0)
        a = agg[kernel_short_name(r[ki])]
        a[0] += 1
        a[1] += us
    tot = sum(a[1] for a in agg.values())
    out = [f"{'kernel':44s} {'launches':>8s} {'total ms':>10s} {'share':>7s} {'avg us':>10s}"]
    for k, (c, t) in sorted(agg.items(), key=lambda x: -x[1][1]):
        out.append(f"{k[:44]:44s} {c:8d} {t / 1e3:10.3f} {100 * t / tot:6.2f}% {t / c:10.1f}")
    out.append(f"{'total':44s} {sum(a[0] for a in agg.values()):8d} {tot / 1e3:10.3f}")
    return "\n".join(out)


RAW_KEYS = ("gpu__time_duration.sum", "dram__bytes_read.sum", "dram__bytes_write.sum", "dram__cycles_active",
            "gpu__dram_throughput", "sm__pipe_tensor_cycles_active", "sm__warps_active",
            "smsp__average_warps_issue_stalled", "launch__registers_per_thread", "sm__throughput",
            "sm__inst_executed_pipe_fp64", "smsp__inst_executed.sum", "l1tex__data_bank_conflicts",
            "launch__shared_mem_per_block", "sm__pipe_fp64_cycles_active")


def summarize_raw(path: str) -> str:
    rows = list(csv.reader(open(path)))
    hdr = rows[0]
    units = rows[1] if len(rows) > 1 else [""] * len(hdr)
    out = []
    for r in rows[2:]:
        name = r[hdr.index("Kernel Name")] if "Kernel Name" in hdr else "?"
        out.append(f"== {kernel_short_name(name)}")
        for i, col in enumerate(hdr):
            if any(col.startswith(k) for k in RAW_KEYS):
                out.append(f"  {col} = {r[i]} {units[i]}")
    return "\n".join(out)


def run_ipm(n_vertices: int, repeats: int, torus: bool = False) -> None:
    """Bound the root of a seeded G(n, 0.5) +-1 instance (torus: of the
    n x n x n 3D torus with Gaussian couplings x 1e5, seed 1) `repeats` times
    through ipm_mc_pk (a small, self-contained case for kernel profiling;
    above 128 vertices it runs the multi-CTA IPM)."""
    import ctypes as C
    import time

    import numpy as np

    from . import _lib, instances

    lib = _lib.load()
    assert lib.bqb_init(0) == 0, lib.bqb_last_error()
    A = instances.torus3d(n_vertices, 1) if torus else instances.gnp_pm1(n_vertices, 0.5, seed=1)
    nv = A.shape[0]
    Lc = _lib.colmajor(instances.root_matrix(A))
    X = np.zeros(nv * nv)
    phi = C.c_double()
    for _ in range(repeats):
        t0 = time.perf_counter()
        lib.ipm_mc_pk(_lib.dptr(Lc), nv, _lib.dptr(X), C.byref(phi), 0)
        print(f"n={nv} phi={phi.value:.6f} wall={1e3 * (time.perf_counter() - t0):.3f} ms")


def run_fused(n_vertices: int, count: int, kmax: int) -> None:
    """Bound `count` subproblems (k ~ U[0, kmax] fixed vertices) of a seeded
    G(n, 0.5) +-1 instance with the fused node kernel, once (a small,
    self-contained case for profiling nodek_kernel)."""
    import ctypes as C

    import numpy as np

    from . import _lib, instances

    lib = _lib.load()
    assert lib.bqb_init(0) == 0, lib.bqb_last_error()
    A = np.ascontiguousarray(instances.gnp_pm1(n_vertices, 0.5, seed=1))
    _lib.set_params(lib, _lib.make_params(adjust_TriIneq=0, TriIneq=3 * n_vertices))
    lib.process_adj_matrix(_lib.dptr(A.copy()), n_vertices)
    glob = _lib.GlobalArrays(lib, n_vertices)
    sol = (C.c_int * _lib.NMAX)()
    C.c_void_p.in_dll(lib, "BabSol").value = C.addressof(sol)
    SP = C.cast(C.c_void_p.in_dll(lib, "SP").value, C.POINTER(_lib.Problem))
    PP = C.cast(C.c_void_p.in_dll(lib, "PP").value, C.POINTER(_lib.Problem))
    C.CDLL("libc.so.6").srand(2020)
    root = _lib.BabNode()
    rb = lib.Evaluate(C.byref(root), SP, PP, 0)
    nodes = (_lib.BabNode * count)()
    for q, (xf, sx) in enumerate(instances.random_fixings(n_vertices, count, kmax, seed=2)):
        nodes[q].xfixed[: n_vertices - 1] = [int(v) for v in xf]
        nodes[q].sol[: n_vertices - 1] = [int(v) for v in sx]
    b = np.zeros(count)
    assert lib.bqb_bound_nodes_fused(nodes, count, 1, _lib.dptr(b)) == 0, lib.bqb_last_error()
    print(f"n={n_vertices} root={rb:.6f} nodes={count} mean_bound={b.mean():.6f} "
          f"fallbacks={lib.bqb_fused_fallbacks()}")
    del glob


if __name__ == "__main__":
    mode = sys.argv[1]
    if mode == "ipm":
        run_ipm(int(sys.argv[2]), int(sys.argv[3]))
    elif mode == "ipm_torus":
        run_ipm(int(sys.argv[2]), int(sys.argv[3]), torus=True)
    elif mode == "fused":
        run_fused(int(sys.argv[2]), int(sys.argv[3]), int(sys.argv[4]))
    else:
        path = sys.argv[2]
        print(summarize_launches(path) if mode == "launches" else summarize_raw(path))
