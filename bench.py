#!/usr/bin/env python
"""Benchmark: B&B node-bounding throughput (nodes/s) on B200.

Workload (the batched node-bounding configuration): a G(100, 0.5) Max-Cut
instance with edge weights uniform in {-1, +1} (seeded, synthetic), and 512
of its B&B subproblems, each with k uniform in [0, 40] vertices fixed to
uniform 0/1 values (subproblem sizes n = 60..100), triangle budget
TriIneq = 3n (adjust_TriIneq = 0), otherwise the reference's shipped
parameters.  First the root is bounded with rank 0 (this sets the incumbent
and `diff` as the reference's master does); then every subproblem is bounded
as a worker bounds a node (rank 1): IPM, heuristic, prune / give-up tests,
cutting planes and bundle iterations to the reference's stopping rules.
A step bounds one batch of subproblems with the fused node kernel
(bqb_bound_nodes_fused: one persistent kernel, one CTA per SM, each CTA
bounding whole nodes on the device); the metric is nodes/s.

  value : device time of the fused kernel (CUDA events around its launch),
          plus any node it hands back to the engines
  e2e   : the same C-ABI call from host node structs, every host<->device
          copy inside the timed region
  engines : bqb_bound_nodes with --threads concurrent engines (one step)
  dropin_serial : the reference-facing Evaluate(node, SP, PP, 1), one node
          at a time on the library stream, as the reference's worker calls it

`--impl reference` times the reference's own C implementation (built
unmodified into oracle/_ref/libbqb_ref.so) on the host cores, one process per
core, each bounding its share of a sample of the same subproblems.

Multi-GPU (torchrun): B&B nodes are independent, so each rank bounds its own
share of the subproblems (weak scaling, no data-path collective); time is
the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import faulthandler
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from parallel_biqbin_maxcut_b200 import _lib, instances  # noqa: E402

NV = 100
N_SUB = 512
KMAX = 40
TRI_PER_N = 3
METRIC = "B&B nodes/s & time-to-optimality: batched+learned vs plain GPU, bounds ±1e-6 rel"
WORKLOAD = "G(100,0.5) ±1 weights; 512 subproblems, k~U[0,40] fixed (n=60..100); TriIneq=3n"
# Algorithmic flops of one IPM iteration at size n (the dense work of
# src/ipm_mc_pk.c per iteration: two SYMMs 4n^3, POTRF+POTRI of Z n^3,
# Cholesky of Zi.*X n^3/3 (reused for both solves), two line-search
# Cholesky factorizations 2n^3/3): 6.0 n^3; the reference's count with its
# second POSV is 6.33 n^3.  The smaller count is used.
FLOP_PER_ITER_N3 = 6.0
# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of the fused
# kernel per node, from one ncu capture of a 512-node launch of this workload
# (1.85 GB read + 3.97 GB written, 1 pass); the line reports it scaled to the
# average nodes per launch.
NODEK_DRAM_BYTES_PER_NODE = (1.85e9 + 3.97e9) / 512
NODEK_TRAFFIC_NOTE = ("ncu capture of one 512-node launch of this workload (1.85 GB read + 3.97 GB written), "
                      "scaled to the average nodes per launch")
FP64_NOMINAL_TFLOPS = 37.0


# Time-to-optimality instance: the batched configuration's graph itself,
# G(100, 0.5) with +-1 weights (seed 1), solved from scratch to optimality
# with the shipped parameters.
TTO_NAME = "G(100,0.5) +-1 weights, seed 1, full B&B, shipped params"
TORUS_NAME = ("3D torus 7x7x7 (n = 343), couplings N(0,1) x 1e5 rounded, seed 1, full B&B, shipped params "
              "(pentagonal and heptagonal cuts on)")
LEG_CALLS = {
    "fused": "bqb_solve_fused (batches of 2 x SMs, 8 in flight), FP64",
    "fused_learned": "bqb_solve_fused (batches of 2 x SMs, 8 in flight) with the shipped warm-start model",
    "engines": "bqb_solve_parallel (16 concurrent engines; above 128 vertices the fused kernel does not apply), "
               "GW rounding with 4096 hyperplanes per round projected on the tensor cores (TF32), root effort "
               "(the root runs every outer round of SDPbound unless pruned)",
    "engines_parent_start": "16 engines and 4096-hyperplane rounding as the engines leg, with parent start "
                            "(each child starts from its parent's final triangle, pentagonal and heptagonal cuts "
                            "and multipliers when that start's dual value is lower) and without root effort (the "
                            "root gives up as the reference's rule says; its children are cheap with parent start)",
    "engines_learned": "the engines leg with the shipped warm-start model (children start from the parent's "
                       "multipliers where the model keeps them)",
    "plain_dropin": "bqb_solve: serial best-first B&B, one node at a time through the drop-in SDPbound",
    "device_pool": "bqb_solve_device: the whole tree in one persistent launch, open-node pool on the device",
}


def tto_instance():
    return np.ascontiguousarray(instances.gnp_pm1(NV, 0.5, seed=1))


def workload():
    A = instances.gnp_pm1(NV, 0.5, seed=1)
    subs = instances.random_fixings(NV, N_SUB, KMAX, seed=2)
    return np.ascontiguousarray(A), subs


def workload_params() -> dict:
    p = dict(_lib.PARAMS_FILE)
    p.update(adjust_TriIneq=0, TriIneq=TRI_PER_N * NV)
    return p


def peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"],
                "bf16_tflops_sustained": d.get("bf16_tflops_sustained", d["bf16_tflops"]),
                "source": "measured"}
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0,
                "source": "fallback"}


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_node(xf, sol) -> _lib.BabNode:
    nd = _lib.BabNode()
    nd.xfixed[: len(xf)] = [int(v) for v in xf]
    nd.sol[: len(sol)] = [int(v) for v in sol]
    nd.level = int(np.sum(xf))
    return nd


# --------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------
class GpuArm:
    def __init__(self, device: int):
        import torch
        self.torch = torch
        self.lib = lib = _lib.load()
        assert lib.bqb_init(device) == 0, lib.bqb_last_error()
        self.device = device
        self.A, self.subs = workload()
        self.N0 = self.A.shape[0]
        _lib.set_params(lib, _lib.make_params(**workload_params()))
        lib.process_adj_matrix(_lib.dptr(self.A.copy()), self.N0)
        self.glob = _lib.GlobalArrays(lib, self.N0)
        self.babsol = (C.c_int * _lib.NMAX)()
        C.c_void_p.in_dll(lib, "BabSol").value = C.addressof(self.babsol)
        self.SP = C.cast(C.c_void_p.in_dll(lib, "SP").value, C.POINTER(_lib.Problem))
        self.PP = C.cast(C.c_void_p.in_dll(lib, "PP").value, C.POINTER(_lib.Problem))
        # keep the host address as an integer: a pointer read from a ctypes
        # structure field aliases the field itself
        self.PP_L_host = C.cast(self.PP.contents.L, C.c_void_p).value
        C.CDLL("libc.so.6").srand(2020)
        root = _lib.BabNode()
        self.root_bound = lib.Evaluate(C.byref(root), self.SP, self.PP, 0)
        self.lb = lib.Bab_LBGet()
        self.nodes = [make_node(xf, sol) for xf, sol in self.subs]
        self.flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{device}")
        torch.cuda.synchronize()

    def lib_sms(self) -> int:
        import torch
        return torch.cuda.get_device_properties(self.device).multi_processor_count

    def reset_problem(self):
        """Set the bench workload's problem up again (after a solver run)."""
        lib = self.lib
        _lib.set_params(lib, _lib.make_params(**workload_params()))
        lib.process_adj_matrix(_lib.dptr(self.A.copy()), self.N0)
        self.glob = _lib.GlobalArrays(lib, self.N0)
        C.c_void_p.in_dll(lib, "BabSol").value = C.addressof(self.babsol)
        self.SP = C.cast(C.c_void_p.in_dll(lib, "SP").value, C.POINTER(_lib.Problem))
        self.PP = C.cast(C.c_void_p.in_dll(lib, "PP").value, C.POINTER(_lib.Problem))
        self.PP_L_host = C.cast(self.PP.contents.L, C.c_void_p).value

    def node_array(self, idx):
        arr = (_lib.BabNode * len(idx))()
        for q, i in enumerate(idx):
            C.memmove(C.byref(arr[q]), C.byref(self.nodes[i]), C.sizeof(_lib.BabNode))
        return arr

    def bound_e2e(self, idx, threads):
        """engines leg: bqb_bound_nodes with host nodes; every subproblem is
        built on the host (createSubproblem) and copied in, and the bounds
        and fractional solutions come back to the host."""
        arr = self.node_array(idx)
        out = np.zeros(len(idx))
        rc = self.lib.bqb_bound_nodes(arr, len(idx), 1, threads, None, _lib.dptr(out))
        assert rc == 0, self.lib.bqb_last_error()
        return out

    def restore_host_L(self):
        self.PP.contents.L = C.cast(C.c_void_p(self.PP_L_host), C.POINTER(C.c_double))
        assert C.cast(self.PP.contents.L, C.c_void_p).value == self.PP_L_host

    def dropin_serial(self, idx):
        """The reference-facing drop-in: Evaluate one node at a time on the
        library stream, as the reference's worker calls it."""
        lib = self.lib
        return [lib.Evaluate(C.byref(self.nodes[i]), self.SP, self.PP, 1) for i in idx]

    def l2_flush(self):
        self.flush.zero_()


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def rank_batches(rank: int, B: int, nsteps: int, n_sub: int):
    """The subproblem indices rank `rank` bounds, as `nsteps` batches of B
    (weak scaling: every rank has its own share, per-rank work fixed)."""
    order = [(i * 7919 + rank * 131) % n_sub for i in range(B * nsteps)]
    return [order[s * B:(s + 1) * B] for s in range(nsteps)]


def make_collectives(pg, device: str, sync=None):
    """barrier() and max_over_ranks(x) over the process group `pg` (None:
    one process).  `sync` (e.g. torch.cuda.synchronize) runs on both sides
    of the barrier; the tensors live on `device`."""
    import torch

    def barrier():
        if sync:
            sync()
        if pg:
            pg.barrier()
        if sync:
            sync()

    def max_over_ranks(x):
        if not pg:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=device)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        return float(t.item())

    return barrier, max_over_ranks


def aggregate_rate(units_per_rank: int, world_size: int, ms_max: float) -> float:
    """Whole-job throughput: the units all ranks processed over the slowest
    rank's time."""
    return units_per_rank * world_size / (ms_max / 1e3)


def run_gpu(args):
    import torch
    ws, rank, local = _dist()
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    arm = GpuArm(local)
    lib = arm.lib
    B = args.nodes_per_step
    T = args.threads
    # rank r bounds its own share of the subproblems (weak scaling: per-GPU
    # work fixed); each step is a batch of B subproblems
    batches = rank_batches(rank, B, args.warmup + args.steps, N_SUB)
    timed = range(args.warmup, args.warmup + args.steps)
    barrier, max_over_ranks = make_collectives(pg, "cuda", torch.cuda.synchronize)

    def fused(arr):
        lib.bqb_reset_incumbent(arm.lb)   # every batch starts from the root's incumbent
        out = np.zeros(len(arr))
        rc = lib.bqb_bound_nodes_fused(arr, len(arr), 1, _lib.dptr(out))
        assert rc == 0, lib.bqb_last_error()
        return out

    def pipelined(arrs, depth):
        """Submit the batches with up to `depth` in flight; each submission
        is one launch of B nodes from the root's incumbent."""
        outs = [np.zeros(len(a)) for a in arrs]
        tickets = []
        for q, a in enumerate(arrs):
            if len(tickets) == depth:
                t, j = tickets.pop(0)
                assert lib.bqb_fused_collect(t, arrs[j], _lib.dptr(outs[j])) == 0, lib.bqb_last_error()
            lib.bqb_reset_incumbent(arm.lb)
            t = lib.bqb_fused_submit(a, len(a), 1)
            assert t >= 0, lib.bqb_last_error()
            tickets.append((t, q))
        for t, j in tickets:
            assert lib.bqb_fused_collect(t, arrs[j], _lib.dptr(outs[j])) == 0, lib.bqb_last_error()
        return outs

    stream = torch.cuda.current_stream()
    # warm-up: at least twice the window, so that every launch record's
    # arena and buffers are sized before the timed region
    nwarm = max(args.warmup, 2 * args.depth)
    pipelined([arm.node_array(batches[s % len(batches)]) for s in range(nwarm)], args.depth)

    # ---- value: the fused kernel (+ any node it hands back to an engine),
    # device time from CUDA events around the launch on its stream ----
    arrays = [arm.node_array(b) for b in batches]
    lib.bqb_stats_reset()
    lib.bqb_fused_stats_reset()
    clocks = ClockSampler(local)
    launches0 = lib.bqb_kernel_launches()
    barrier()
    clocks.start()
    arm.l2_flush()
    torch.cuda.synchronize()
    v0 = torch.cuda.Event(enable_timing=True)
    v1 = torch.cuda.Event(enable_timing=True)
    v0.record(stream)
    bounds_dev = pipelined([arrays[s] for s in timed], args.depth)
    v1.record(stream)
    torch.cuda.synchronize()
    nt = np.zeros(B)
    lib.bqb_fused_node_times(_lib.dptr(nt), B)
    node_ms = [nt]
    barrier()
    clk = clocks.stop()
    launches = lib.bqb_kernel_launches() - launches0
    stats = (C.c_double * 6)()
    lib.bqb_ipm_stats(stats)
    fst = (C.c_double * 5)()
    lib.bqb_fused_stats(fst)
    n_launch = int(lib.bqb_fused_launches())
    span_ms = v0.elapsed_time(v1)
    prof = (C.c_double * 11)()
    lib.bqb_fused_profile(prof)
    phase_names = ["subproblem", "ipm", "heuristic", "tri_scan", "tri_list", "kgon", "cut_upload", "opBt",
                   "opB", "lambda_eta", "bundle_step"]
    tot_cta_s = max(sum(prof), 1e-30)
    ms = span_ms
    ms_max = max_over_ranks(ms)
    value = aggregate_rate(B * args.steps, ws, ms_max)

    # ---- e2e: the same C-ABI call from host node structs, every copy in
    # the timed region (events on the idle current stream around the call) ----
    barrier()
    arm.l2_flush()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    pipelined([arm.node_array(batches[s]) for s in timed], args.depth)
    t1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = t0.elapsed_time(t1)
    barrier()
    ms_e2e = max_over_ranks(ms_e2e)
    e2e = aggregate_rate(B * args.steps, ws, ms_e2e)
    b0 = batches[args.warmup]
    N = NV - 1
    h2d = B * 2 * N * 4 + 8
    d2h = B * (8 + N * 8 + 8 + N * 4 + 4)

    # ---- concurrent engines (bqb_bound_nodes, host nodes) ----
    eng = None
    if T > 0 and args.engine_nodes > 0:
        ne = min(args.engine_nodes, B)
        lib.bqb_reset_incumbent(arm.lb)
        arm.bound_e2e(batches[0][:ne], T)   # warm the engine pool
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        lib.bqb_reset_incumbent(arm.lb)
        e0.record(stream)
        arm.bound_e2e(b0[:ne], T)
        e1.record(stream)
        torch.cuda.synchronize()
        eng = {"value": ne / (e0.elapsed_time(e1) / 1e3), "unit": "nodes/s", "engines": T, "nodes": ne,
               "call": "bqb_bound_nodes, host nodes, one step (after one warm-up step)"}

    # ---- FP64 certificates of node bounds (engines; one more IPM and a
    # Cholesky factorisation per node, after the timed region) ----
    cert = None
    if T > 0 and args.cert_nodes > 0:
        nc = min(args.cert_nodes, B)
        st = np.zeros(6)
        lib.bqb_certify_stats(_lib.dptr(st), 1)
        lib.bqb_certify_enable(1)
        lib.bqb_reset_incumbent(arm.lb)
        try:
            arm.bound_e2e(b0[:nc], min(T, 16))
        finally:
            lib.bqb_certify_enable(0)
        lib.bqb_certify_stats(_lib.dptr(st), 1)
        cert = {"nodes": int(st[0]), "max_rel_excess": float(st[1]), "mean_rel_excess": float(st[2]),
                "failed": int(st[3]), "max_shift": float(st[4]), "max_rerun_mismatch": float(st[5]),
                "call": "bqb_certify_enable(1) + bqb_bound_nodes on 16 engines, the first nodes of a timed batch",
                "meaning": "per node: (certified bound - node bound) / max(1, |node bound|); the certified bound is "
                           "sum(y) + n max(0, -lambda_lb(Diag(y) - L + B^T gamma)) + sum(gamma) + fixed value, "
                           "lambda_lb an FP64 lower bound from a completed Cholesky factorisation and its backward error"}

    # ---- the plain drop-in (one node at a time, library stream) ----
    drop = None
    if args.dropin_nodes > 0:
        idx = b0[: args.dropin_nodes]
        barrier()
        d0 = torch.cuda.Event(enable_timing=True)
        d1 = torch.cuda.Event(enable_timing=True)
        lib.bqb_reset_incumbent(arm.lb)
        d0.record(stream)
        arm.dropin_serial(idx)
        d1.record(stream)
        torch.cuda.synchronize()
        drop = {"value": len(idx) / (d0.elapsed_time(d1) / 1e3), "unit": "nodes/s",
                "nodes": len(idx), "call": "Evaluate(node, SP, PP, 1), host buffers, serial"}

    # ---- time to optimality: batched (+learned) vs the plain GPU drop-in ----
    tto = None
    if args.tto and rank == 0:
        from parallel_biqbin_maxcut_b200 import warm
        p_w, _ = warm.load_model(warm.MODEL_C5)
        sms = arm.lib_sms()
        fused_kw = dict(fused_batch=2 * sms, fused_depth=8)
        cases = [("n100", TTO_NAME, tto_instance(),
                  [("fused", fused_kw, None), ("fused_learned", fused_kw, p_w),
                   ("device_pool", dict(device_pool=True), None)])]
        if args.tto_torus:
            # the multi-CTA IPM's per-size schedule for the torus's sizes
            # (n = 343 and its subproblems, the same panel count)
            tto_sched = _lib.autotune_ipm([343], reps=2)
            cases.append(("torus343", TORUS_NAME, instances.torus3d(7, 1),
                          [("engines", dict(threads=16, gw_hyperplanes=4096, root_effort=True), None),
                           ("engines_parent_start", dict(threads=16, gw_hyperplanes=4096, root_effort=False,
                                                         parent_start=True), None),
                           ("engines_learned", dict(threads=16, gw_hyperplanes=4096, root_effort=True), p_w)]))
        tto = {}
        for key, name, A, legs in cases:
            e = {"instance": name}
            for leg, kw, model in legs:
                warm.use_model(arm.lib, model)
                t0 = time.perf_counter()
                r = _lib.solve(A, **kw)
                e[leg] = {"seconds": time.perf_counter() - t0, "optimum": r["best_value"], "nodes": r["nodes"],
                          "root_bound": r["root_bound"], "call": LEG_CALLS[leg]}
            warm.use_model(arm.lib, None)
            if args.tto_plain:
                t0 = time.perf_counter()
                r = _lib.solve(A)
                e["plain_dropin"] = {"seconds": time.perf_counter() - t0, "optimum": r["best_value"],
                                     "nodes": r["nodes"], "root_bound": r["root_bound"],
                                     "call": LEG_CALLS["plain_dropin"]}
                best = min(e[leg]["seconds"] for leg, _, _ in legs)
                e["speedup_batched_vs_plain"] = e["plain_dropin"]["seconds"] / best
                assert all(e[leg]["optimum"] == e["plain_dropin"]["optimum"] for leg, _, _ in legs), e
            if key == "torus343":
                e["ipm_schedule"] = tto_sched
            tto[key] = e
        # restore the bench's problem (the solver set up its own)
        arm.reset_problem()

    # ---- learned warm start: B&B to optimality, plain vs warm-started bundle ----
    learned = None
    if args.learned and rank == 0:
        from parallel_biqbin_maxcut_b200 import warm
        p_w, _ = warm.load_model(warm.MODEL_C5)
        A = warm.c5_instance(80, 913)
        learned = {"instance": "G(80,0.9), integer weights U[-10,10], seed 913 (held out from the model's "
                               "training instances)"}
        paths = (("engines", dict(threads=16)), ("fused", dict(fused_batch=2 * arm.lib_sms(), fused_depth=4)))
        # untimed first solves size every buffer for this instance; then
        # plain, warm, warm, plain per path (the order cancels drifts)
        for _, kw in paths:
            warm.use_model(arm.lib, None)
            _lib.solve(A, time_limit=300, **kw)
        runs = []
        if args.learned_plain:   # the plain GPU drop-in: serial B&B, one node at a time
            runs.append(("dropin_plain", None, dict()))
        for path, kw in paths:
            for mode in ("plain", "warm", "warm", "plain"):
                runs.append((f"{path}_{mode}", p_w if mode == "warm" else None, kw))
        for name, model, kw in runs:
            warm.use_model(arm.lib, model)
            kst = (C.c_longlong * 2)()
            arm.lib.bqb_warm_stats(kst, 1)
            t0 = time.perf_counter()
            r = _lib.solve(A, time_limit=300, **kw)
            sec = time.perf_counter() - t0
            arm.lib.bqb_warm_stats(kst, 1)
            e = learned.setdefault(name, {"seconds_runs": [], "optimum": r["best_value"], "nodes": [],
                                          "proposals_kept": 0, "proposals_rejected": 0})
            assert e["optimum"] == r["best_value"]
            e["seconds_runs"].append(sec)
            e["nodes"].append(r["nodes"])
            e["proposals_kept"] += int(kst[0])
            e["proposals_rejected"] += int(kst[1])
        for e in learned.values():
            if isinstance(e, dict):
                e["seconds"] = float(np.mean(e["seconds_runs"]))
        warm.use_model(arm.lib, None)
        learned["call"] = ("bqb_solve_parallel (16 engines) and bqb_solve_fused (batches of 2 x SMs, 4 in flight); "
                           "after an untimed solve per path, runs in the order plain, warm, warm, plain; "
                           "seconds = mean of the two runs")
        learned["speedup_warm_vs_plain_engines"] = (learned["engines_plain"]["seconds"] /
                                                    learned["engines_warm"]["seconds"])
        learned["speedup_warm_vs_plain_fused"] = learned["fused_plain"]["seconds"] / learned["fused_warm"]["seconds"]
        if "dropin_plain" in learned:
            learned["speedup_batched_learned_vs_plain_dropin"] = (learned["dropin_plain"]["seconds"] /
                                                                  learned["fused_warm"]["seconds"])
        arm.reset_problem()

    # ---- the torus configuration's IPM (n = 343: the multi-CTA IPM above n = 128) ----
    ipm343 = None
    if args.ipm_large and rank == 0:
        L343 = instances.root_matrix(instances.torus3d(7, 1))
        n343 = L343.shape[0]
        Lc = _lib.colmajor(L343)
        Xc = np.zeros(n343 * n343)
        phi = C.c_double()
        times = []
        for _ in range(4):
            t0 = time.perf_counter()
            arm.lib.ipm_mc_pk(_lib.dptr(Lc), n343, _lib.dptr(Xc), C.byref(phi), 0)
            times.append(time.perf_counter() - t0)
        ipm343 = {"instance": "3D torus 7x7x7 (n = 343), couplings N(0,1) x 1e5 rounded, seed 1, root node",
                  "call": "ipm_mc_pk with host buffers (copies inside the time)",
                  "ms_per_call": 1e3 * min(times[1:]), "ms_first_call": 1e3 * times[0], "phi": phi.value}

    pk = peaks()
    kernel_ms = fst[2]
    flops = FLOP_PER_ITER_N3 * stats[0]
    # the pipelined launches of the fused kernel cover the timed span (a
    # later launch starts while an earlier one's last nodes run), so the
    # achieved rate is the counted work over the span, not over the summed
    # (overlapping) launch durations
    achieved = flops / (span_ms / 1e3) / 1e12 if span_ms > 0 else 0.0
    peak = pk["bf16_tflops_sustained"]
    roof = {"kernel": "nodek_kernel", "bound": "tensor", "achieved": achieved, "peak": peak,
            "unit": "TFLOP/s", "frac": achieved / peak,
            "traffic": NODEK_DRAM_BYTES_PER_NODE * int(fst[0]) * B / max(n_launch, 1),
            "traffic_note": NODEK_TRAFFIC_NOTE,
            "peak_source": f"{pk['source']} bf16 sustained (the contract's compute denominator); the kernel "
                           "computes in FP64 on the CUDA cores (no tensor-core instruction), so its own ceiling "
                           f"is B200's nominal FP64 37 TFLOP/s: frac of that {achieved / FP64_NOMINAL_TFLOPS:.4f}",
            "pipe": "fp64 (CUDA cores)", "frac_of_fp64_nominal": achieved / FP64_NOMINAL_TFLOPS,
            "achieved_over": "span of the pipelined launches (CUDA events on the idle current stream around "
                             "every submission and collection)",
            "launches": n_launch, "submissions": int(fst[0]), "span_ms": span_ms,
            "avg_launch_ms": kernel_ms / max(n_launch, 1), "kernel_ms_summed": kernel_ms,
            "flops_counted": "IPM only: sum over IPM solves of iterations * 6 n^3",
            "ipm_iterations": int(stats[2]), "ipm_problems": int(stats[1]),
            "linesearch_factorizations": int(stats[3]),
            "fallback_nodes": int(fst[3]), "fallback_ms": fst[4],
            "node_ms": {"mean": float(np.mean(np.concatenate(node_ms))),
                        "p90": float(np.percentile(np.concatenate(node_ms), 90)),
                        "max": float(np.max(np.concatenate(node_ms))),
                        "sum_over_slots": float(np.sum(np.concatenate(node_ms)) / 1e3 / max(fst[0], 1)),
                        "note": "device time per node; sum_over_slots = CTA-seconds of node work per step"},
            "phase_share": {nm: round(prof[i] / tot_cta_s, 4) for i, nm in enumerate(phase_names)},
            "phase_cta_seconds": {nm: round(prof[i], 3) for i, nm in enumerate(phase_names)}}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "nodes/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "nodes_per_step": B, "nodes_per_step_total": B * ws,
                       "l2": "flushed (256 MB write) before every step", "precision": "FP64 throughout",
                       "mode": "fused node kernel: one CTA bounds a whole node; one launch per batch of "
                               f"{B} nodes, launches pipelined {args.depth} deep (bqb_fused_submit/collect)",
                       "root_bound": arm.root_bound, "incumbent": arm.lb,
                       "mean_bound": float(np.mean(np.concatenate(bounds_dev))),
                       "parallelism": f"replicas over nodes x{ws}"},
            "e2e": {"value": e2e, "unit": "nodes/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": ms_e2e / args.steps,
                    "call": "bqb_fused_submit/collect with host node structs"},
            "engines": eng,
            "certificate": cert,
            "dropin_serial": drop,
            "time_to_optimality": tto,
            "learned_warm_start": learned,
            "ipm_n343": ipm343,
            "gpu_launches": int(launches),
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


# --------------------------------------------------------------------------
# reference (CPU) arm -- the reference's own code, oracle/_ref
# --------------------------------------------------------------------------
def _ref_worker(conn, wid, nworkers):
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    from oracle import refbind
    A, subs = workload()
    ref = refbind.RefLib()
    ref.setup(A, workload_params())
    L = ref.lib
    SP = C.pointer(ref.problem("SP"))
    PP = C.pointer(ref.problem("PP"))
    C.CDLL("libc.so.6").srand(2020)
    root = refbind.BabNode()
    L.Evaluate(C.byref(root), SP, PP, 0)
    conn.send(("ready", L.Bab_LBGet()))
    while True:
        msg = conn.recv()
        if msg is None:
            break
        idx = msg
        t0 = time.perf_counter()
        for i in idx:
            xf, sol = subs[i]
            nd = refbind.BabNode()
            nd.xfixed[: len(xf)] = [int(v) for v in xf]
            nd.sol[: len(sol)] = [int(v) for v in sol]
            L.Evaluate(C.byref(nd), SP, PP, 1)
        conn.send(("done", time.perf_counter() - t0))


class RefPool:
    def __init__(self, nworkers: int):
        ctx = mp.get_context("spawn")
        self.conns, self.procs = [], []
        for w in range(nworkers):
            a, b = ctx.Pipe()
            p = ctx.Process(target=_ref_worker, args=(b, w, nworkers), daemon=True)
            p.start()
            self.conns.append(a)
            self.procs.append(p)
        self.lbs = [c.recv()[1] for c in self.conns]

    def run(self, assignments):
        for c, idx in zip(self.conns, assignments):
            c.send(idx)
        return [c.recv()[1] for c in self.conns]

    def run_dynamic(self, indices):
        """Hand the nodes out one at a time to whichever process is idle (as
        the reference's MPI master hands open nodes to free workers)."""
        from multiprocessing.connection import wait
        todo = list(indices)
        busy = {}
        for c in self.conns:
            if not todo:
                break
            c.send([todo.pop(0)])
            busy[c] = True
        while busy:
            for c in wait(list(busy)):
                c.recv()
                del busy[c]
                if todo:
                    c.send([todo.pop(0)])
                    busy[c] = True

    def close(self):
        for c in self.conns:
            c.send(None)
        for p in self.procs:
            p.join(timeout=10)


def cpu_baseline(seconds: float) -> dict:
    """One core, the reference's Evaluate on a bounded sample of the workload."""
    from oracle import refbind
    if not refbind.available():
        return {"value": None, "unit": "nodes/s", "cores": 1, "kind": "reference",
                "sample": "unavailable: oracle/_ref not built"}
    pool = RefPool(1)
    done, t = 0, 0.0
    i = 0
    while t < seconds and done < N_SUB:
        idx = [(i * 7919) % N_SUB, ((i + 1) * 7919) % N_SUB]
        t += pool.run([idx])[0]
        done += 2
        i += 2
    pool.close()
    return {"value": done / t, "unit": "nodes/s", "cores": 1, "kind": "reference",
            "sample": f"{done} of the 512 subproblems, same root state, serial reference build "
                      f"(-O3 -ffast-math, OpenBLAS 1 thread), {t:.1f} s"}


def run_reference(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return
    from oracle import refbind
    if not refbind.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (needs the reference sources)"}))
        return
    P = max(1, min(os.cpu_count() or 1, args.ref_procs))
    B = max(1, args.ref_nodes_per_step)
    pool = RefPool(P)
    # the GPU arm's node order; warm-up and timed steps are B nodes each, the
    # timed steps handed out as one stream (nodes of the next step start as
    # soon as a process is free, as the GPU arm's pipelined launches do)
    order = [(i * 7919) % N_SUB for i in range(B * (args.warmup + args.steps))]
    pool.run_dynamic(order[:B * args.warmup])
    t0 = time.perf_counter()
    pool.run_dynamic(order[B * args.warmup:])
    wall = time.perf_counter() - t0
    pool.close()
    nodes = B * args.steps
    v = nodes / wall
    tto = None
    if args.tto:
        import re
        import tempfile
        cases = [("n100", TTO_NAME, tto_instance())]
        if args.tto_torus:
            cases.append(("torus343", TORUS_NAME, instances.torus3d(7, 1)))
        tto = {}

        def ref_solve(key, name, A):
            with tempfile.TemporaryDirectory() as td:
                inst, prm = os.path.join(td, "g.rudy"), os.path.join(td, "params")
                instances.write_rudy(inst, A)
                instances.write_params(prm, _lib.PARAMS_FILE)
                env = dict(os.environ, OPENBLAS_NUM_THREADS="1")
                t0 = time.perf_counter()
                outp = subprocess.run([refbind.REF_BAB, inst, prm], capture_output=True, text=True, env=env,
                                      timeout=1800).stdout
                t_r = time.perf_counter() - t0
            mv = re.search(r"Maximum value = (\S+)", outp)
            mn = re.search(r"Nodes = (\d+)", outp)
            tto[key] = {"instance": name, "reference_serial": {
                "seconds": t_r, "optimum": float(mv.group(1)) if mv else None,
                "nodes": int(mn.group(1)) if mn else None,
                "call": "the reference's serial best-first B&B (oracle/_ref/bqb_ref_bab), 1 core, OpenBLAS 1 thread "
                        "(the instances run side by side, one core each)"}}

        # one serial process per instance, side by side on separate cores
        ths = [threading.Thread(target=ref_solve, args=c) for c in cases]
        for th in ths:
            th.start()
        for th in ths:
            th.join()
    ipm343 = None
    if args.ipm_large:   # the GPU arm's ipm_n343 case through the reference's own ipm_mc_pk
        os.environ["OPENBLAS_NUM_THREADS"] = "1"
        ref = refbind.RefLib()
        L343 = instances.root_matrix(instances.torus3d(7, 1))
        times = []
        for _ in range(2):
            t0 = time.perf_counter()
            _, phi = ref.ipm(L343)
            times.append(time.perf_counter() - t0)
        ipm343 = {"instance": "3D torus 7x7x7 (n = 343), couplings N(0,1) x 1e5 rounded, seed 1, root node",
                  "call": "the reference's ipm_mc_pk (oracle/_ref), 1 core, OpenBLAS 1 thread",
                  "ms_per_call": 1e3 * min(times), "phi": phi}
    line = {"metric": METRIC, "value": v, "unit": "nodes/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "time_to_optimality": tto, "ipm_n343": ipm343,
            "config": {"workload": WORKLOAD, "nodes_per_step": B, "processes": P,
                       "dispatch": "dynamic: one node at a time to the next idle process, steps back to back"},
            "cpu_baseline": {"value": v, "unit": "nodes/s", "cores": P, "kind": "reference",
                             "sample": f"{B} subproblems per step, {args.steps} steps, {P} processes "
                                       f"(the reference's Evaluate, OpenBLAS 1 thread each)"},
            "e2e": {"value": v, "unit": "nodes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)



# --------------------------------------------------------------------------
# small self-contained cases for kernel profiling (ncu -k ... -c ...)
# --------------------------------------------------------------------------
def run_case(args):
    """`--case ipm`: the root of a seeded G(n, 0.5) +-1 instance through
    ipm_mc_pk, `--repeats` times (above 128 vertices the multi-CTA IPM);
    `--case ipm-torus`: the same for the side^3-vertex 3D torus (`--n` is
    the side; 7 gives n = 343); `--case fused`: `--count` subproblems
    (k ~ U[0, --kmax] fixed) of a seeded G(n, 0.5) +-1 instance bounded by
    one fused-kernel launch, after the root on the engine path;
    `--case torus-root`: the 7x7x7 torus's root node on one engine;
    `--case kgon`: the pentagonal (--kgon-k 5, 3 types) or heptagonal (7, 4
    types) annealing chains on the IPM solution X of the torus root
    (`--count` chains, `--repeats` launches); `--case cert`: the FP64
    certificate of the torus root's IPM bound, `--repeats` times."""
    lib = _lib.load()
    assert lib.bqb_init(0) == 0, lib.bqb_last_error()
    if args.case in ("kgon", "cert"):
        L343 = instances.root_matrix(instances.torus3d(7, 1))
        n = L343.shape[0]
        Lc = _lib.colmajor(L343)
        X = np.zeros(n * n)
        y = np.zeros(n)
        out = np.zeros(4)
        assert lib.bqb_ipm_dual(_lib.dptr(Lc), n, _lib.dptr(X), _lib.dptr(y), _lib.dptr(out)) == 0
        for rep in range(args.repeats):
            t0 = time.perf_counter()
            if args.case == "kgon":
                k, types = (5, 3) if args.kgon_k == 5 else (7, 4)
                cost = np.zeros(args.count)
                perm = np.zeros(args.count * 7, np.int32)
                rc = lib.bqb_kgon_sa(_lib.dptr(X), n, k, types, args.count, 0x5eed + rep, _lib.dptr(cost),
                                     _lib.iptr(perm))
                print(f"kgon k={k} chains={args.count} rc={rc} best={cost.min():.6f} "
                      f"wall={1e3 * (time.perf_counter() - t0):.2f} ms", flush=True)
            else:
                c = np.zeros(4)
                assert lib.bqb_sdp_certificate(_lib.dptr(Lc), _lib.dptr(y), n, _lib.dptr(c)) == 0
                print(f"cert n={n} phi={out[0]:.6f} certified={c[0]:.6f} rel={(c[0] - out[0]) / abs(out[0]):.3e} "
                      f"shift={c[2]} wall={1e3 * (time.perf_counter() - t0):.2f} ms", flush=True)
        return
    if args.case == "torus-root":
        # the torus's root node on one engine (rank 0), batched GW rounding
        A = np.ascontiguousarray(instances.torus3d(7, 1))
        nv = A.shape[0]
        _lib.set_params(lib, _lib.make_params(**({"include_Pent": 0, "include_Hepta": 0} if args.no_kgon else {})))
        lib.process_adj_matrix(_lib.dptr(A.copy()), nv)
        lib.bqb_set_gw_hyperplanes(max(args.hyperplanes, 0))
        glob = _lib.GlobalArrays(lib, nv)
        sol = (C.c_int * _lib.NMAX)()
        C.c_void_p.in_dll(lib, "BabSol").value = C.addressof(sol)
        SP = C.cast(C.c_void_p.in_dll(lib, "SP").value, C.POINTER(_lib.Problem))
        PP = C.cast(C.c_void_p.in_dll(lib, "PP").value, C.POINTER(_lib.Problem))
        lib.bqb_set_root_effort(1 if args.root_effort else 0)
        for rep in range(args.repeats):
            seed = args.seed + rep
            nodes = (_lib.BabNode * 1)()
            b = np.zeros(1)
            lib.bqb_reset_incumbent(0.0)
            lib.bqb_bundle_iterations(1)
            lib.bqb_bound_trace_enable(1)
            t0 = time.perf_counter()
            if args.hyperplanes < 0:   # the drop-in: Evaluate on the library's default engine
                C.CDLL("libc.so.6").srand(seed)
                b[0] = lib.Evaluate(C.byref(nodes[0]), SP, PP, 0)
            else:
                assert lib.bqb_seed_engines(seed) == 0
                assert lib.bqb_bound_nodes(nodes, 1, 0, 1, None, _lib.dptr(b)) == 0, lib.bqb_last_error()
            wall = time.perf_counter() - t0
            rows = lib.bqb_bound_trace(None, 0)
            tr = np.zeros(rows * 9)
            lib.bqb_bound_trace(_lib.dptr(tr), rows)
            lib.bqb_bound_trace_enable(0)
            tr = tr.reshape(rows, 9)
            print(f"torus root seed={seed} root_effort={int(args.root_effort)} bound={b[0]:.3f} "
                  f"incumbent={lib.Bab_LBGet():.0f} wall={wall:.3f} s "
                  f"bundle_iterations={lib.bqb_bundle_iterations(1)}", flush=True)
            for r in tr:
                print(f"  round {int(r[2]):2d} bound={r[3]:.1f} incumbent={r[4]:.0f} cuts={int(r[5])}/{int(r[6])}/"
                      f"{int(r[7])} t={r[8]:.2f} s", flush=True)
        lib.bqb_set_root_effort(0)
        del glob
        return
    if args.case in ("ipm", "ipm-torus"):
        A = instances.torus3d(args.n, 1) if args.case == "ipm-torus" else instances.gnp_pm1(args.n, 0.5, seed=1)
        nv = A.shape[0]
        Lc = _lib.colmajor(instances.root_matrix(A))
        X = np.zeros(nv * nv)
        phi = C.c_double()
        lib.bqb_stats_reset()
        lib.bqb_stats_enable(1)
        if nv > 128 and args.coop_profile:
            lib.bqb_ipm_coop_profile_enable(1)
        for _ in range(args.repeats):
            t0 = time.perf_counter()
            lib.ipm_mc_pk(_lib.dptr(Lc), nv, _lib.dptr(X), C.byref(phi), 0)
            print(f"n={nv} phi={phi.value:.6f} wall={1e3 * (time.perf_counter() - t0):.3f} ms", flush=True)
            st = (C.c_double * 6)()
            lib.bqb_ipm_stats(st)
            lib.bqb_stats_reset()
            print(f"  IPM iterations {int(st[2])}, line-search trials {int(st[3])}", flush=True)
            if nv > 128 and args.coop_profile:
                pr = (C.c_double * 8)()
                lib.bqb_ipm_coop_profile(pr, 1)
                print("  parts (ms): barrier waits %.3f, panel factors %.3f, tile updates %.3f, products %.3f, "
                      "call %.3f; %d barriers, %d sweep phases; panel block loads %.3f ms" % tuple(pr[:8]),
                      flush=True)
        return
    nv, count = args.n, args.count
    A = np.ascontiguousarray(instances.gnp_pm1(nv, 0.5, seed=1))
    _lib.set_params(lib, _lib.make_params(adjust_TriIneq=0, TriIneq=TRI_PER_N * nv))
    lib.process_adj_matrix(_lib.dptr(A.copy()), nv)
    glob = _lib.GlobalArrays(lib, nv)
    sol = (C.c_int * _lib.NMAX)()
    C.c_void_p.in_dll(lib, "BabSol").value = C.addressof(sol)
    SP = C.cast(C.c_void_p.in_dll(lib, "SP").value, C.POINTER(_lib.Problem))
    PP = C.cast(C.c_void_p.in_dll(lib, "PP").value, C.POINTER(_lib.Problem))
    C.CDLL("libc.so.6").srand(2020)
    root = _lib.BabNode()
    rb = lib.Evaluate(C.byref(root), SP, PP, 0)
    nodes = (_lib.BabNode * count)()
    for q, (xf, sx) in enumerate(instances.random_fixings(nv, count, args.kmax, seed=2)):
        nodes[q].xfixed[: nv - 1] = [int(v) for v in xf]
        nodes[q].sol[: nv - 1] = [int(v) for v in sx]
    b = np.zeros(count)
    assert lib.bqb_bound_nodes_fused(nodes, count, 1, _lib.dptr(b)) == 0, lib.bqb_last_error()
    print(f"n={nv} root={rb:.6f} nodes={count} mean_bound={b.mean():.6f} "
          f"fallbacks={lib.bqb_fused_fallbacks()}", flush=True)
    del glob


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--nodes-per-step", type=int, default=512)
    ap.add_argument("--threads", type=int, default=32, help="concurrent bounding engines per GPU")
    ap.add_argument("--depth", type=int, default=8, help="fused launches in flight (1..8)")
    ap.add_argument("--no-tto", dest="tto", action="store_false",
                    help="skip the time-to-optimality run")
    ap.add_argument("--no-learned", dest="learned", action="store_false",
                    help="skip the learned warm-start comparison (two B&B runs, about 10 s)")
    ap.add_argument("--no-ipm-large", dest="ipm_large", action="store_false",
                    help="skip timing the n = 343 torus IPM (four calls, about 2 s with the first)")
    ap.add_argument("--no-tto-plain", dest="tto_plain", action="store_false",
                    help="skip the plain drop-in solver's time to optimality (about 40 s on the n = 100 "
                         "instance, 60 s on the torus)")
    ap.add_argument("--no-tto-torus", dest="tto_torus", action="store_false",
                    help="skip the time to optimality on the n = 343 torus")
    ap.add_argument("--learned-plain", action="store_true",
                    help="also time the plain drop-in solver on the learned leg's instance")
    ap.add_argument("--engine-nodes", type=int, default=128,
                    help="nodes timed through the concurrent engines (0: skip)")
    ap.add_argument("--cert-nodes", type=int, default=64,
                    help="nodes whose bounds are certified in FP64 after the timed region (0: none)")
    ap.add_argument("--dropin-nodes", type=int, default=16,
                    help="nodes timed through the serial drop-in Evaluate (0: skip)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-procs", type=int, default=64)
    ap.add_argument("--ref-nodes-per-step", type=int, default=256,
                    help="subproblems per step of the reference arm (bounded CPU sample)")
    ap.add_argument("--kgon-k", type=int, default=5, choices=[5, 7], help="--case kgon: 5 or 7")
    ap.add_argument("--case", choices=["ipm", "ipm-torus", "fused", "torus-root", "kgon", "cert"], default=None,
                    help="run one small profiling case instead of the benchmark")
    ap.add_argument("--n", type=int, default=100, help="--case: vertices (ipm-torus: the side)")
    ap.add_argument("--repeats", type=int, default=3, help="--case ipm/ipm-torus: calls")
    ap.add_argument("--count", type=int, default=16, help="--case fused: subproblems")
    ap.add_argument("--kmax", type=int, default=20, help="--case fused: most fixed vertices")
    ap.add_argument("--no-kgon", action="store_true", help="--case torus-root: no pentagonal / heptagonal cuts")
    ap.add_argument("--root-effort", action="store_true",
                    help="--case torus-root: every outer round at the root unless pruned (no early give-up)")
    ap.add_argument("--seed", type=int, default=2020,
                    help="--case torus-root: srand seed of the drop-in, or the engines' seed base (+1 per repeat)")
    ap.add_argument("--coop-profile", action="store_true", help="--case ipm/ipm-torus: time the multi-CTA IPM by parts")
    ap.add_argument("--hyperplanes", type=int, default=4096,
                    help="--case torus-root: GW hyperplanes per round on an engine (0: the reference's count; "
                         "-1: the drop-in Evaluate instead of an engine)")
    args = ap.parse_args()
    faulthandler.enable(all_threads=True)
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    if args.case:
        run_case(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
