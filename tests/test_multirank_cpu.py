"""CPU, two ranks over gloo: the multi-GPU logic of bench.py (each rank its
own share of the subproblems, barrier, timing as the max over ranks,
whole-job throughput).  B&B nodes are independent, so there is no data-path
collective to test; these are the bench's only collectives."""
import datetime
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}",
                            timeout=datetime.timedelta(seconds=60))
    try:
        barrier, max_over_ranks = bench.make_collectives(dist, "cpu")
        barrier()
        ms = 100.0 + 50.0 * rank        # rank 1 is the slower one
        m = max_over_ranks(ms)
        batches = bench.rank_batches(rank, 16, 3, bench.N_SUB)
        q.put((rank, m, bench.aggregate_rate(16 * 3, world, m), batches))
        barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_share_work_and_time_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        rank, m, rate, batches = q.get(timeout=120)
        out[rank] = (m, rate, batches)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0] == 150.0
    assert out[0][1] == pytest.approx(2 * 48 / 0.15)
    b0, b1 = out[0][2], out[1][2]
    assert [len(b) for b in b0] == [16, 16, 16]
    assert b0 != b1 and all(0 <= i < bench.N_SUB for b in b0 + b1 for i in b)


def test_single_process_collectives_are_identity():
    barrier, max_over_ranks = bench.make_collectives(None, "cpu")
    barrier()
    assert max_over_ranks(3.5) == 3.5
    assert bench.aggregate_rate(512, 1, 1000.0) == 512.0
