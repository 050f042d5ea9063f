"""B&B with the open-node pool on the device (bqb_solve_device): one
persistent launch of the fused node kernel pops, bounds, branches and pushes
nodes until the tree is closed (src/heap.c:27-133, src/bab_functions.c:
224-336 on the device).  The optimum must be the one the reference's serial
B&B printed for the same instance (tests/golden/bab_optima.json), and the
cut returned must have that value."""
import json
import os

import pytest

from helpers import O, instances
from parallel_biqbin_maxcut_b200 import _lib

HERE = os.path.dirname(os.path.abspath(__file__))


def _golden():
    with open(os.path.join(HERE, "golden", "bab_optima.json")) as fh:
        return json.load(fh)


def _adj(kind, nv, seed):
    if kind == "unit":
        return instances.gnp_unit(nv, 0.5, seed)
    if kind == "pm1":
        return instances.gnp_pm1(nv, 0.5, seed)
    if kind == "int10":
        return instances.gnp_int(nv, 0.9, 10, seed)
    return instances.qubo_to_maxcut(instances.qubo_dense(nv, 0.1, seed))


@pytest.mark.gpu
@pytest.mark.parametrize("case", [c for c in _golden() if c["nv"] <= 128], ids=lambda c: f"{c['kind']}{c['nv']}-{c['seed']}")
def test_device_pool_optimum_matches_reference(lib, case):
    A = _adj(case["kind"], case["nv"], case["seed"])
    r = _lib.solve(A, device_pool=True)
    assert r["best_value"] == case["max_value"], (r["best_value"], case)
    assert O.evaluateSolution(O.build_SP_L(A), r["x"]) == r["best_value"]
    assert r["nodes"] >= 1


@pytest.mark.gpu
def test_device_pool_matches_host_pool(lib):
    """The same instance through the host-pool fused batches: same optimum
    and the same root bound (the root is bounded the same way)."""
    A = instances.gnp_pm1(70, 0.5, 8)
    d = _lib.solve(A, device_pool=True)
    f = _lib.solve(A, fused_batch=64, fused_depth=4)
    assert d["best_value"] == f["best_value"]
    assert d["root_bound"] == f["root_bound"]


@pytest.mark.gpu
def test_device_pool_reports_a_full_pool(lib):
    """A pool too small for the tree is reported as an error, not a hang."""
    case = next(c for c in _golden() if c["kind"] == "int10" and c["nv"] == 80)
    A = _adj(case["kind"], case["nv"], case["seed"])
    with pytest.raises(RuntimeError, match="full"):
        _lib.solve(A, device_pool=True, pool_nodes=4)
