"""The larger single-instance configuration: Max-Cut on the 7 x 7 x 7 3D
torus (n = 343, 6-regular, Gaussian couplings x 1e5 rounded to integers,
seed 1) with the reference's shipped parameters (pentagonal and heptagonal
cuts on).  Every node goes through the multi-CTA IPM (n > 128).

The B&B with 16 concurrent engines and the batched Goemans-Williamson
rounding (4096 hyperplanes per round, projected on the tensor cores)
reaches the optimum the reference's serial B&B prints for this instance
(oracle/_ref/bqb_ref_bab, recorded in tests/golden/bab_optima.json:
Maximum value = 25532237, 3 nodes); the cut it returns has that value."""
import json
import os

import pytest

from helpers import O, instances
from parallel_biqbin_maxcut_b200 import _lib

with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "bab_optima.json")) as _fh:
    TORUS_OPT = next(r for r in json.load(_fh) if r["kind"] == "torus")["max_value"]


@pytest.mark.gpu
def test_torus_bab_optimum_batched_rounding(lib):
    A = instances.torus3d(7, 1)
    r = _lib.solve(A, threads=16, gw_hyperplanes=4096)
    assert r["best_value"] == TORUS_OPT, r["best_value"]
    assert O.evaluateSolution(O.build_SP_L(A), r["x"]) == r["best_value"]
    assert r["root_bound"] >= TORUS_OPT
