"""The drop-in: the reference's own host B&B code (bab_functions.c,
bounding.c, evaluate.c, heap.c, process_input.c, allocate_free.c, compiled
unmodified) linked against libbqb_gpu.so instead of ipm_mc_pk.c, bundle.c,
operators.c, cutting_planes.c, qap_simulated_annealing.c and heuristic.c
(oracle/_ref/bqb_dropin_bab, built by `make -C oracle dropin`).  Its
"Maximum value" and "Solution" lines must equal the all-CPU reference
binary's on the same instance, as the reference's tests/test.sh compares
them."""
import os
import re
import subprocess

import pytest

from oracle import refbind
from parallel_biqbin_maxcut_b200 import _lib, instances

DROPIN = os.path.join(os.path.dirname(refbind.REF_BAB), "bqb_dropin_bab")

pytestmark = pytest.mark.skipif(not (os.path.exists(DROPIN) and os.path.exists(refbind.REF_BAB)),
                                reason="drop-in binary not built (needs the reference sources)")


def _run(binary, inst, prm):
    env = dict(os.environ, OPENBLAS_NUM_THREADS="1")
    r = subprocess.run([binary, inst, prm], capture_output=True, text=True, env=env, timeout=1200)
    assert r.returncode == 0, r.stderr[-2000:]
    keep = [ln for ln in r.stdout.splitlines() if ln.startswith(("Maximum value =", "Solution ="))]
    nodes = int(re.search(r"Nodes = (\d+)", r.stdout).group(1))
    return keep, nodes


@pytest.mark.gpu
@pytest.mark.parametrize("kind,nv,seed", [("unit", 50, 1), ("pm1", 60, 2), ("qubo", 40, 3)])
def test_dropin_matches_reference_binary(tmp_path, kind, nv, seed):
    if kind == "unit":
        A = instances.gnp_unit(nv, 0.5, seed)
    elif kind == "pm1":
        A = instances.gnp_pm1(nv, 0.5, seed)
    else:
        A = instances.qubo_to_maxcut(instances.qubo_dense(nv, 0.1, seed))
    out = {}
    for tag, binary in (("ref", refbind.REF_BAB), ("gpu", DROPIN)):
        d = tmp_path / tag
        d.mkdir()
        inst, prm = str(d / "g.rudy"), str(d / "params")
        instances.write_rudy(inst, A)
        instances.write_params(prm, _lib.PARAMS_FILE)
        out[tag] = _run(binary, inst, prm)
    assert out["gpu"][0] == out["ref"][0]
