"""The per-size schedule of the multi-CTA IPM (n > 128): the autotuner picks
one of its candidate grids, and the IPM gives the oracle's result (the IPM
tests' bar: phi to 1e-6 relative, X to 1e-6) with every grid -- the same
bits with every grid, since the grid only changes which CTA owns which tile
and the sums over all entries run over a fixed partition."""
import ctypes as C

import numpy as np
import pytest

from helpers import O, instances, root_L
from parallel_biqbin_maxcut_b200 import _lib


@pytest.mark.gpu
def test_autotune_picks_a_candidate_and_every_grid_is_exact(lib):
    L = root_L(instances.gnp_pm1(200, 0.5, 31))
    n = L.shape[0]
    table = _lib.autotune_ipm([n], reps=1)
    T = (n + 31) // 32
    g = table[str(n)]["grid"]
    assert g in {T * T, (T * T + 1) // 2, (T * T + 3) // 4, (T * T + 7) // 8, 148} and table[str(n)]["ms"] > 0
    ref = O.ipm_mc_pk(L)
    first = None
    try:
        for grid in (T * T, 148, 13, 1):
            lib.bqb_ipm_schedule_set(n, grid)
            Xc = np.zeros(n * n)
            phi = C.c_double()
            lib.ipm_mc_pk(_lib.dptr(_lib.colmajor(L)), n, _lib.dptr(Xc), C.byref(phi), 0)
            assert abs(phi.value - ref.phi) <= 1e-6 * abs(ref.phi), (grid, phi.value, ref.phi)
            assert np.max(np.abs(_lib.from_colmajor(Xc, n) - ref.X)) <= 1e-6
            if first is None:
                first = (phi.value, Xc.copy())
            else:
                assert phi.value == first[0] and np.array_equal(Xc, first[1]), grid
    finally:
        lib.bqb_ipm_schedule_set(n, 0)
