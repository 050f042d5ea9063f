"""CPU: the C-ABI library loads and exports every function include/bqb_gpu.h
declares, and the reference-layout structs have the reference's sizes.  No
GPU work is launched."""
import ctypes as C
import os
import re

import pytest

from parallel_biqbin_maxcut_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "bqb_gpu.h")

pytestmark = pytest.mark.skipif(not os.path.exists(_lib.LIB_PATH), reason="library not built")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    txt = re.sub(r"^typedef\b[^;]*;", "", txt, flags=re.M | re.S)
    names = set()
    for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b([A-Za-z_]\w*)\s*\(", txt, flags=re.M):
        name = m.group(1)
        if name not in {"if", "while", "for", "return", "sizeof", "defined"}:
            names.add(name)
    return names


def test_every_declared_function_is_exported():
    lib = C.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) > 40
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_reference_globals_exported():
    lib = C.CDLL(_lib.LIB_PATH)
    for g in ("params", "SP", "PP", "X", "Z", "X_bundle", "X_test", "dual_gamma", "dgamma", "gamma_test",
              "lambda", "eta", "F", "G", "g", "f", "Cuts", "List", "Pent_Cuts", "Pent_List", "Hepta_Cuts",
              "Hepta_List", "BabPbSize"):
        assert hasattr(lib, g), g


def test_struct_layouts_match_reference():
    assert C.sizeof(_lib.TriIneq) == 32
    assert C.sizeof(_lib.PentIneq) == 40
    assert C.sizeof(_lib.HeptIneq) == 48
    assert C.sizeof(_lib.Problem) == 32
    assert C.sizeof(_lib.Params) == 88
    assert C.sizeof(_lib.BabNode) == 4 * 1024 * 2 + 8 * 1024 + 8 + 8


def test_params_reader_and_defaults(tmp_path):
    lib = C.CDLL(_lib.LIB_PATH)
    lib.bqb_read_params.argtypes = [C.c_char_p, C.POINTER(_lib.Params)]
    lib.bqb_default_params.argtypes = [C.POINTER(_lib.Params)]
    p = _lib.Params()
    lib.bqb_default_params(C.byref(p))
    for k, v in _lib.PARAM_DEFAULTS.items():
        assert getattr(p, k) == v, k
    path = tmp_path / "params"
    path.write_text("init_bundle_iter  = 5\nviolated_TriIneq  = 0.05\nTriIneq \t  = 77\n")
    assert lib.bqb_read_params(str(path).encode(), C.byref(p)) == 0
    assert (p.init_bundle_iter, p.violated_TriIneq, p.TriIneq, p.max_bundle_iter) == (5, 0.05, 77, 15)


def test_host_annealing_matches_golden():
    """The host simulated annealing (no GPU involved) against the reference
    build's output from the same rand() state."""
    import numpy as np
    G = np.load(os.path.join(ROOT, "tests", "golden", "components.npz"))
    lib = C.CDLL(_lib.LIB_PATH)
    lib.qap_simulated_annealing.restype = C.c_double
    lib.qap_simulated_annealing.argtypes = [C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_double), C.c_int,
                                           C.POINTER(C.c_int)]
    libc = C.CDLL("libc.so.6")
    libc.rand.restype = C.c_int
    X = G["sa_X"]
    n = X.shape[0]
    Xc = _lib.colmajor(X)
    H = np.ascontiguousarray(G["sa_H"], dtype=np.int32)
    p = np.zeros(5, np.int32)
    libc.srand(int(G["sa_seed"][0]))
    v = lib.qap_simulated_annealing(_lib.iptr(H), 5, _lib.dptr(Xc), n, _lib.iptr(p))
    assert v == G["sa_value"][0]
    assert np.array_equal(p, G["sa_perm"])
    assert libc.rand() == G["sa_rand_after"][0]
