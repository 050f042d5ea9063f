import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (B200) device")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def lib():
    """The product library; GPU tests fail loudly when it is not built."""
    from parallel_biqbin_maxcut_b200 import _lib
    L = _lib.load()
    assert L.bqb_init(0) == 0, L.bqb_last_error()
    return L


@pytest.fixture(scope="session")
def _global_arrays(lib):
    from parallel_biqbin_maxcut_b200 import _lib
    return _lib.GlobalArrays(lib, 344)


@pytest.fixture
def lib_globals(_global_arrays):
    """The product library's reference-layout globals, sized for n <= 344,
    bound for this test (a solve in an earlier test re-points them)."""
    _global_arrays.bind()
    return _global_arrays


@pytest.fixture(scope="session")
def ref():
    """The reference's own C code (oracle/_ref), globals sized for n <= 101.
    Skips when the reference build is absent."""
    from oracle import refbind
    from parallel_biqbin_maxcut_b200 import instances
    if not refbind.available():
        pytest.skip("reference build absent (oracle/Makefile)")
    r = refbind.RefLib()
    r.setup(instances.gnp_unit(101, 0.5, 99), {"init_bundle_iter": 5, "violated_TriIneq": 0.05})
    return r
