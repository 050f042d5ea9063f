"""The tcgen05 TF32 GEMM (csrc/gw_tc.cu) that projects many Goemans-Williamson
hyperplanes at once (S = Lf V, src/heuristic.c:142-151 for one hyperplane):
D = A B^T through the C ABI against an FP64 product of the same FP32 inputs.
TF32 keeps 10 mantissa bits, so each product carries a relative error of
about 2^-11 and a sum of K of them about sqrt(K) times that: with entries in
[-1, 1] the tolerance is 2e-3 * sqrt(K) absolute (several times the expected
error)."""
import ctypes as C

import numpy as np
import pytest

from parallel_biqbin_maxcut_b200 import _lib


def _fn(lib):
    f = lib.bqb_tc_gemm_tf32
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]
    return f


def _gemm(lib, A, B):
    import torch
    M, K = A.shape
    N = B.shape[0]
    Kp = (K + 31) // 32 * 32
    Ap = np.zeros((M, Kp), np.float32)
    Bp = np.zeros((N, Kp), np.float32)
    Ap[:, :K] = A
    Bp[:, :K] = B
    dA = torch.from_numpy(Ap).cuda()
    dB = torch.from_numpy(Bp).cuda()
    dD = torch.zeros(M * N, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    rc = _fn(lib)(dA.data_ptr(), dB.data_ptr(), dD.data_ptr(), M, N, Kp)
    assert rc == 0, lib.bqb_last_error()
    return dD.cpu().numpy().reshape(N, M).T   # column-major M x N


@pytest.mark.gpu
@pytest.mark.parametrize("M,N,K", [(128, 128, 32), (343, 4096, 343), (100, 200, 64), (257, 130, 300)])
def test_tc_gemm_matches_fp64(lib, M, N, K):
    rng = np.random.default_rng(M + N + K)
    A = rng.uniform(-1, 1, (M, K)).astype(np.float32)
    B = rng.uniform(-1, 1, (N, K)).astype(np.float32)
    D = _gemm(lib, A, B)
    ref = A.astype(np.float64) @ B.astype(np.float64).T
    err = np.abs(D - ref).max()
    assert err <= 2e-3 * np.sqrt(K), err
    # a wrong operand layout or swizzle would still give numbers; make sure
    # they are the product: the error is far below the size of the entries
    assert err <= 1e-2 * np.abs(ref).max()


@pytest.mark.gpu
def test_tc_gemm_rejects_bad_pitch(lib):
    dummy = (C.c_float * 64)()
    assert _fn(lib)(C.addressof(dummy), C.addressof(dummy), C.addressof(dummy), 4, 4, 30) == 1
