"""The allocation-free split-BF16 entry point (GPU).

hml_sgemm_ex_config_noalloc serves callers that must not allocate device
memory during a call (a process that reserved its whole HBM budget for its
own pool, a latency-critical path that cannot take cudaMalloc's implicit
synchronisation, a host that forbids allocation after start-up).  It keeps
its scratch -- the BF16 planes of B -- in a fixed 4 MiB array compiled into
the library instead of the workspace that hml_sgemm_ex_config grows with
cudaMalloc.  These tests call it through the C ABI twice in a row on
different problems and compare each result with hml_sgemm_ex_config's on the
same inputs, within the split-BF16 tolerances of the other tensor-core tests
(normwise 2e-6 for BF16X6, 1e-5 for BF16X3), and check that a problem too
large for the array is refused.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

import hiperml_b200 as hml
from hiperml_b200._lib import SgemmConfig, bind, lib

pytestmark = pytest.mark.gpu

_noalloc = bind("hml_sgemm_ex_config_noalloc", ctypes.c_int,
                [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                 ctypes.c_int, ctypes.c_float, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                 ctypes.c_int, ctypes.c_float, ctypes.c_void_p, ctypes.c_int,
                 ctypes.POINTER(SgemmConfig), ctypes.c_void_p])

VAR = {16: 0, 32: 1, 64: 2, 128: 3}
TOL = {hml.ALGO_BF16X3: 1e-5, hml.ALGO_BF16X6: 2e-6}


def _problem(M, N, K, seed):
    import torch
    A = torch.empty(M * K, device="cuda")
    B = torch.empty(K * N, device="cuda")
    C0 = torch.empty(M * N, device="cuda")
    hml.fill_random(A, seed, 0)
    hml.fill_random(B, seed, 1)
    hml.fill_random(C0, seed, 2)
    return A, B, C0


def _both(algo, bn, M, N, K, seed, alpha=1.5, beta=-0.5):
    """Column-major C = alpha*A*B + beta*C0 through the allocation-free entry
    point and through hml_sgemm_ex_config; returns both results."""
    import torch
    A, B, C0 = _problem(M, N, K, seed)
    cfg = SgemmConfig(algo, 128, bn, 1, 4, VAR[bn])
    stream = torch.cuda.current_stream().cuda_stream
    c_ref = C0.clone()
    st = lib.hml_sgemm_ex_config(0, 0, 0, M, N, K, alpha, A.data_ptr(), M, B.data_ptr(), K, beta,
                                 c_ref.data_ptr(), M, ctypes.byref(cfg), stream)
    assert st == 0, lib.hml_last_error()
    c_na = C0.clone()
    st = _noalloc(0, 0, 0, M, N, K, alpha, A.data_ptr(), M, B.data_ptr(), K, beta,
                  c_na.data_ptr(), M, ctypes.byref(cfg), stream)
    assert st == 0, lib.hml_last_error()
    torch.cuda.synchronize()
    return c_ref.cpu().numpy().astype(np.float64), c_na.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("algo", [hml.ALGO_BF16X3, hml.ALGO_BF16X6])
def test_noalloc_matches_allocating_entry_point_twice(cuda, algo):
    # two calls in a row on different problems: the second reuses the array
    # that still holds the first call's planes
    for (M, N, K, bn, seed) in ((1000, 64, 4096, 64, 11), (700, 100, 1000, 128, 12)):
        ref, got = _both(algo, bn, M, N, K, seed)
        rel = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
        assert rel <= TOL[algo], (M, N, K, rel)


def test_noalloc_rejects_problems_beyond_the_scratch(cuda):
    import torch
    M, N, K = 256, 128, 8192  # BF16X6: 3 x 128 x 8192 x 2 B = 6 MiB > 4 MiB
    A, B, C0 = _problem(M, N, K, 13)
    cfg = SgemmConfig(hml.ALGO_BF16X6, 128, 128, 1, 4, VAR[128])
    st = _noalloc(0, 0, 0, M, N, K, 1.0, A.data_ptr(), M, B.data_ptr(), K, 0.0, C0.data_ptr(), M,
                  ctypes.byref(cfg), torch.cuda.current_stream().cuda_stream)
    assert st == 1  # HML_STATUS_INVALID_VALUE
    assert b"4 MiB" in lib.hml_last_error()


def test_noalloc_requires_a_split_bf16_config(cuda):
    cfg = SgemmConfig(hml.ALGO_SIMT, 128, 16, 1, 3, 0)
    assert _noalloc(0, 0, 0, 64, 16, 64, 1.0, 8, 64, 8, 64, 0.0, 8, 64, ctypes.byref(cfg),
                    None) == 1
