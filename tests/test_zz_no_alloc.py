"""The allocation-free split-BF16 entry point (GPU).

hml_sgemm_ex_config_noalloc serves callers that must not allocate device
memory during a call: a process that reserved its whole HBM budget for its
own pool, a latency-critical path that cannot take cudaMalloc's implicit
synchronisation, a host that forbids allocation after start-up.  It keeps its
scratch -- the BF16 planes of B -- in a fixed 4 MiB array compiled into the
library instead of the workspace that hml_sgemm_ex_config grows with
cudaMalloc, and its error word in a file-scope device variable.

It runs the same kernel with the same configuration as hml_sgemm_ex_config,
so these tests call both through the C ABI and require equal results bit for
bit: two calls in a row on different problems (the second reuses the array
that still holds the first call's planes), over both operand orders of A
(column-major NN, transposed A, row-major), cluster split-K and a problem
with N > M that the library computes transposed.  They also check that a
problem too large for the array is refused before any device work and that
no bounded wait expired.

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

# (order, transA, M, N, K, tile_n, split_k, stages, seed)
CASES = [
    (hml.COL_MAJOR, hml.OP_N, 1000, 64, 4096, 64, 1, 4, 11),   # A M-contiguous
    (hml.COL_MAJOR, hml.OP_T, 700, 100, 1000, 128, 2, 4, 12),  # A K-contiguous, split-K 2
    (hml.ROW_MAJOR, hml.OP_N, 513, 40, 2000, 32, 4, 4, 13),    # row-major, split-K 4
    (hml.COL_MAJOR, hml.OP_N, 64, 1000, 1024, 64, 1, 4, 14),   # N > M: computed transposed
]


def _problem(order, transA, M, N, K, seed):
    """Dense device operands of the BLAS problem and their leading dimensions."""
    import torch
    a_rows, a_cols = (M, K) if transA == hml.OP_N else (K, M)
    A = torch.empty(M * K, device="cuda")
    B = torch.empty(K * N, device="cuda")
    C0 = torch.empty(M * N, device="cuda")
    hml.fill_random(A, seed, 0)
    hml.fill_random(B, seed, 1)
    hml.fill_random(C0, seed, 2)
    col = order == hml.COL_MAJOR
    lda = a_rows if col else a_cols
    ldb = K if col else N
    ldc = M if col else N
    return A, B, C0, lda, ldb, ldc


def _both(algo, case, alpha=1.5, beta=-0.5):
    """C = alpha*op(A)*B + beta*C0 through the allocation-free entry point and
    through hml_sgemm_ex_config; returns both results."""
    import torch
    order, ta, M, N, K, bn, split, stages, seed = case
    A, B, C0, lda, ldb, ldc = _problem(order, ta, M, N, K, seed)
    cfg = SgemmConfig(algo, 128, bn, split, stages, VAR[bn])
    stream = torch.cuda.current_stream().cuda_stream
    c_ref = C0.clone()
    st = lib.hml_sgemm_ex_config(order, ta, 0, M, N, K, alpha, A.data_ptr(), lda, B.data_ptr(),
                                 ldb, beta, c_ref.data_ptr(), ldc, ctypes.byref(cfg), stream)
    assert st == 0, lib.hml_last_error()
    c_na = C0.clone()
    st = _noalloc(order, ta, 0, M, N, K, alpha, A.data_ptr(), lda, B.data_ptr(), ldb, beta,
                  c_na.data_ptr(), ldc, ctypes.byref(cfg), stream)
    assert st == 0, lib.hml_last_error()
    torch.cuda.synchronize()
    return c_ref.cpu().numpy(), c_na.cpu().numpy()


@pytest.mark.parametrize("algo", [hml.ALGO_BF16X3, hml.ALGO_BF16X6])
def test_noalloc_equals_allocating_entry_point_bitwise(cuda, algo):
    # calls in a row on different problems: each one reuses the array that
    # still holds the previous call's planes
    for case in CASES:
        ref, got = _both(algo, case)
        assert np.isfinite(ref).all()
        assert np.array_equal(got, ref), (case, float(np.max(np.abs(got - ref))))
    assert hml.device_error() == 0


def test_noalloc_repeated_call_is_stable(cuda):
    # the same problem twice through the allocation-free entry point, with a
    # larger problem in between that overwrites more of the array
    first = _both(hml.ALGO_BF16X6, CASES[1])[1]
    _both(hml.ALGO_BF16X6, CASES[0])
    again = _both(hml.ALGO_BF16X6, CASES[1])[1]
    assert np.array_equal(first, again)
    assert hml.device_error() == 0


def test_noalloc_rejects_problems_beyond_the_scratch(cuda):
    import torch
    M, N, K = 256, 128, 8192  # BF16X6: 3 x 128 x 8192 x 2 B = 6 MiB > 4 MiB
    A, B, C0, lda, ldb, ldc = _problem(hml.COL_MAJOR, hml.OP_N, M, N, K, 13)
    cfg = SgemmConfig(hml.ALGO_BF16X6, 128, 128, 1, 4, VAR[128])
    st = _noalloc(0, 0, 0, M, N, K, 1.0, A.data_ptr(), lda, B.data_ptr(), ldb, 0.0,
                  C0.data_ptr(), ldc, ctypes.byref(cfg), torch.cuda.current_stream().cuda_stream)
    assert st == 1  # HML_STATUS_INVALID_VALUE
    assert b"4 MiB" in lib.hml_last_error()


def test_noalloc_requires_a_split_bf16_config(cuda):
    cfg = SgemmConfig(hml.ALGO_SIMT, 128, 16, 1, 3, 0)
    assert _noalloc(0, 0, 0, 64, 16, 64, 1.0, 8, 64, 8, 64, 0.0, 8, 64, ctypes.byref(cfg),
                    None) == 1
