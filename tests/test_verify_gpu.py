"""The GPU FP64 checker (hml_sgemm_error_fp64) pinned to the CPU oracle (GPU).

Every full-size accuracy figure of this repository (the precision sweep, the
square 8192^3 problem, the batched sample, the bench line's max_rel_err_fp64)
comes from the GPU checker: an FP64 GEMM over the FP32 operands and the error
reductions normwise = max|dC| / max|C64|, RMS = ||dC|| / ||C64|| and
componentwise = max |dC| / (|alpha||A||B| + |beta||C0|).  These tests compute
the same three numbers on the CPU with oracle.dgemm + oracle.rel_errors for
the same result C and require agreement to 1e-12 relative.  Both FP64 GEMMs
add exact FP32 x FP32 products in increasing k from zero and round the
alpha/beta epilogue the same way, so their FP64 values agree exactly; only the
order of the RMS sums differs.  A result with one element moved by 1e6 ulps,
and a result holding a NaN, must be flagged.
"""
import numpy as np
import pytest

import hiperml_b200 as hml
import oracle
from hiperml_b200 import datagen as dg
from tests.test_sgemm_gpu import fetch, store

pytestmark = pytest.mark.gpu

SHAPES = [(2048, 64, 1024), (1000, 130, 777), (130, 1000, 777)]
LAYOUTS = [(0, 0, 0), (0, 1, 1), (1, 0, 0), (1, 1, 0)]  # (order, transA, transB)
REL = 1e-12


def _setup(M, N, K, layout, seed, dist=dg.UNIFORM):
    order, ta, tb = layout
    A = dg.matrix(K if ta else M, M if ta else K, seed, 0, dist, order="C")
    B = dg.matrix(N if tb else K, K if tb else N, seed, 1, dist, order="C")
    C0 = dg.matrix(M, N, seed, 2, dg.UNIFORM, order="C")
    dev = {}
    dev["A"] = store(A, order, 0, 0)
    dev["B"] = store(B, order, 0, 0)
    dev["C0"] = store(C0, order, 0, 0)
    dev["C"] = store(C0, order, 0, 0)
    return A, B, C0, dev


def _gpu_errors(M, N, K, layout, alpha, beta, dev):
    order, ta, tb = layout
    _, Ap, lda = dev["A"]
    _, Bp, ldb = dev["B"]
    _, C0p, ldc = dev["C0"]
    _, Cp, _ = dev["C"]
    return hml.error_fp64(order, ta, tb, M, N, K, alpha, Ap, lda, Bp, ldb, beta, C0p, Cp, ldc)


def _close(a, b):
    return abs(a - b) <= REL * max(abs(a), abs(b), 1e-300)


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_fp64_checker_equals_cpu_oracle(cuda, shape, layout):
    import torch
    M, N, K = shape
    order, ta, tb = layout
    alpha, beta = 1.5, -0.75
    A, B, C0, dev = _setup(M, N, K, layout, seed=61)
    Cb, Cp, ldc = dev["C"]
    hml.sgemm_ex(order, ta, tb, M, N, K, alpha, dev["A"][1], dev["A"][2], dev["B"][1],
                 dev["B"][2], beta, Cp, ldc)
    torch.cuda.synchronize()
    got = fetch(Cb, 0, order, ldc, M, N)
    D, absD = oracle.dgemm(A, B, C0, alpha, beta, transA=bool(ta), transB=bool(tb),
                           with_abs=True)
    cpu = oracle.rel_errors(got, D, absD)
    gpu = _gpu_errors(M, N, K, layout, alpha, beta, dev)
    assert cpu["normwise"] > 0.0  # an FP32 result is never exact here
    assert _close(gpu[0], cpu["normwise"]), (gpu, cpu)
    assert _close(gpu[1], cpu["rms"]), (gpu, cpu)
    assert _close(gpu[2], cpu["compwise"]), (gpu, cpu)
    assert _close(gpu[3], float(np.max(np.abs(D)))), (gpu[3], np.max(np.abs(D)))

    # one element moved by 1e6 ulps: both checkers see it, and agree
    i, j = M // 3, N // 2
    bad = got.copy()
    bad[i, j] = np.float32(bad[i, j] + np.float32(1e6) * np.spacing(bad[i, j]))
    Cb.copy_(store(bad, order, 0, 0)[0])
    cpu_bad = oracle.rel_errors(bad, D, absD)
    gpu_bad = _gpu_errors(M, N, K, layout, alpha, beta, dev)
    assert gpu_bad[0] >= abs(float(bad[i, j]) - D[i, j]) / np.max(np.abs(D)) * (1 - 1e-12)
    assert gpu_bad[0] > 100 * cpu["normwise"] or gpu_bad[2] > 100 * cpu["compwise"]
    assert _close(gpu_bad[0], cpu_bad["normwise"]), (gpu_bad, cpu_bad)
    assert _close(gpu_bad[1], cpu_bad["rms"]), (gpu_bad, cpu_bad)
    assert _close(gpu_bad[2], cpu_bad["compwise"]), (gpu_bad, cpu_bad)


def test_fp64_checker_flags_nan(cuda):
    M, N, K = 300, 20, 100
    layout = (0, 0, 0)
    A, B, C0, dev = _setup(M, N, K, layout, seed=62)
    Cb, Cp, ldc = dev["C"]
    hml.sgemm_ex(0, 0, 0, M, N, K, 1.0, dev["A"][1], dev["A"][2], dev["B"][1], dev["B"][2],
                 0.0, Cp, ldc)
    Cb[7] = float("nan")
    err = _gpu_errors(M, N, K, layout, 1.0, 0.0, dev)
    assert err[0] == float("inf")


def test_fp64_checker_exact_result_reports_zero(cuda):
    # integer-valued operands whose products and sums are exact in FP32: every
    # path computes C exactly, so all three errors are exactly zero
    import torch
    M, N, K = 256, 16, 64
    rng = np.random.default_rng(5)
    A = rng.integers(-8, 9, (M, K)).astype(np.float32)
    B = rng.integers(-8, 9, (K, N)).astype(np.float32)
    Ab, Ap, lda = store(A, 0, 0, 0)
    Bb, Bp, ldb = store(B, 0, 0, 0)
    Cb, Cp, ldc = store(np.zeros((M, N), np.float32), 0, 0, 0)
    hml.sgemm_ex(0, 0, 0, M, N, K, 1.0, Ap, lda, Bp, ldb, 0.0, Cp, ldc)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(fetch(Cb, 0, 0, ldc, M, N), A.astype(np.float64) @ B)
    err = hml.error_fp64(0, 0, 0, M, N, K, 1.0, Ap, lda, Bp, ldb, 0.0, None, Cp, ldc)
    assert err[0] == 0.0 and err[1] == 0.0 and err[2] == 0.0
