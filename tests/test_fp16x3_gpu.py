"""The FP16X3 split form's power-of-two scales on inputs that span FP32's
range (GPU).

FP16 has FP32-like precision in its hi/lo pair (22 significant bits) but only
5 exponent bits, so the form scales every row of each 32-deep block of A and
every column of B by a power of two before splitting.  These tests give it
operands whose rows, columns and K blocks differ by many orders of magnitude,
values near FP32's extremes, zero blocks and non-finite entries, and require
the FP32 componentwise bound elementwise against the FP64 oracle:
|C - C64| <= 2 gamma_{K+2} (|alpha||A||B| + |beta||C0|).
"""
import numpy as np
import pytest

import hiperml_b200 as hml
import oracle
from hiperml_b200 import datagen as dg
from hiperml_b200._lib import SgemmConfig
from tests.gpu_util import gamma
from tests.test_sgemm_gpu import fetch, store

pytestmark = pytest.mark.gpu
FH = hml.ALGO_FP16X3
VAR = {16: 0, 32: 1, 64: 2, 128: 3}


def run(A, B, C0, alpha, beta, bn=64, split=1, order=0, stages=4):
    import torch
    M, K = A.shape
    N = B.shape[1]
    Ab, Ap, lda = store(A, order, 0, 0)
    Bb, Bp, ldb = store(B, order, 0, 0)
    Cb, Cp, ldc = store(C0, order, 0, 0)
    cfg = SgemmConfig(FH, 128, bn, split, stages, VAR[bn])
    hml.sgemm_ex(order, 0, 0, M, N, K, alpha, Ap, lda, Bp, ldb, beta, Cp, ldc, config=cfg)
    torch.cuda.synchronize()
    return fetch(Cb, 0, order, ldc, M, N).astype(np.float64)


def check_compwise(got, A, B, C0, alpha, beta, what):
    K = A.shape[1]
    D, absD = oracle.dgemm(A, B, C0, alpha, beta, with_abs=True)
    err = np.abs(got - D)
    bound = 2 * gamma(K + 2) * absD + 1e-45
    bad = err > bound
    assert not bad.any(), (what, int(bad.sum()), float(np.max(err / np.maximum(absD, 1e-300))))
    return D


@pytest.mark.parametrize("bn,split", [(32, 1), (64, 2), (128, 4)])
def test_rows_and_columns_spanning_fp32_range(cuda, bn, split):
    """Rows of A scaled by 10^[-15, 15], columns of B by 10^[-15, 15]: each
    element of C keeps the FP32 bound of its own magnitude."""
    rng = np.random.default_rng(1)
    M, N, K = 300, bn + 7, 500
    A = dg.matrix(M, K, 81, 0, dg.UNIFORM, order="C")
    B = dg.matrix(K, N, 81, 1, dg.UNIFORM, order="C")
    A *= (10.0 ** rng.uniform(-15, 15, (M, 1))).astype(np.float32)
    B *= (10.0 ** rng.uniform(-15, 15, (1, N))).astype(np.float32)
    C0 = dg.matrix(M, N, 81, 2, dg.UNIFORM, order="C")
    got = run(A, B, C0, 1.0, 0.0, bn=bn, split=split)
    check_compwise(got, A, B, C0, 1.0, 0.0, "row/column scales")


def test_k_blocks_of_different_magnitudes(cuda):
    """Alternate 32-deep K blocks of each row are 1e-12 and 1e+12 times the
    others: every block is scaled on its own."""
    M, N, K = 256, 40, 1024
    A = dg.matrix(M, K, 82, 0, dg.UNIFORM, order="C")
    B = dg.matrix(K, N, 82, 1, dg.UNIFORM, order="C")
    f = np.ones(K, np.float32)
    f[(np.arange(K) // 32) % 3 == 1] = 1e-12
    f[(np.arange(K) // 32) % 3 == 2] = 1e12
    A *= f[None, :]
    C0 = np.zeros((M, N), np.float32)
    got = run(A, B, C0, 1.0, 0.0, bn=64)
    check_compwise(got, A, B, C0, 1.0, 0.0, "K blocks")


def test_values_near_fp32_extremes(cuda):
    """Rows of A near 1e-35 (their scale hits its upper clamp, and the factor
    that undoes it lies below the normal range) and near 1e+18, B near 1e+3:
    every product and result stays a normal FP32 number, and keeps FP32
    accuracy."""
    M, N, K = 200, 16, 256
    A = dg.matrix(M, K, 83, 0, dg.UNIFORM, order="C")
    B = dg.matrix(K, N, 83, 1, dg.UNIFORM, order="C")
    A[: M // 2] *= np.float32(1e-35)
    A[M // 2:] *= np.float32(1e18)
    B *= np.float32(1e3)
    C0 = np.zeros((M, N), np.float32)
    got = run(A, B, C0, 1.0, 0.0, bn=16)
    D = check_compwise(got, A, B, C0, 1.0, 0.0, "extremes")
    assert np.all(got != 0.0) and np.all(np.isfinite(got))
    for rows in (slice(0, M // 2), slice(M // 2, M)):
        e = oracle.rel_errors(got[rows], D[rows])
        assert e["normwise"] <= 2e-6, (rows, e)


def test_zero_blocks_rows_and_columns(cuda):
    M, N, K = 300, 50, 320
    A = dg.matrix(M, K, 84, 0, dg.UNIFORM, order="C")
    B = dg.matrix(K, N, 84, 1, dg.UNIFORM, order="C")
    A[:, 64:128] = 0.0       # two whole K blocks
    A[17] = 0.0               # a row
    B[:, 5] = 0.0             # a column
    C0 = dg.matrix(M, N, 84, 2, dg.UNIFORM, order="C")
    got = run(A, B, C0, 2.0, -0.5, bn=64)
    check_compwise(got, A, B, C0, 2.0, -0.5, "zeros")
    np.testing.assert_array_equal(got[17], (np.float32(-0.5) * C0[17]).astype(np.float64))


def test_non_finite_inputs_give_non_finite_outputs(cuda):
    M, N, K = 256, 32, 128
    A = dg.matrix(M, K, 85, 0, dg.UNIFORM, order="C")
    B = dg.matrix(K, N, 85, 1, dg.UNIFORM, order="C")
    A[3, 40] = np.inf
    A[100, 7] = np.nan
    C0 = np.zeros((M, N), np.float32)
    got = run(A, B, C0, 1.0, 0.0, bn=32)
    assert not np.isfinite(got[3]).any() and not np.isfinite(got[100]).any()
    rest = np.ones(M, bool)
    rest[[3, 100]] = False
    assert np.isfinite(got[rest]).all()


@pytest.mark.parametrize("layout", [(0, 0, 0), (0, 1, 1), (1, 0, 0), (1, 1, 0)])
def test_loguniform_layouts_split_k(cuda, layout):
    """Log-uniform 1e-3..1e3 operands in every layout, split-K 1 and 8."""
    import torch
    order, ta, tb = layout
    M, N, K = 1000, 100, 2048
    A = dg.matrix(K if ta else M, M if ta else K, 86, 0, dg.LOGUNIFORM, order="C")
    B = dg.matrix(N if tb else K, K if tb else N, 86, 1, dg.LOGUNIFORM, order="C")
    C0 = dg.matrix(M, N, 86, 2, dg.UNIFORM, order="C")
    D, absD = oracle.dgemm(A, B, C0, 1.0, 1.0, transA=bool(ta), transB=bool(tb), with_abs=True)
    for split in (1, 8):
        Ab, Ap, lda = store(A, order, 0, 0)
        Bb, Bp, ldb = store(B, order, 0, 0)
        Cb, Cp, ldc = store(C0, order, 0, 0)
        cfg = SgemmConfig(FH, 128, 128, split, 4, VAR[128])
        hml.sgemm_ex(order, ta, tb, M, N, K, 1.0, Ap, lda, Bp, ldb, 1.0, Cp, ldc, config=cfg)
        torch.cuda.synchronize()
        got = fetch(Cb, 0, order, ldc, M, N)
        e = oracle.rel_errors(got, D, absD)
        assert e["normwise"] <= 2e-6 and e["compwise"] <= 2 * gamma(K + 2), (layout, split, e)
    assert hml.device_error() == 0
