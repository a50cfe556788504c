"""Split-precision tcgen05 SGEMM (BF16X3, BF16X6, TF32X3, FP16X3) against the
FP64 oracle and the reference fixtures (GPU).

Tolerances (normwise = max|dC| / max|C64|, componentwise = max |dC| /
(|alpha||A||B| + |beta||C|)):
  BF16X6, TF32X3, FP16X3  normwise <= 2e-6 and componentwise <= 2 gamma_{K+2}
          (the FP32 bound; TF32X3's and FP16X3's hi + lo keep 22 significant
          bits of each operand, the one product they drop, lo x lo, is below
          2**-22)
  BF16X3  normwise <= 1e-5 and componentwise <= 2**-16 + 2 gamma_{K+2}
          (the two-term split keeps ~16 significant bits of each operand)
"""
import numpy as np
import pytest

import hiperml_b200 as hml
import oracle
from hiperml_b200 import datagen as dg
from hiperml_b200._lib import SgemmConfig
from tests.golden_cases import load
from tests.gpu_util import gamma
from tests.test_sgemm_gpu import fetch, store

pytestmark = pytest.mark.gpu
META, ARR = load()

X3, X6, TF, FH = hml.ALGO_BF16X3, hml.ALGO_BF16X6, hml.ALGO_TF32X3, hml.ALGO_FP16X3
FP32_LEVEL = (X6, TF, FH)
VAR = {16: 0, 32: 1, 64: 2, 128: 3}


def check_tol(algo, got, D, absD, K, what=""):
    e = oracle.rel_errors(got, D, absD)
    if algo in FP32_LEVEL:
        assert e["normwise"] <= 2e-6, (what, e)
        assert e["compwise"] <= 2 * gamma(K + 2), (what, e)
    else:
        assert e["normwise"] <= 1e-5, (what, e)
        assert e["compwise"] <= 2.0 ** -16 + 2 * gamma(K + 2), (what, e)
    return e


def run_tc(M, N, K, algo, bn, split=1, stages=4, order=0, ta=0, tb=0, alpha=1.0, beta=0.0,
           dist=dg.UNIFORM, seed=5, offset=0, tile_m=128):
    import torch
    A = dg.matrix(K if ta else M, M if ta else K, seed, 0, dist, order="C")
    B = dg.matrix(N if tb else K, K if tb else N, seed, 1, dist, order="C")
    C = dg.matrix(M, N, seed, 2, dg.UNIFORM, order="C")
    Ab, Ap, lda = store(A, order, 0, offset)
    Bb, Bp, ldb = store(B, order, 0, 0)
    Cb, Cp, ldc = store(C, order, 0, 0)
    var = VAR[bn]
    cfg = SgemmConfig(algo, tile_m, bn, split, stages, var)
    hml.sgemm_ex(order, ta, tb, M, N, K, alpha, Ap, lda, Bp, ldb, beta, Cp, ldc, config=cfg)
    torch.cuda.synchronize()
    got = fetch(Cb, 0, order, ldc, M, N)
    D, absD = oracle.dgemm(A, B, C, alpha, beta, transA=bool(ta), transB=bool(tb), with_abs=True)
    return got, D, absD


@pytest.mark.parametrize("algo", [X3, X6, TF, FH])
@pytest.mark.parametrize("bn", [16, 32, 64, 128])
@pytest.mark.parametrize("layout", [(0, 0, 0), (0, 1, 0), (0, 0, 1), (1, 0, 0), (1, 1, 1)])
def test_tc_tiles_and_layouts(cuda, algo, bn, layout):
    order, ta, tb = layout
    for (M, N, K) in ((300, max(1, bn - 5), 224), (132, bn, 96)):
        got, D, absD = run_tc(M, N, K, algo, bn, order=order, ta=ta, tb=tb, alpha=0.5, beta=-2.0)
        check_tol(algo, got, D, absD, K, what=f"{algo} {bn} {layout} {(M, N, K)}")


@pytest.mark.parametrize("algo", [X3, X6, TF, FH])
@pytest.mark.parametrize("split", [2, 4, 8, 16])
def test_tc_cluster_split_k(cuda, algo, split):
    for K in (64, 1000, 4096):
        got, D, absD = run_tc(256, 40, K, algo, 64, split=split)
        check_tol(algo, got, D, absD, K, what=f"split {split} K {K}")


@pytest.mark.parametrize("stages", [2, 4, 6, 8])
def test_tc_ring_depths(cuda, stages):
    for algo, bn in ((X3, 128), (X6, 64), (TF, 32), (TF, 128), (FH, 16), (FH, 64), (FH, 128)):
        cfg = SgemmConfig(algo, 128, bn, 1, stages, VAR[bn])
        if hml.config_check(0, 0, 0, 500, bn, 800, 500, 800, 500, cfg) != 0:
            continue
        got, D, absD = run_tc(500, bn, 800, algo, bn, stages=stages)
        check_tol(algo, got, D, absD, 800)


def test_tc_rejects_unaligned_a(cuda):
    cfg = SgemmConfig(X6, 128, 16, 1, 4, 0)
    # lda = 301 floats is not a multiple of 16 bytes: TMA cannot address A
    assert hml.config_check(0, 0, 0, 300, 16, 64, 301, 64, 300, cfg) == 2


def test_tc_beta_zero_does_not_read_c(cuda):
    import torch
    M, N, K = 384, 64, 256
    A = torch.empty(M * K, device="cuda")
    B = torch.empty(K * N, device="cuda")
    hml.fill_random(A, 9, 0)
    hml.fill_random(B, 9, 1)
    C = torch.full((M * N,), float("nan"), device="cuda")
    hml.sgemm_ex(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, C, M,
                 config=SgemmConfig(X6, 128, 64, 1, 4, 2))
    assert torch.isfinite(C).all()


@pytest.mark.parametrize("algo", [X3, X6, TF, FH])
@pytest.mark.parametrize("case", [c for c in META["sgemm"] if (c["K"] * 4) % 16 == 0],
                         ids=lambda c: c["name"])
def test_tc_matches_reference_golden(cuda, algo, case):
    """Split-BF16 (row-major, the reference's layout) vs hmlSgemmCpu's output."""
    M, N, K = case["M"], case["N"], case["K"]
    A = dg.matrix(M, K, case["seed"], 0, case["dist"], order="C")
    B = dg.matrix(K, N, case["seed"], 1, case["dist"], order="C")
    C = dg.matrix(M, N, case["seed"], 2, dg.UNIFORM, order="C")
    Ab, Ap, lda = store(A, 1, 0, 0)
    Bb, Bp, ldb = store(B, 1, 0, 0)
    Cb, Cp, ldc = store(C, 1, 0, 0)
    try:
        cfg = hml.select_algo(1, 0, 0, M, N, K, algo)
    except hml.HmlError:
        pytest.skip("operand strides not addressable by TMA (the automatic path uses SIMT)")
    hml.sgemm_ex(1, 0, 0, M, N, K, case["alpha"], Ap, lda, Bp, ldb, case["beta"], Cp, ldc,
                 config=cfg)
    import torch
    torch.cuda.synchronize()
    got = fetch(Cb, 0, 1, ldc, M, N)
    D, absD = oracle.dgemm(A, B, C, case["alpha"], case["beta"], with_abs=True)
    check_tol(algo, got, D, absD, K, what=case["name"])
    ref = ARR["sgemm_" + case["name"]].astype(np.float64)
    # ours within tolerance of FP64 and the reference within its FP32 bound
    assert np.all(np.abs(ref - D) <= 2 * gamma(K + 2) * absD + 1e-37)


@pytest.mark.parametrize("algo", [X3, X6, TF, FH])
def test_tc_c1_full_size_against_reference_golden(cuda, algo):
    import torch
    M, N, K = 4096, 16, 4096
    A = torch.empty(M * K, device="cuda")
    B = torch.empty(K * N, device="cuda")
    hml.fill_random(A, 0, 0, dg.UNIFORM)
    hml.fill_random(B, 0, 1, dg.UNIFORM)
    C = torch.zeros(M * N, device="cuda")
    cfg = hml.select_algo(0, 0, 0, M, N, K, algo)
    hml.sgemm_ex(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, C, M, config=cfg)
    got = C.cpu().numpy().reshape(N, M).T.astype(np.float64)
    An = A.cpu().numpy().reshape(K, M).T
    Bn = B.cpu().numpy().reshape(N, K).T
    D, absD = oracle.dgemm(An, Bn, with_abs=True)
    check_tol(algo, got, D, absD, K, what="C1")
    ref = ARR["cfg_sgemm_4096x16x4096"].astype(np.float64)
    tol = 2e-6 if algo in FP32_LEVEL else 1e-5
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) <= tol + 4 * 2.0 ** -24 * 64


@pytest.mark.parametrize("algo", [X3, X6, TF, FH])
@pytest.mark.parametrize("N", [8, 32, 64, 128])
def test_tc_precision_sweep_full_size(cuda, algo, N):
    """M = 65536, K = 4096, uniform and log-uniform (1e-3..1e3) inputs,
    checked in FP64 on the GPU."""
    import torch
    M, K = 65536, 4096
    A = torch.empty(M * K, device="cuda")
    B = torch.empty(K * N, device="cuda")
    C = torch.zeros(M * N, device="cuda")
    cfg = hml.select_algo(0, 0, 0, M, N, K, algo)
    for dist in (dg.UNIFORM, dg.LOGUNIFORM):
        hml.fill_random(A, 2, 0, dist)
        hml.fill_random(B, 2, 1, dist)
        hml.sgemm_ex(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, C, M, config=cfg)
        err = hml.error_fp64(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, None, C, M)
        if algo in FP32_LEVEL:
            assert err[0] <= 2e-6 and err[2] <= 2 * gamma(K + 2), err
        else:
            assert err[0] <= 1e-5, err


@pytest.mark.parametrize("dist", [dg.UNIFORM, dg.LOGUNIFORM], ids=["uniform", "loguniform"])
def test_tc_square_8192_full_size(cuda, dist):
    """The precision sweep's square problem, 8192^3, uniform[-1,1] and
    log-uniform (1e-3..1e3, random sign) inputs: the library's automatic
    choice and forced BF16X6, checked in FP64 on the GPU."""
    import torch
    M = N = K = 8192
    A = torch.empty(M * K, device="cuda")
    B = torch.empty(K * N, device="cuda")
    C = torch.zeros(M * N, device="cuda")
    hml.fill_random(A, 4, 0, dist)
    hml.fill_random(B, 4, 1, dist)
    for cfg in (None, hml.select_algo(0, 0, 0, M, N, K, X6), hml.select_algo(0, 0, 0, M, N, K, FH)):
        C.zero_()
        hml.sgemm_ex(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, C, M, config=cfg)
        err = hml.error_fp64(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, None, C, M)
        assert err[0] <= 2e-6 and err[2] <= 2 * gamma(K + 2), (cfg, err)
        assert err[0] > 0.0


def test_no_device_error_left(cuda):
    assert hml.device_error() == 0


def test_tc_tiles_are_128_rows(cuda):
    """Only 128-row tiles exist: a 256-row configuration is refused."""
    assert all(c.tile_m == 128 for c in hml.configs() if c.algo in (X3, X6))
    for algo in (X3, X6, TF):
        assert hml.config_check(0, 0, 0, 512, 64, 256, 512, 256, 512,
                                SgemmConfig(algo, 256, 64, 1, 4, VAR[64])) == 1


def test_tf32x3_explicit_only(cuda):
    """TF32X3 is an explicit configuration: outside the autotuner's space."""
    assert all(c.algo != TF for c in hml.configs())
    assert hml.config_check(0, 0, 0, 4096, 64, 4096, 4096, 4096, 4096,
                            SgemmConfig(TF, 128, 64, 1, 4, VAR[64])) == 0
