"""SGEMM kernels against the oracle (GPU): every SIMT micro-tile, storage
order, transpose, alignment and split-K, plus the reference fixtures."""
import ctypes

import numpy as np
import pytest

import hiperml_b200 as hml
import oracle
from hiperml_b200 import datagen as dg
from hiperml_b200._lib import SgemmConfig
from tests.golden_cases import load
from tests.gpu_util import assert_within_fp32_bound, to_dev, to_host

pytestmark = pytest.mark.gpu
META, ARR = load()


def store(logical, order, pad, offset):
    """Device storage of a logical matrix in `order` with ld padded by `pad`
    and the base shifted by `offset` floats.  Returns (tensor, base, ld)."""
    import torch
    r, c = logical.shape
    if order == hml.COL_MAJOR:
        ld = max(1, r + pad)
        buf = torch.zeros(c * ld + offset + 4, dtype=torch.float32, device="cuda")
        buf[offset:offset + c * ld].view(c, ld)[:, :r].copy_(
            torch.from_numpy(np.ascontiguousarray(logical.T)))
    else:
        ld = max(1, c + pad)
        buf = torch.zeros(r * ld + offset + 4, dtype=torch.float32, device="cuda")
        buf[offset:offset + r * ld].view(r, ld)[:, :c].copy_(torch.from_numpy(logical))
    return buf, buf.data_ptr() + 4 * offset, ld


def fetch(buf, offset, order, ld, r, c):
    h = buf.cpu().numpy()[offset:]
    if order == hml.COL_MAJOR:
        return h[:c * ld].reshape(c, ld)[:, :r].T
    return h[:r * ld].reshape(r, ld)[:, :c]


def run_case(M, N, K, order, ta, tb, alpha, beta, config=None, pad=0, offset=0, seed=1,
             dist=dg.UNIFORM):
    A = dg.matrix(K if ta else M, M if ta else K, seed, 0, dist, order="C")
    B = dg.matrix(N if tb else K, K if tb else N, seed, 1, dist, order="C")
    C = dg.matrix(M, N, seed, 2, dg.UNIFORM, order="C")
    Ab, Ap, lda = store(A, order, pad, offset)
    Bb, Bp, ldb = store(B, order, pad, offset)
    Cb, Cp, ldc = store(C, order, pad, offset)
    hml.sgemm_ex(order, ta, tb, M, N, K, alpha, Ap, lda, Bp, ldb, beta, Cp, ldc, config=config)
    import torch
    torch.cuda.synchronize()
    got = fetch(Cb, offset, order, ldc, M, N)
    D, absD = oracle.dgemm(A, B, C, alpha, beta, transA=bool(ta), transB=bool(tb), with_abs=True)
    return got, D, absD


# SIMT variants from this index on are the stream-K kernel for N <= 8
# (tests/test_stream_gpu.py); the tiled kernel's shapes come first.
STREAM_VARIANT0 = 9


def simt_configs():
    out = []
    seen = set()
    for c in hml.configs():
        if c.algo != hml.ALGO_SIMT or c.variant >= STREAM_VARIANT0:
            continue
        key = (c.variant, c.split_k)
        if key in seen or c.split_k not in (1, 4) or c.stages != 3:
            continue
        seen.add(key)
        out.append(c)
    return out


SIMT = simt_configs()


@pytest.mark.parametrize("cfg", SIMT, ids=lambda c: f"v{c.variant}_s{c.split_k}")
@pytest.mark.parametrize("layout", [(0, 0, 0), (0, 1, 0), (0, 0, 1), (0, 1, 1),
                                    (1, 0, 0), (1, 1, 1)])
def test_simt_every_tile_and_layout(cuda, cfg, layout):
    order, ta, tb = layout
    M = 2 * cfg.tile_m + 37
    N = max(2, cfg.tile_n - 3)
    K = 333
    for pad in (0, 1):  # pad 1: strides not 16-byte multiples -> cp.async path
        got, D, absD = run_case(M, N, K, order, ta, tb, 0.75, -0.5, config=cfg, pad=pad)
        assert_within_fp32_bound(got, D, absD, K, what=f"{cfg} {layout} pad{pad}")


@pytest.mark.parametrize("split", [1, 2, 4, 8, 16])
def test_simt_cluster_split_k(cuda, split):
    cfg = SgemmConfig(hml.ALGO_SIMT, 128, 16, split, 4, 0)
    for K in (31, 32, 100, 1000, 4097):
        got, D, absD = run_case(300, 16, K, 0, 0, 0, 1.0, 0.0, config=cfg)
        assert_within_fp32_bound(got, D, absD, K, what=f"split{split} K{K}")


@pytest.mark.parametrize("stages", [2, 3, 4, 6])
def test_simt_pipeline_depths(cuda, stages):
    for var, (bm, bn) in ((0, (128, 16)), (4, (256, 64))):
        cfg = SgemmConfig(hml.ALGO_SIMT, bm, bn, 1, stages, var)
        if hml.config_check(0, 0, 0, 600, 50, 700, 600, 700, 600, cfg) != 0:
            assert stages == 6 and var == 4  # (256 + 64) x 128 B x 6 > 227 KB
            continue
        got, D, absD = run_case(600, 50, 700, 0, 0, 0, 1.0, 1.0, config=cfg)
        assert_within_fp32_bound(got, D, absD, 700)


@pytest.mark.parametrize("shape", [(1, 1, 1), (5, 3, 1), (1, 7, 64), (2, 2, 2), (17, 130, 9),
                                   (300, 200, 1), (64, 64, 0), (257, 1, 129), (3000, 33, 17)])
@pytest.mark.parametrize("order", [0, 1])
def test_auto_edge_shapes(cuda, shape, order):
    M, N, K = shape
    got, D, absD = run_case(M, N, K, order, 0, 0, 1.25, 0.5, offset=1)
    assert_within_fp32_bound(got, D, absD, max(K, 1), what=str(shape))


def test_beta_zero_does_not_read_c(cuda):
    import torch
    M, N, K = 500, 24, 300
    A = to_dev(np.asfortranarray(dg.matrix(M, K, 3, 0, order="C")))
    B = to_dev(np.asfortranarray(dg.matrix(K, N, 3, 1, order="C")))
    C = torch.full((N, M), float("nan"), device="cuda").t()
    hml.sgemm(A, B, C, 1.0, 0.0)
    assert torch.isfinite(C).all()


def test_alpha_zero_scales_c(cuda):
    import torch
    C = torch.ones((40, 30), device="cuda")
    A = torch.ones((40, 7), device="cuda")
    B = torch.ones((7, 30), device="cuda")
    hml.sgemm(A, B, C, 0.0, 2.5)
    assert torch.all(C == 2.5)


@pytest.mark.parametrize("case", META["sgemm"], ids=lambda c: c["name"])
def test_sgemm_matches_reference_golden(cuda, case):
    """Our SGEMM (row-major, the reference's layout) vs hmlSgemmCpu's output."""
    M, N, K = case["M"], case["N"], case["K"]
    got, D, absD = run_case(M, N, K, hml.ROW_MAJOR, 0, 0, case["alpha"], case["beta"],
                            seed=case["seed"], dist=case["dist"])
    ref = ARR["sgemm_" + case["name"]]
    assert_within_fp32_bound(got, D, absD, K, what="ours")
    assert_within_fp32_bound(ref, D, absD, K, what="reference")
    assert np.all(np.abs(got.astype(np.float64) - ref) <= 4 * (K + 2) * 2.0 ** -24 * absD + 1e-37)


def test_c1_full_size_against_reference_golden(cuda):
    """Column-major 4096 x 16 x 4096, uniform seed 0, vs the reference loop."""
    import torch
    M, N, K = 4096, 16, 4096
    A = torch.empty(M * K, dtype=torch.float32, device="cuda")
    B = torch.empty(K * N, dtype=torch.float32, device="cuda")
    hml.fill_random(A, 0, 0, dg.UNIFORM)
    hml.fill_random(B, 0, 1, dg.UNIFORM)
    C = torch.zeros(M * N, dtype=torch.float32, device="cuda")
    hml.sgemm_ex(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, C, M)
    got = C.cpu().numpy().reshape(N, M).T.astype(np.float64)
    ref = ARR["cfg_sgemm_4096x16x4096"].astype(np.float64)
    An = A.cpu().numpy().reshape(K, M).T
    Bn = B.cpu().numpy().reshape(N, K).T
    np.testing.assert_array_equal(An, dg.matrix(M, K, 0, 0, dg.UNIFORM, order="F"))
    D, absD = oracle.dgemm(An, Bn, with_abs=True)
    assert_within_fp32_bound(got, D, absD, K, what="ours")
    assert np.all(np.abs(got - ref) <= 4 * (K + 2) * 2.0 ** -24 * absD)
    err = hml.error_fp64(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, None, C, M)
    assert err[0] < 1e-6 and err[2] <= 2 * (K + 2) * 2.0 ** -24, err


@pytest.mark.parametrize("N", [8, 32, 64, 128])
def test_precision_sweep_full_size_simt(cuda, N):
    """M = 65536, K = 4096 through the SIMT path, checked in FP64 on the GPU
    (the FP32 yardstick the split-BF16 forms are compared with)."""
    import torch
    M, K = 65536, 4096
    A = torch.empty(M * K, dtype=torch.float32, device="cuda")
    B = torch.empty(K * N, dtype=torch.float32, device="cuda")
    C = torch.zeros(M * N, dtype=torch.float32, device="cuda")
    for dist in (dg.UNIFORM, dg.LOGUNIFORM):
        hml.fill_random(A, 2, 0, dist)
        hml.fill_random(B, 2, 1, dist)
        cfg = hml.select_algo(0, 0, 0, M, N, K, hml.ALGO_SIMT)
        hml.sgemm_ex(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, C, M, config=cfg)
        err = hml.error_fp64(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, None, C, M)
        assert err[2] <= 2 * (K + 2) * 2.0 ** -24, err
        # plain FP32 with a 4096-long sequential sum per thread: normwise
        # error grows like sqrt(K) u (measured 2.5e-6 .. 3.0e-6 at N = 128)
        assert err[0] < 1e-5, err


def test_no_device_error_left(cuda):
    assert hml.device_error() == 0
