"""The reference-facing host-pointer API (hmlSgemm / hmlSgemv) (GPU)."""
import os

import numpy as np
import pytest

import hiperml_b200 as hml
import oracle
from hiperml_b200 import datagen as dg
from tests.golden_cases import load
from tests.gpu_util import assert_within_fp32_bound

pytestmark = pytest.mark.gpu
META, ARR = load()


@pytest.mark.parametrize("basic", [False, True])
@pytest.mark.parametrize("case", META["sgemm"], ids=lambda c: c["name"])
def test_hmlSgemm_matches_reference_golden(cuda, case, basic):
    M, N, K = case["M"], case["N"], case["K"]
    A = dg.matrix(M, K, case["seed"], 0, case["dist"], order="C")
    B = dg.matrix(K, N, case["seed"], 1, case["dist"], order="C")
    C = dg.matrix(M, N, case["seed"], 2, dg.UNIFORM, order="C")
    D, absD = oracle.dgemm(A, B, C, case["alpha"], case["beta"], with_abs=True)
    out = C.copy()
    (hml.hmlSgemmBasic if basic else hml.hmlSgemm)(out, A, B, M, N, K, case["alpha"], case["beta"])
    assert_within_fp32_bound(out, D, absD, max(K, 1))
    ref = ARR["sgemm_" + case["name"]]
    assert np.all(np.abs(out.astype(np.float64) - ref) <= 4 * (K + 2) * 2.0 ** -24 * absD + 1e-37)


def test_hmlSgemm_large_chunked_overlap(cuda):
    """A >= 64 MiB goes through the chunked copy/compute pipeline."""
    M, N, K = 8192, 16, 2048
    A = dg.matrix(M, K, 41, 0, order="C")
    B = dg.matrix(K, N, 41, 1, order="C")
    C = np.zeros((M, N), np.float32)
    hml.hmlSgemm(C, A, B, M, N, K, 1.0, 0.0)
    D, absD = oracle.dgemm(A, B, with_abs=True)
    assert_within_fp32_bound(C, D, absD, K)


@pytest.mark.parametrize("basic", [False, True])
@pytest.mark.parametrize("case", META["sgemv"], ids=lambda c: c["name"])
def test_hmlSgemv_matches_reference_golden(cuda, case, basic):
    M, N = case["M"], case["N"]
    A = dg.matrix(M, N, case["seed"], 0, case["dist"], order="C")
    x = dg.fill(N, case["seed"], 1, case["dist"])
    y = dg.fill(M, case["seed"], 2, dg.UNIFORM)
    D, absD = oracle.dgemm(A, x.reshape(-1, 1), y.reshape(-1, 1), case["alpha"], case["beta"],
                           with_abs=True)
    out = y.copy()
    (hml.hmlSgemvBasic if basic else hml.hmlSgemv)(out, A, x, M, N, case["alpha"], case["beta"])
    assert_within_fp32_bound(out, D[:, 0], absD[:, 0], N)
    # the reference's own hmlSgemvCpu output on the same inputs: both FP32
    # results lie within the FP32 bound of the FP64 value, so within twice it
    # of each other
    ref = ARR["sgemv_" + case["name"]].astype(np.float64)
    assert np.all(np.abs(out.astype(np.float64) - ref) <= 4 * (N + 2) * 2.0 ** -24 * absD[:, 0]
                  + 1e-37)
    assert np.all(np.abs(ref - D[:, 0]) <= 2 * (N + 2) * 2.0 ** -24 * absD[:, 0] + 1e-37)


def test_errors_raise_instead_of_exit(cuda):
    with pytest.raises(ValueError):
        hml.hmlSgemm(np.zeros(4, np.float32), np.zeros(4, np.float32), np.zeros(4, np.float32),
                     4, 4, 4, 1.0, 0.0)
    with pytest.raises(hml.HmlError):
        hml.hmlSgemm(np.zeros(4, np.float32), np.zeros(4, np.float32), np.zeros(4, np.float32),
                     -1, 1, 1, 1.0, 0.0)


def test_fill_random_matches_host_generator(cuda):
    import torch
    for dist in (dg.UNIFORM, dg.NORMAL, dg.LOGUNIFORM):
        t = torch.empty(100003, dtype=torch.float32, device="cuda")
        hml.fill_random(t, 77, 3, dist)
        h = dg.fill(100003, 77, 3, dist)
        d = t.cpu().numpy()
        if dist == dg.UNIFORM:
            np.testing.assert_array_equal(d, h)
        else:
            np.testing.assert_allclose(d, h, rtol=3e-7, atol=0)
