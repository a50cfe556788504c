"""The CPU oracle, pinned against the reference (CPU only)."""
import numpy as np
import pytest

import oracle
from hiperml_b200 import datagen as dg
from tests.golden_cases import load

META, ARR = load()
U = 2.0 ** -24


def _sgemm_inputs(c):
    A = dg.matrix(c["M"], c["K"], c["seed"], 0, c["dist"], order="C")
    B = dg.matrix(c["K"], c["N"], c["seed"], 1, c["dist"], order="C")
    C = dg.matrix(c["M"], c["N"], c["seed"], 2, dg.UNIFORM, order="C")
    return A, B, C


def _sgemv_inputs(c):
    A = dg.matrix(c["M"], c["N"], c["seed"], 0, c["dist"], order="C")
    x = dg.fill(c["N"], c["seed"], 1, c["dist"])
    y = dg.fill(c["M"], c["seed"], 2, dg.UNIFORM)
    return A, x, y


@pytest.mark.parametrize("case", META["sgemm"], ids=lambda c: c["name"])
def test_restatement_matches_reference_sgemm_golden(case):
    """hml_oracle.c reproduces hmlSgemmCpu bit for bit on every fixture."""
    A, B, C = _sgemm_inputs(case)
    out = oracle.sgemm_rm_f32(A, B, C, case["alpha"], case["beta"])
    np.testing.assert_array_equal(out, ARR["sgemm_" + case["name"]])
    assert oracle.csum(out) == case["csum"]


@pytest.mark.parametrize("case", META["sgemv"], ids=lambda c: c["name"])
def test_restatement_matches_reference_sgemv_golden(case):
    A, x, y = _sgemv_inputs(case)
    out = oracle.sgemv_rm_f32(A, x, y, case["alpha"], case["beta"])
    np.testing.assert_array_equal(out, ARR["sgemv_" + case["name"]])
    assert oracle.csum(out) == case["csum"]


def test_restatement_matches_reference_c1_golden():
    """The column-major 4096 x 16 x 4096 workload through its exact row-major copy."""
    c = [x for x in META["configs"] if x["name"] == "sgemm_4096x16x4096"][0]
    A = dg.matrix(4096, 4096, 0, 0, dg.UNIFORM, order="F")
    B = dg.matrix(4096, 16, 0, 1, dg.UNIFORM, order="F")
    out = oracle.sgemm_rm_f32(np.ascontiguousarray(A), np.ascontiguousarray(B), threads=8)
    np.testing.assert_array_equal(out, ARR["cfg_sgemm_4096x16x4096"])
    assert oracle.csum(out) == c["csum"]


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
def test_restatement_matches_reference_loops_live():
    rng = np.random.default_rng(5)
    for (M, N, K) in [(33, 17, 65), (2, 97, 3), (64, 1, 200)]:
        A = rng.standard_normal((M, K)).astype(np.float32)
        B = rng.standard_normal((K, N)).astype(np.float32)
        C = rng.standard_normal((M, N)).astype(np.float32)
        np.testing.assert_array_equal(oracle.sgemm_rm_f32(A, B, C, -0.5, 3.0),
                                      oracle.ref_sgemm_cpu(A, B, C, -0.5, 3.0))
        x = rng.standard_normal(K).astype(np.float32)
        y = rng.standard_normal(M).astype(np.float32)
        np.testing.assert_array_equal(oracle.sgemv_rm_f32(A, x, y, 1.25, -1.0),
                                      oracle.ref_sgemv_cpu(A, x, y, 1.25, -1.0))


@pytest.mark.parametrize("tA,tB", [(False, False), (True, False), (False, True), (True, True)])
def test_fp64_oracle_against_numpy(tA, tB):
    rng = np.random.default_rng(7)
    M, N, K = 45, 13, 77
    A = rng.standard_normal((K, M) if tA else (M, K)).astype(np.float32)
    B = rng.standard_normal((N, K) if tB else (K, N)).astype(np.float32)
    C = rng.standard_normal((M, N)).astype(np.float32)
    for Aa in (A, np.asfortranarray(A)):
        D, absD = oracle.dgemm(Aa, B, C, 1.5, -0.5, transA=tA, transB=tB, with_abs=True)
        opA = A.astype(np.float64).T if tA else A.astype(np.float64)
        opB = B.astype(np.float64).T if tB else B.astype(np.float64)
        ref = 1.5 * opA @ opB - 0.5 * C.astype(np.float64)
        np.testing.assert_allclose(D, ref, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(absD, 1.5 * np.abs(opA) @ np.abs(opB) + 0.5 * np.abs(C),
                                   rtol=1e-12)


def test_fp32_loop_within_classical_bound():
    """The reference loop's error obeys |dC| <= gamma_K |A||B| (Higham 3.5)."""
    c = META["sgemm"][2]
    A, B, C = _sgemm_inputs(c)
    out = ARR["sgemm_" + c["name"]]
    D, absD = oracle.dgemm(A, B, C, c["alpha"], c["beta"], with_abs=True)
    K = c["K"]
    gamma = (K + 2) * U / (1 - (K + 2) * U)
    assert np.all(np.abs(out - D) <= gamma * absD + 1e-30)


def test_rel_errors_metric():
    exact = np.array([[1.0, -2.0], [4.0, 0.5]])
    approx = exact + np.array([[0.0, 0.01], [0.0, 0.0]])
    e = oracle.rel_errors(approx, exact)
    assert e["normwise"] == pytest.approx(0.01 / 4.0)
