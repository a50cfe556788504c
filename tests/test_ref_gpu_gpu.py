"""Parity with the reference's own GPU kernels (GPU).

oracle/_ref/libhml_ref_gpu_{sgemm,sgemv}.so hold HiperML's SGEMM / SGEMV
kernel repositories and selectors compiled from its unmodified sources
(oracle/Makefile `refgpu`, texture references replaced by the stand-in of
oracle/ref_gpu_compat.h, which keeps a fetch past the bound range at 0).
With the shipped K40 rules loaded (rebuilt from tests/golden/cfg_rules.npz),
each case runs the kernel the reference would pick, on the same row-major
operands as this library's hml_sgemm_ex / hml_sgemv_ex.  Both results must
lie within the FP32 bound of the FP64 value (2 gamma_{K+2} |alpha||A||B| +
...), hence within twice it of each other, and the reference GPU result
within twice the bound of the reference CPU loop's golden output.
"""
import os

import numpy as np
import pytest

import hiperml_b200 as hml
import oracle
from hiperml_b200 import datagen as dg
from tests.golden_cases import load
from tests.gpu_util import assert_within_fp32_bound, gamma
from tests.test_cfg_roundtrip import v1_text

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_gpu_available(),
                                 reason="reference GPU libraries not built (make -C oracle refgpu)")]
META, ARR = load()


@pytest.fixture(scope="module")
def k40_rules(tmp_path_factory):
    d = tmp_path_factory.mktemp("cfg")
    sg = d / "hml_sgemm_k40.cfg"
    sg.write_text(v1_text("hml_sgemm_k40"))
    sv = d / "hml_sgemv_k40.cfg"
    sv.write_text(v1_text("hml_sgemv_k40"))
    oracle.ref_gpu_load_rules("sgemm", sg)
    oracle.ref_gpu_load_rules("sgemv", sv)
    return True


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy().astype(np.float64)


def both_sgemm(A, B, C0, alpha, beta):
    """(reference GPU kernel, this library) on row-major operands."""
    M, K = A.shape
    N = B.shape[1]
    dA, dB = dev(A), dev(B)
    c_ref, c_ours = dev(C0), dev(C0)
    oracle.ref_gpu_sgemm(c_ref.data_ptr(), dA.data_ptr(), dB.data_ptr(), M, N, K, alpha, beta)
    hml.sgemm_ex(hml.ROW_MAJOR, 0, 0, M, N, K, alpha, dA, max(1, K), dB, max(1, N), beta, c_ours,
                 max(1, N))
    return host(c_ref), host(c_ours)


@pytest.mark.parametrize("case", META["sgemm"], ids=lambda c: c["name"])
def test_sgemm_against_reference_gpu_kernel(cuda, k40_rules, case):
    M, N, K = case["M"], case["N"], case["K"]
    A = dg.matrix(M, K, case["seed"], 0, case["dist"], order="C")
    B = dg.matrix(K, N, case["seed"], 1, case["dist"], order="C")
    C0 = dg.matrix(M, N, case["seed"], 2, dg.UNIFORM, order="C")
    ref, ours = both_sgemm(A, B, C0, case["alpha"], case["beta"])
    D, absD = oracle.dgemm(A, B, C0, case["alpha"], case["beta"], with_abs=True)
    Kb = max(K, 1)
    assert_within_fp32_bound(ref, D, absD, Kb, what="reference GPU " + case["name"])
    assert_within_fp32_bound(ours, D, absD, Kb, what="ours " + case["name"])
    bound = 4 * gamma(Kb + 2) * absD + 1e-37
    assert np.all(np.abs(ours - ref) <= bound), case["name"]
    golden = ARR["sgemm_" + case["name"]].astype(np.float64)
    assert np.all(np.abs(ref - golden) <= bound), case["name"]


def test_c1_against_reference_gpu_kernel(cuda, k40_rules):
    """4096 x 16 x 4096 (the row-major copy of the column-major problem): the
    K40 rule "96 1 : 1 8" picks the var-K kernel with 8 row stops."""
    is_const, grid, block = oracle.ref_gpu_select("sgemm", 4096, 16, 4096)
    assert not is_const and block == (64, 4, 1)
    A = np.ascontiguousarray(dg.matrix(4096, 4096, 0, 0, dg.UNIFORM, order="F"))
    B = np.ascontiguousarray(dg.matrix(4096, 16, 0, 1, dg.UNIFORM, order="F"))
    C0 = np.zeros((4096, 16), np.float32)
    ref, ours = both_sgemm(A, B, C0, 1.0, 0.0)
    D, absD = oracle.dgemm(A, B, with_abs=True)
    assert_within_fp32_bound(ref, D, absD, 4096, what="reference GPU C1")
    assert_within_fp32_bound(ours, D, absD, 4096, what="ours C1")
    golden = ARR["cfg_sgemm_4096x16x4096"].astype(np.float64)
    assert np.all(np.abs(ref - golden) <= 4 * gamma(4098) * absD + 1e-37)


K40_SGEMV = {int(r[0]): tuple(int(v) for v in r[1:]) for r in
             np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                  "cfg_rules.npz"))["hml_sgemv_k40"]}


def k40_sgemv_rule(N):
    """The K40 SGEMV rule the reference applies to N (src/hml_sgemv_kernel.cu:
    323-332): (type, blockStops, rowStops); type 0 is the basic kernel."""
    return K40_SGEMV[N if N <= 1024 else 0]


@pytest.mark.parametrize("case", META["sgemv"], ids=lambda c: c["name"])
def test_sgemv_against_reference_gpu_kernel(cuda, k40_rules, case):
    """For N > 1024 the K40 rules pick the basic kernel (hmlSgemvKernelBasicN,
    include/hml_sgemv_kernel_template.h:19-106), whose last reduction steps
    read and write a shared array through a volatile pointer with no warp
    synchronisation (:88-98).  That relies on the 32 lanes of a warp running
    in lockstep, which GPUs with independent thread scheduling (Volta and
    later, B200 included) do not promise: on B200 it returns wrong sums.  For
    those cases this library is checked against FP64 and the reference's
    result is not compared (the test reports it as an expected failure of
    the reference); every other case compares both."""
    M, N = case["M"], case["N"]
    A = dg.matrix(M, N, case["seed"], 0, case["dist"], order="C")
    x = dg.fill(N, case["seed"], 1, case["dist"])
    y0 = dg.fill(M, case["seed"], 2, dg.UNIFORM)
    dA, dx = dev(A), dev(x)
    y_ref, y_ours = dev(y0), dev(y0)
    oracle.ref_gpu_sgemv(y_ref.data_ptr(), dA.data_ptr(), dx.data_ptr(), M, N, case["alpha"],
                         case["beta"])
    hml.sgemv_ex(hml.ROW_MAJOR, hml.OP_N, M, N, case["alpha"], dA, max(1, N), dx, case["beta"],
                 y_ours)
    ref, ours = host(y_ref), host(y_ours)
    D, absD = oracle.dgemm(A, x.reshape(-1, 1), y0.reshape(-1, 1), case["alpha"], case["beta"],
                           with_abs=True)
    assert_within_fp32_bound(ours, D[:, 0], absD[:, 0], max(N, 1), what="ours " + case["name"])
    bound = 4 * gamma(max(N, 1) + 2) * absD[:, 0] + 1e-37
    if k40_sgemv_rule(N)[0] == 0:
        wrong = int(np.sum(np.abs(ref - D[:, 0]) > bound))
        pytest.xfail(f"reference basic SGEMV kernel: unsynchronised warp reduction "
                     f"({wrong} of {M} results outside the FP32 bound)")
    assert_within_fp32_bound(ref, D[:, 0], absD[:, 0], max(N, 1), what="reference GPU " + case["name"])
    assert np.all(np.abs(ours - ref) <= bound), case["name"]
    golden = ARR["sgemv_" + case["name"]].astype(np.float64)
    assert np.all(np.abs(ref - golden) <= bound), case["name"]
