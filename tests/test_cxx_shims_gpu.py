"""The reference's six C++ entry points, called by their mangled names (GPU).

A program written against the reference's ``include/hml_sgemm.h`` /
``include/hml_sgemv.h`` links these symbols; they are called here exactly as
such a program calls them (host pointers, row-major, C++ linkage), on the
golden cases whose outputs the reference's own CPU loops produced.  Each
result must lie within the FP32 bound of the FP64 value, and within twice it
of the reference output.  ``hmlSgemmKernelConfig`` / ``hmlSgemvKernelConfig``
load a shipped K40 tuning file (rebuilt from the fixture of its rules); the
calls after it run with the rules mapped onto this library's kernels.
"""
import ctypes
import os

import numpy as np
import pytest

import oracle
from hiperml_b200 import datagen as dg
from hiperml_b200._lib import LIB_PATH, SgemmConfig, lib
from tests.golden_cases import load
from tests.gpu_util import assert_within_fp32_bound
from tests.test_cfg_roundtrip import v1_text

pytestmark = pytest.mark.gpu
META, ARR = load()

_so = ctypes.CDLL(LIB_PATH)
_fp = ctypes.POINTER(ctypes.c_float)
_i, _f = ctypes.c_int, ctypes.c_float


def _sym(name, args):
    f = getattr(_so, name)
    f.restype = None
    f.argtypes = args
    return f


hmlSgemm = _sym("_Z8hmlSgemmPfPKfS1_iiiff", [_fp, _fp, _fp, _i, _i, _i, _f, _f])
hmlSgemmBasic = _sym("_Z13hmlSgemmBasicPfPKfS1_iiiff", [_fp, _fp, _fp, _i, _i, _i, _f, _f])
hmlSgemmKernelConfig = _sym("_Z20hmlSgemmKernelConfigPc", [ctypes.c_char_p])
hmlSgemv = _sym("_Z8hmlSgemvPfPKfS1_iiff", [_fp, _fp, _fp, _i, _i, _f, _f])
hmlSgemvBasic = _sym("_Z13hmlSgemvBasicPfPKfS1_iiff", [_fp, _fp, _fp, _i, _i, _f, _f])
hmlSgemvKernelConfig = _sym("_Z20hmlSgemvKernelConfigPc", [ctypes.c_char_p])


def p(a):
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_fp)


def _sgemm_case(fn, case):
    M, N, K = case["M"], case["N"], case["K"]
    A = dg.matrix(M, K, case["seed"], 0, case["dist"], order="C")
    B = dg.matrix(K, N, case["seed"], 1, case["dist"], order="C")
    C = dg.matrix(M, N, case["seed"], 2, dg.UNIFORM, order="C")
    out = C.copy()
    fn(p(out), p(A), p(B), M, N, K, case["alpha"], case["beta"])
    D, absD = oracle.dgemm(A, B, C, case["alpha"], case["beta"], with_abs=True)
    assert_within_fp32_bound(out, D, absD, max(K, 1), what=case["name"])
    ref = ARR["sgemm_" + case["name"]].astype(np.float64)
    assert np.all(np.abs(out.astype(np.float64) - ref) <= 4 * (K + 2) * 2.0 ** -24 * absD
                  + 1e-37), case["name"]


def _sgemv_case(fn, case):
    M, N = case["M"], case["N"]
    A = dg.matrix(M, N, case["seed"], 0, case["dist"], order="C")
    x = dg.fill(N, case["seed"], 1, case["dist"])
    y = dg.fill(M, case["seed"], 2, dg.UNIFORM)
    out = y.copy()
    fn(p(out), p(A), p(x), M, N, case["alpha"], case["beta"])
    D, absD = oracle.dgemm(A, x.reshape(-1, 1), y.reshape(-1, 1), case["alpha"], case["beta"],
                           with_abs=True)
    assert_within_fp32_bound(out, D[:, 0], absD[:, 0], N, what=case["name"])
    ref = ARR["sgemv_" + case["name"]].astype(np.float64)
    assert np.all(np.abs(out.astype(np.float64) - ref) <= 4 * (N + 2) * 2.0 ** -24 * absD[:, 0]
                  + 1e-37), case["name"]


@pytest.mark.parametrize("fn", [hmlSgemm, hmlSgemmBasic], ids=["hmlSgemm", "hmlSgemmBasic"])
def test_cxx_sgemm_symbols_on_golden_cases(cuda, fn):
    lib.hml_cfg_v1_clear()
    for case in META["sgemm"]:
        _sgemm_case(fn, case)


@pytest.mark.parametrize("fn", [hmlSgemv, hmlSgemvBasic], ids=["hmlSgemv", "hmlSgemvBasic"])
def test_cxx_sgemv_symbols_on_golden_cases(cuda, fn):
    lib.hml_cfg_v1_clear()
    for case in META["sgemv"]:
        _sgemv_case(fn, case)


def test_cxx_kernel_config_with_shipped_k40_files(cuda, tmp_path):
    sg = tmp_path / "hml_sgemm_k40.cfg"
    sg.write_text(v1_text("hml_sgemm_k40"))
    sv = tmp_path / "hml_sgemv_k40.cfg"
    sv.write_text(v1_text("hml_sgemv_k40"))
    try:
        hmlSgemmKernelConfig(str(sg).encode())
        hmlSgemvKernelConfig(str(sv).encode())
        # the rules are in force: the golden shapes map onto SIMT tiles
        c = SgemmConfig()
        ruled = 0
        for case in META["sgemm"]:
            if lib.hml_sgemm_v1_config(case["M"], case["N"], case["K"], ctypes.byref(c)) == 0:
                ruled += 1
            _sgemm_case(hmlSgemm, case)
        assert ruled >= 5
        for case in META["sgemv"]:
            _sgemv_case(hmlSgemv, case)
        # C1 through the K40 rule "96 1 : 1 8": row-major copy of the
        # column-major 4096 x 16 x 4096 problem, against the reference output
        A = np.ascontiguousarray(dg.matrix(4096, 4096, 0, 0, dg.UNIFORM, order="F"))
        B = np.ascontiguousarray(dg.matrix(4096, 16, 0, 1, dg.UNIFORM, order="F"))
        C = np.zeros((4096, 16), np.float32)
        hmlSgemm(p(C), p(A), p(B), 4096, 16, 4096, 1.0, 0.0)
        ref = ARR["cfg_sgemm_4096x16x4096"].astype(np.float64)
        D, absD = oracle.dgemm(A, B, with_abs=True)
        assert_within_fp32_bound(C, D, absD, 4096, what="C1 with K40 rules")
        assert np.all(np.abs(C - ref) <= 4 * 4098 * 2.0 ** -24 * absD + 1e-37)
    finally:
        lib.hml_cfg_v1_clear()
