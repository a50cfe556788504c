"""The C ABI boundary without a GPU: the library loads, exports every
declared symbol, validates arguments and parses tuning files."""
import ctypes
import os
import re
import subprocess

import pytest

import hiperml_b200 as hml
from hiperml_b200._lib import LIB_PATH, SgemmConfig, lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
# the reference tree, when the environment names it (the shipped .cfg files)
REF = os.environ.get("HML_REFERENCE_DIR", "")

INVALID = 1


def declared_c_functions():
    names = set()
    for fn in os.listdir(INC):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(INC, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(hml_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def exported():
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_every_declared_c_symbol_is_exported():
    decl = declared_c_functions()
    assert len(decl) >= 20
    missing = decl - exported()
    assert not missing, missing


def test_reference_cxx_symbols_are_exported():
    # the reference's six public entry points keep their C++ linkage
    want = {"_Z8hmlSgemmPfPKfS1_iiiff", "_Z13hmlSgemmBasicPfPKfS1_iiiff",
            "_Z20hmlSgemmKernelConfigPc", "_Z8hmlSgemvPfPKfS1_iiff",
            "_Z13hmlSgemvBasicPfPKfS1_iiff", "_Z20hmlSgemvKernelConfigPc"}
    assert want <= exported()


def test_status_strings_and_version():
    assert lib.hml_status_string(0) == b"success"
    assert lib.hml_status_string(6) == b"device wait timed out"
    assert b"sm_100a" in lib.hml_version()


@pytest.mark.parametrize("args", [
    (0, 0, 0, -1, 4, 4, 1.0, 8, 4, 8, 4, 0.0, 8, 4),      # negative M
    (0, 0, 0, 8, 4, 4, 1.0, 8, 7, 8, 4, 0.0, 8, 4),       # lda < M (col-major)
    (1, 0, 0, 8, 4, 4, 1.0, 8, 3, 8, 4, 0.0, 8, 4),       # lda < K (row-major)
    (0, 0, 0, 8, 4, 4, 1.0, 8, 8, 8, 3, 0.0, 8, 8),       # ldb < K
    (0, 0, 0, 8, 4, 4, 1.0, 8, 8, 8, 4, 0.0, 8, 7),       # ldc < M
    (2, 0, 0, 8, 4, 4, 1.0, 8, 8, 8, 4, 0.0, 8, 8),       # bad order
    (0, 5, 0, 8, 4, 4, 1.0, 8, 8, 8, 4, 0.0, 8, 8),       # bad op
])
def test_sgemm_argument_validation(args):
    o, ta, tb, M, N, K, al, A, lda, B, ldb, be, C, ldc = args
    st = lib.hml_sgemm_ex(o, ta, tb, M, N, K, al, A, lda, B, ldb, be, C, ldc, None)
    assert st == INVALID


def test_sgemm_null_pointers_rejected():
    assert lib.hml_sgemm_ex(0, 0, 0, 8, 4, 4, 1.0, None, 8, 8, 4, 0.0, 8, 8, None) == INVALID
    assert lib.hml_sgemm_ex(0, 0, 0, 8, 4, 4, 1.0, 8, 8, 8, 4, 0.0, None, 8, None) == INVALID


def test_empty_problems_succeed_without_device():
    assert lib.hml_sgemm_ex(0, 0, 0, 0, 4, 4, 1.0, None, 1, None, 4, 0.0, None, 1, None) == 0
    assert lib.hml_sgemv_ex(0, 0, 0, 5, 1.0, None, 1, None, 0.0, None, None) == 0


def test_sgemv_argument_validation():
    assert lib.hml_sgemv_ex(0, 0, 8, 4, 1.0, 8, 7, 8, 0.0, 8, None) == INVALID
    assert lib.hml_sgemv_ex(1, 0, 8, 4, 1.0, 8, 3, 8, 0.0, 8, None) == INVALID
    assert lib.hml_sgemv_ex(0, 2, 8, 4, 1.0, 8, 8, 8, 0.0, 8, None) == INVALID


def test_config_space_roundtrip():
    cfgs = hml.configs()
    assert len(cfgs) >= 100
    assert len({c.as_tuple() for c in cfgs}) == len(cfgs)
    for i in (0, len(cfgs) // 2, len(cfgs) - 1):
        assert lib.hml_sgemm_config_index(ctypes.byref(cfgs[i])) == i
    bad = SgemmConfig(1, 128, 16, 3, 4, 0)  # split 3 is not a power of two
    assert lib.hml_sgemm_config_index(ctypes.byref(bad)) == -1
    assert hml.config_check(0, 0, 0, 4096, 16, 4096, 4096, 4096, 4096, bad) == INVALID


def test_selection_heuristic_shapes():
    c = hml.select(0, 0, 0, 4096, 16, 4096)
    assert c.tile_n == 16 and c.split_k > 1           # skinny: split K over a cluster
    # N <= 8 with contiguous columns of A: the stream-K kernel (SIMT variants
    # from 9 on), which spreads K over all SMs by itself
    c = hml.select(0, 0, 0, 65536, 4, 4096)
    assert c.tile_n == 4 and c.variant >= 9 and c.split_k == 1
    c = hml.select(0, 0, 0, 65536, 128, 4096)
    assert c.tile_n == 128 and c.split_k == 1
    c = hml.select(0, 0, 0, 65536, 8, 4096)
    assert c.tile_n == 8
    # short-fat problems are transposed to tall-skinny
    c = hml.select(1, 0, 0, 16, 4096, 4096)
    assert c.tile_n == 16


REF_CFG = os.path.join(REF, "config")


@pytest.mark.skipif(not os.path.isdir(REF_CFG), reason="reference tree absent")
@pytest.mark.parametrize("name", ["hml_sgemm_k40.cfg", "hml_sgemm_titanblack.cfg",
                                  "hml_sgemm_gtx480.cfg", "hml_sgemm_gtx580.cfg",
                                  "hml_sgemm_header.cfg"])
def test_reference_sgemm_cfg_files_parse(name):
    n = ctypes.c_int()
    assert lib.hml_cfg_v1_load(0, os.path.join(REF_CFG, name).encode(), ctypes.byref(n)) == 0
    expect = {"hml_sgemm_k40.cfg": 570, "hml_sgemm_titanblack.cfg": 570,
              "hml_sgemm_gtx480.cfg": 1710, "hml_sgemm_gtx580.cfg": 1710,
              "hml_sgemm_header.cfg": 0}[name]
    assert n.value == expect
    lib.hml_cfg_v1_clear()


@pytest.mark.skipif(not os.path.isdir(REF_CFG), reason="reference tree absent")
def test_reference_sgemm_rule_lookup_matches_reference_keying():
    n = ctypes.c_int()
    assert lib.hml_cfg_v1_load(0, os.path.join(REF_CFG, "hml_sgemm_k40.cfg").encode(),
                               ctypes.byref(n)) == 0
    t, r = ctypes.c_int(), ctypes.c_int()
    # K > 96 uses the K = 96 row; N = 16 -> colStops 1 (config/hml_sgemm_k40.cfg:583)
    assert lib.hml_cfg_v1_sgemm_rule(4096, 16, ctypes.byref(t), ctypes.byref(r)) == 0
    assert (t.value, r.value) == (1, 8)
    # N > 96 clamps to colStops 6; "96 6 : 0 6"
    assert lib.hml_cfg_v1_sgemm_rule(4096, 128, ctypes.byref(t), ctypes.byref(r)) == 0
    assert (t.value, r.value) == (0, 6)
    assert lib.hml_cfg_v1_sgemm_rule(2, 1, ctypes.byref(t), ctypes.byref(r)) == 0
    assert (t.value, r.value) == (2, 8)
    lib.hml_cfg_v1_clear()
    assert lib.hml_cfg_v1_sgemm_rule(2, 1, ctypes.byref(t), ctypes.byref(r)) == 5


@pytest.mark.skipif(not os.path.isdir(REF_CFG), reason="reference tree absent")
@pytest.mark.parametrize("name", ["hml_sgemv_k40.cfg", "hml_sgemv_titanblack.cfg",
                                  "hml_sgemv_gtx480.cfg"])
def test_reference_sgemv_cfg_files_parse(name):
    n = ctypes.c_int()
    assert lib.hml_cfg_v1_load(1, os.path.join(REF_CFG, name).encode(), ctypes.byref(n)) == 0
    assert n.value == 1025
    t, b, r = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    # N > 1024 uses rule 0 (src/hml_sgemv_kernel.cu:330-333)
    assert lib.hml_cfg_v1_sgemv_rule(32768, ctypes.byref(t), ctypes.byref(b), ctypes.byref(r)) == 0
    assert t.value == 0 and b.value in (8, 10)
    lib.hml_cfg_v1_clear()


@pytest.mark.parametrize("line", ["97 1 : 1 8\n", "2 17 : 1 8\n", "2 1 : 3 8\n", "2 1 : 1 17\n",
                                  "2 1 : 1\n", "two 1 : 1 8\n", "2 1 : 1 8 9\n"])
def test_bad_sgemm_rules_rejected(tmp_path, line):
    f = tmp_path / "bad.cfg"
    f.write_text("#SGEMM smart kernel config file v1.0\n2 1 : 2 8\n" + line)
    n = ctypes.c_int(-1)
    assert lib.hml_cfg_v1_load(0, str(f).encode(), ctypes.byref(n)) == 5  # CONFIG_ERROR
    assert n.value == -1


@pytest.mark.parametrize("line", ["1025 : 0 8 1\n", "-1 : 0 8 1\n", "5 : 0 17 1\n", "5 : 4 8 1\n"])
def test_bad_sgemv_rules_rejected(tmp_path, line):
    f = tmp_path / "bad.cfg"
    f.write_text("#SGEMV\n0 : 0 10 1\n" + line)
    assert lib.hml_cfg_v1_load(1, str(f).encode(), None) == 5


def test_missing_cfg_file_is_io_error(tmp_path):
    assert lib.hml_cfg_v1_load(0, str(tmp_path / "nope.cfg").encode(), None) == 7
    with pytest.raises(hml.HmlError):
        hml.hmlSgemmKernelConfig(str(tmp_path / "nope.cfg"))


def test_duplicate_rules_last_wins(tmp_path):
    f = tmp_path / "dup.cfg"
    f.write_text("2 1 : 2 8\n2 1 : 1 4\n")
    assert lib.hml_cfg_v1_load(0, str(f).encode(), None) == 0
    t, r = ctypes.c_int(), ctypes.c_int()
    assert lib.hml_cfg_v1_sgemm_rule(2, 16, ctypes.byref(t), ctypes.byref(r)) == 0
    assert (t.value, r.value) == (1, 4)
    lib.hml_cfg_v1_clear()
