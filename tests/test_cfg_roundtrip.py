"""The reference's v1 tuning files through the library's reader and writer
(CPU).

The rules of every shipped ``config/*.cfg`` of the reference are committed as
a fixture (``tests/golden/cfg_rules.npz``, made by
``tests/golden/make_cfg_rules.py``).  Each file is rebuilt as v1 text, loaded
with ``hml_cfg_v1_load``, written back with ``hml_cfg_v1_save`` and loaded
again.  Checked: the number of rules read, every lookup with the reference's
keying (src/hml_sgemm_kernel.cu:189-237, src/hml_sgemv_kernel.cu:315-355)
against the last-wins table of the fixture, the written rules against the
reference printers' form and order (src/hml_sgemm_kernel.cu:557-568,
src/hml_sgemv_kernel.cu:634-645), and the mapping of a loaded SGEMM rule onto
the SIMT configuration hmlSgemm runs.  With the reference tree named by
HML_REFERENCE_DIR the shipped files themselves are read as well.
"""
import ctypes
import os

import numpy as np
import pytest

import hiperml_b200 as hml
from hiperml_b200._lib import SgemmConfig, lib

HERE = os.path.dirname(os.path.abspath(__file__))
RULES = dict(np.load(os.path.join(HERE, "golden", "cfg_rules.npz")))
REF_DIR = os.environ.get("HML_REFERENCE_DIR", "")
SGEMM_FILES = sorted(k for k in RULES if k.startswith("hml_sgemm"))
SGEMV_FILES = sorted(k for k in RULES if k.startswith("hml_sgemv"))


def v1_text(name):
    rows = RULES[name]
    if name.startswith("hml_sgemm"):
        body = "".join(f"{k} {c} : {t} {r}\n" for k, c, t, r in rows)
        return "#SGEMM smart kernel config file v1.0\n#rebuilt from the fixture\n" + body
    body = "".join(f"{n} : {t} {b} {r}\n" for n, t, b, r in rows)
    return "#SGEMV smart kernel config file v1.0\n#rebuilt from the fixture\n" + body


def last_wins(name):
    table = {}
    for row in RULES[name]:
        key = tuple(int(v) for v in row[:2]) if name.startswith("hml_sgemm") else int(row[0])
        table[key] = tuple(int(v) for v in (row[2:] if name.startswith("hml_sgemm") else row[1:]))
    return table


def printed_sgemm(table):
    return [f"{K} {c} : {t} {r}" for K in range(2, 97) for c in range(1, 17)
            if (K, c) in table and table[(K, c)][1] > 0 for t, r in [table[(K, c)]]]


def printed_sgemv(table):
    return [f"{N} : {t} {b} {r}" for N in range(0, 1025)
            if N in table and table[N][2] > 0 for t, b, r in [table[N]]]


def rule_lines(path):
    with open(path) as f:
        return [ln.rstrip("\n") for ln in f if not ln.startswith("#")]


def check_sgemm_lookups(table):
    t, r = ctypes.c_int(), ctypes.c_int()
    for (K, c), (typ, rs) in table.items():
        if c > 6 or rs <= 0:
            continue  # N is clamped to 96 (6 column stops) by the keying
        assert lib.hml_cfg_v1_sgemm_rule(K, 16 * c, ctypes.byref(t), ctypes.byref(r)) == 0
        assert (t.value, r.value) == (typ, rs), (K, c)


def check_sgemv_lookups(table):
    t, b, r = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    for N, (typ, bs, rs) in table.items():
        if N == 0 or bs <= 0 or rs <= 0:
            continue
        assert lib.hml_cfg_v1_sgemv_rule(N, ctypes.byref(t), ctypes.byref(b),
                                         ctypes.byref(r)) == 0
        assert (t.value, b.value, r.value) == (typ, bs, rs), N


def roundtrip(kind, name, path, tmp_path):
    n = ctypes.c_int(-1)
    assert lib.hml_cfg_v1_load(kind, str(path).encode(), ctypes.byref(n)) == 0
    assert n.value == len(RULES[name])
    table = last_wins(name)
    (check_sgemm_lookups if kind == 0 else check_sgemv_lookups)(table)
    out = tmp_path / (name + ".out.cfg")
    assert lib.hml_cfg_v1_save(kind, str(out).encode()) == 0
    expect = printed_sgemm(table) if kind == 0 else printed_sgemv(table)
    assert rule_lines(out) == expect
    with open(out) as f:
        first = f.readline()
    assert first.startswith("#SGEMM smart kernel config file v1.0" if kind == 0
                            else "#SGEMV smart kernel config file v1.0")
    # the written file reads back to the same rules
    lib.hml_cfg_v1_clear()
    assert lib.hml_cfg_v1_load(kind, str(out).encode(), ctypes.byref(n)) == 0
    assert n.value == len(expect)
    (check_sgemm_lookups if kind == 0 else check_sgemv_lookups)(table)
    lib.hml_cfg_v1_clear()


@pytest.mark.parametrize("name", SGEMM_FILES)
def test_sgemm_cfg_roundtrip(tmp_path, name):
    src = tmp_path / (name + ".cfg")
    src.write_text(v1_text(name))
    roundtrip(0, name, src, tmp_path)


@pytest.mark.parametrize("name", SGEMV_FILES)
def test_sgemv_cfg_roundtrip(tmp_path, name):
    src = tmp_path / (name + ".cfg")
    src.write_text(v1_text(name))
    roundtrip(1, name, src, tmp_path)


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF_DIR, "config")),
                    reason="HML_REFERENCE_DIR does not name the reference tree")
@pytest.mark.parametrize("name", SGEMM_FILES + SGEMV_FILES)
def test_shipped_cfg_files_roundtrip(tmp_path, name):
    kind = 0 if name.startswith("hml_sgemm") else 1
    roundtrip(kind, name, os.path.join(REF_DIR, "config", name + ".cfg"), tmp_path)


def test_save_without_loaded_rules_is_config_error(tmp_path):
    lib.hml_cfg_v1_clear()
    assert lib.hml_cfg_v1_save(0, str(tmp_path / "x.cfg").encode()) == 5
    assert lib.hml_cfg_v1_save(1, str(tmp_path / "y.cfg").encode()) == 5


def test_loaded_sgemm_rules_map_onto_simt_tiles(tmp_path):
    """hmlSgemm runs a problem a loaded rule covers on the SIMT tile nearest
    to the rule's (16*rowStops rows, 16*colStops columns)."""
    src = tmp_path / "k40.cfg"
    src.write_text(v1_text("hml_sgemm_k40"))
    assert lib.hml_cfg_v1_load(0, str(src).encode(), None) == 0
    table = last_wins("hml_sgemm_k40")
    c = SgemmConfig()
    for (M, N, K) in ((4096, 16, 4096), (4096, 128, 4096), (1000, 40, 50), (3000, 8, 7)):
        assert lib.hml_sgemm_v1_config(M, N, K, ctypes.byref(c)) == 0, (M, N, K)
        typ, rs = table[(min(K, 96), (min(N, 96) + 15) // 16)]
        rows = 96 if typ == 0 else 16 * rs
        assert c.algo == hml.ALGO_SIMT
        assert c.tile_m == (256 if rows >= 192 else 128), (M, N, K, typ, rs, c)
        cols = 96 if typ == 0 else 16 * ((min(N, 96) + 15) // 16)
        assert c.tile_n >= min(N, cols) or c.tile_n == 128, (M, N, K, c)
        assert hml.config_check(1, 0, 0, M, N, K, K, N, N, c) == 0
    # K40 rule "96 1 : 1 8" (config/hml_sgemm_k40.cfg:583): 128 rows x 16 columns
    assert lib.hml_sgemm_v1_config(4096, 16, 4096, ctypes.byref(c)) == 0
    assert (c.tile_m, c.tile_n) == (128, 16)
    # GEMV-shaped problems (N = 1) have no tile: the GEMV kernels serve them
    assert lib.hml_sgemm_v1_config(4096, 1, 4096, ctypes.byref(c)) == 5
    lib.hml_cfg_v1_clear()
    assert lib.hml_sgemm_v1_config(4096, 16, 4096, ctypes.byref(c)) == 5
