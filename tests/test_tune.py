"""Tuned-table files and math mode (CPU only: no measurement)."""
import pytest

import hiperml_b200 as hml
from hiperml_b200._lib import lib


def _write(path, lines):
    path.write_text("#HML-B200 tuning v2\n# device test sms 148\n" + "".join(lines))


def test_v2_table_round_trip(tmp_path):
    hml.tune_clear()
    cfgs = hml.configs()
    c1 = [c for c in cfgs if c.algo == hml.ALGO_SIMT and c.tile_n == 16][0]
    c2 = [c for c in cfgs if c.algo == hml.ALGO_BF16X6 and c.tile_n == 128][0]
    f = tmp_path / "t.cfg"
    _write(f, [f"0 1 4096 16 4096 : {c1.algo} {c1.tile_m} {c1.tile_n} {c1.split_k} {c1.stages} "
               f"{c1.variant} 12.5\n",
               f"0 1 65536 128 4096 : {c2.algo} {c2.tile_m} {c2.tile_n} {c2.split_k} {c2.stages} "
               f"{c2.variant} 230.0\n"])
    assert hml.tune_load(str(f)) == 2
    assert lib.hml_tune_size() == 2
    g = tmp_path / "u.cfg"
    hml.tune_save(str(g))
    hml.tune_clear()
    assert lib.hml_tune_size() == 0
    assert hml.tune_load(str(g)) == 2
    # the exact shape now selects the tuned configuration
    assert hml.select(0, 0, 0, 4096, 16, 4096).as_tuple() == c1.as_tuple()
    # a near shape (within a factor 2) takes its neighbour's configuration
    assert hml.select(0, 0, 0, 3000, 16, 5000).as_tuple() == c1.as_tuple()
    assert hml.select(0, 0, 0, 65536, 128, 4096).as_tuple() == c2.as_tuple()
    hml.tune_clear()


def test_v2_file_through_reference_entry_point(tmp_path):
    hml.tune_clear()
    c = [c for c in hml.configs() if c.algo == hml.ALGO_SIMT][3]
    f = tmp_path / "t.cfg"
    _write(f, [f"0 1 1000 20 300 : {c.algo} {c.tile_m} {c.tile_n} {c.split_k} {c.stages} "
               f"{c.variant} 3.0\n"])
    hml.hmlSgemmKernelConfig(str(f))
    assert lib.hml_tune_size() == 1
    hml.tune_clear()


@pytest.mark.parametrize("line", [
    "0 1 100 20 300 : 1 128 16 1 4\n",                    # too few fields
    "0 1 100 200 300 : 1 128 16 1 4 0 1.0\n",             # N > M (not canonical)
    "2 1 100 20 300 : 1 128 16 1 4 0 1.0\n",              # bad layout flag
    "0 1 100 20 300 : 1 128 16 3 4 0 1.0\n",              # split 3 not in the space
    "0 1 100 20 300 : 9 128 16 1 4 0 1.0\n",              # unknown algorithm
])
def test_v2_bad_records_rejected(tmp_path, line):
    hml.tune_clear()
    f = tmp_path / "bad.cfg"
    _write(f, [line])
    with pytest.raises(hml.HmlError):
        hml.tune_load(str(f))
    assert lib.hml_tune_size() == 0


def test_v2_requires_header(tmp_path):
    f = tmp_path / "nohdr.cfg"
    f.write_text("0 1 100 20 300 : 1 128 16 1 4 0 1.0\n")
    assert lib.hml_tune_load(str(f).encode(), None) == 5


def test_math_mode_controls_automatic_choice():
    hml.tune_clear()
    try:
        assert hml.select(0, 0, 0, 65536, 128, 4096).algo == hml.ALGO_BF16X6
        hml.set_math_mode(hml.MATH_FAST)
        assert hml.select(0, 0, 0, 65536, 128, 4096).algo == hml.ALGO_BF16X3
        # skinny N stays on the SIMT kernels (HBM-bound, measured faster)
        assert hml.select(0, 0, 0, 65536, 8, 4096).algo == hml.ALGO_SIMT
        # A not addressable by TMA (odd leading dimension) -> SIMT
        c = hml.select(1, 0, 0, 65536, 128, 4095)
        assert c.algo in (hml.ALGO_SIMT, hml.ALGO_BF16X3)
    finally:
        hml.set_math_mode(hml.MATH_FP32)
    with pytest.raises(hml.HmlError):
        hml.set_math_mode(7)


SHIPPED = __import__("os").path.join(__import__("os").path.dirname(hml.__file__), "data",
                                     "tuned_b200.txt")


def test_shipped_table_parses_and_covers_the_reference_workloads():
    """The B200 tuned table shipped beside the library loads into this build's
    configuration space and holds an entry for every reference workload."""
    import os

    from hiperml_b200 import tuning_data as td
    if not os.path.exists(SHIPPED):
        pytest.skip("no shipped table")
    hml.tune_clear()
    try:
        assert hml.tune_load(SHIPPED) == len(td.TABLE_SHAPES)
        keys = set()
        for line in open(SHIPPED):
            if line.startswith("#"):
                continue
            akc, bkc, M, N, K = (int(x) for x in line.split(":")[0].split())
            keys.add((M, N, K))
        assert {(M, N, K) for (M, N, K, _ta, _tb) in td.TABLE_SHAPES} <= keys
    finally:
        hml.tune_clear()
