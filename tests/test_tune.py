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
        assert hml.tune_load(SHIPPED) == len(td.TABLE_SHAPES) + len(td.GEMV_TABLE_SHAPES)
        keys = set()
        for line in open(SHIPPED):
            if line.startswith("#") or line.startswith("v "):
                continue
            akc, bkc, M, N, K = (int(x) for x in line.split(":")[0].split())
            keys.add((akc, bkc, M, N, K))
        # column-major NN: A M-contiguous, B K-contiguous; transposed (the
        # reference's row-major storage): A K-contiguous, B N-contiguous
        assert {(ta, 1 - tb, M, N, K) for (M, N, K, ta, tb) in td.TABLE_SHAPES} <= keys
        # every SGEMV shape of the reference workloads has a measured variant
        for (order, trans, M, N) in td.GEMV_TABLE_SHAPES:
            assert hml.sgemv_select(order, trans, M, N) > 0
    finally:
        hml.tune_clear()


def test_gemv_records_round_trip(tmp_path):
    """"v" records: the SGEMV half of the tuned table, keyed by layout and
    (length of y, length of x); hml_sgemv_select reports what hml_sgemv_ex
    would run."""
    hml.tune_clear()
    f = tmp_path / "v.cfg"
    _write(f, ["v 0 32768 4096 : 128 85.0\n",      # rows of A contiguous
               "v 1 32768 4096 : 8 86.5\n"])       # columns contiguous
    assert hml.tune_load(str(f)) == 2
    assert lib.hml_tune_size() == 2
    # row-major y = A x: rows contiguous; column-major: columns contiguous
    assert hml.sgemv_select(hml.ROW_MAJOR, hml.OP_N, 32768, 4096) == 128
    assert hml.sgemv_select(hml.COL_MAJOR, hml.OP_N, 32768, 4096) == 8
    # y = A^T x on a column-major 4096 x 32768 A is the rows-contiguous layout
    assert hml.sgemv_select(hml.COL_MAJOR, hml.OP_T, 4096, 32768) == 128
    # a neighbour within a factor 2 in one dimension takes its variant
    assert hml.sgemv_select(hml.ROW_MAJOR, hml.OP_N, 20000, 4096) == 128
    # further away the heuristic decides
    assert hml.sgemv_select(hml.ROW_MAJOR, hml.OP_N, 4096, 512) == 0
    g = tmp_path / "w.cfg"
    hml.tune_save(str(g))
    text = g.read_text()
    assert "v 0 32768 4096 : 128 85.000" in text and "v 1 32768 4096 : 8 86.500" in text
    hml.tune_clear()
    assert hml.sgemv_select(hml.ROW_MAJOR, hml.OP_N, 32768, 4096) == 0
    # the reference's SGEMV configuration entry point reads this format too
    hml.hmlSgemvKernelConfig(str(g))
    assert lib.hml_tune_size() == 2
    assert hml.sgemv_select(hml.COL_MAJOR, hml.OP_N, 32768, 4096) == 8
    hml.tune_clear()


@pytest.mark.parametrize("line", [
    "v 0 32768 4096 : 100 1.0\n",     # threads per row not a power of two
    "v 0 32768 4096 : 512 1.0\n",     # more than 256 threads per row
    "v 1 32768 4096 : 257 1.0\n",     # column split above 256
    "v 1 32768 4096 : 0 1.0\n",       # column split below 1
    "v 2 32768 4096 : 8 1.0\n",       # bad layout flag
    "v 0 0 4096 : 8 1.0\n",           # empty y
    "v 0 32768 4096 : 8\n",           # too few fields
])
def test_gemv_bad_records_rejected(tmp_path, line):
    hml.tune_clear()
    f = tmp_path / "bad.cfg"
    _write(f, [line])
    with pytest.raises(hml.HmlError):
        hml.tune_load(str(f))
    assert lib.hml_tune_size() == 0


def test_autotune_sgemv_rejects_bad_arguments():
    """Argument checks come before any device work."""
    for args in ((hml.ROW_MAJOR, hml.OP_N, 0, 16), (hml.ROW_MAJOR, hml.OP_N, 16, 0),
                 (7, hml.OP_N, 16, 16), (hml.ROW_MAJOR, 9, 16, 16)):
        with pytest.raises(hml.HmlError):
            hml.autotune_sgemv(*args, reps=1)
    with pytest.raises(hml.HmlError):
        hml.autotune_sgemv(hml.ROW_MAJOR, hml.OP_N, 64, 64, reps=0)
    with pytest.raises(hml.HmlError):
        hml.sgemv_select(hml.ROW_MAJOR, hml.OP_N, 64, 64, lda=10)  # lda < N


def test_sgemv_negative_variant_rejected():
    """A forced SGEMV variant is >= 0 (0 = heuristic); a negative one is an
    argument error, returned before any device work (the pointers are never
    dereferenced)."""
    with pytest.raises(hml.HmlError):
        hml.sgemv_ex(hml.ROW_MAJOR, hml.OP_N, 64, 64, 1.0, 256, 64, 512, 0.0, 768, variant=-1)
