"""The seeded generator shared by host and device (CPU only)."""
import numpy as np

from hiperml_b200 import datagen as dg


def test_splitmix_known_values():
    # SplitMix64 finaliser of the published algorithm on fixed inputs
    assert dg._mix_int(0) == 0
    assert dg._mix_int(0x9E3779B97F4A7C15) == 0xE220A8397B1DCDAF
    z = dg.raw64(3, 0, 0)
    key = dg.stream_key(0, 0)
    for i in range(3):
        assert int(z[i]) == dg._mix_int(key + (i + 1) * 0x9E3779B97F4A7C15)


def test_uniform_exact_and_in_range():
    v = dg.fill(100000, 3, 0, dg.UNIFORM)
    assert v.dtype == np.float32
    assert v.min() >= -1.0 and v.max() < 1.0
    assert abs(float(v.mean())) < 0.01
    # values are k * 2**-23 - 1 exactly
    k = (v.astype(np.float64) + 1.0) * 2.0 ** 23
    assert np.all(k == np.round(k))


def test_normal_moments():
    v = dg.fill(200000, 4, 1, dg.NORMAL).astype(np.float64)
    assert abs(v.mean()) < 0.01 and abs(v.std() - 1.0) < 0.01


def test_loguniform_range_and_sign():
    v = dg.fill(100000, 5, 2, dg.LOGUNIFORM).astype(np.float64)
    a = np.abs(v)
    assert a.min() >= 0.999e-3 and a.max() <= 1.001e3
    assert 0.45 < (v < 0).mean() < 0.55
    h, _ = np.histogram(np.log10(a), bins=6, range=(-3, 3))
    assert h.min() > 0.8 * h.mean()


def test_streams_and_chunking_independent():
    a = dg.fill(5000, 9, 0)
    b = dg.fill(5000, 9, 1)
    assert not np.array_equal(a, b)
    np.testing.assert_array_equal(dg.fill(5000, 9, 0, chunk=777), a)


def test_matrix_orders_are_storage_filled():
    F = dg.matrix(3, 5, 1, 0, order="F")
    C = dg.matrix(5, 3, 1, 0, order="C")
    np.testing.assert_array_equal(F, C.T)
