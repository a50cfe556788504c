"""The k-means assignment oracle (CPU): the C restatement of the reference
kernel's arithmetic (oracle/hml_oracle.c oracle_kmeans_assign, after
include/hml_kmeans_kernel_template.h:19-90) against an FP64 argmin, and its
tie rule (the first of equal distances wins)."""
import numpy as np

import oracle


def test_restatement_agrees_with_fp64_away_from_ties():
    rng = np.random.default_rng(1)
    P = rng.standard_normal((4000, 12)).astype(np.float32)
    C = rng.standard_normal((37, 12)).astype(np.float32)
    a = oracle.kmeans_assign(P, C)
    d = ((P[:, None, :].astype(np.float64) - C[None].astype(np.float64)) ** 2).sum(-1)
    srt = np.sort(d, axis=1)
    clear = (srt[:, 1] - srt[:, 0]) > 1e-4 * srt[:, 1]
    assert clear.mean() > 0.99
    np.testing.assert_array_equal(a[clear], d.argmin(1)[clear])


def test_restatement_ties_take_the_first_index():
    rng = np.random.default_rng(2)
    C = rng.standard_normal((6, 5)).astype(np.float32)
    C = np.concatenate([C, C[::-1]])  # every centroid twice: indices i and 11 - i
    P = rng.standard_normal((500, 5)).astype(np.float32)
    a = oracle.kmeans_assign(P, C)
    assert a.max() < 6
    P2 = np.concatenate([P, C])  # points on the centroids themselves
    a2 = oracle.kmeans_assign(P2, C)
    np.testing.assert_array_equal(a2[500:], np.minimum(np.arange(12), 11 - np.arange(12)))
