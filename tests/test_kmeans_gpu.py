"""The k-means assignment step on the skinny SGEMM (GPU).

hml_kmeans_assign computes argmin_k ||c_k||^2 - 2 x.c_k from one GEMM -- in
the tiled form (a register-tiled SIMT GEMM with the argmin in its epilogue),
the SGEMM form (the products through HBM, then a pick kernel) or the
tensor-core form (TF32X3 products in TMEM, the argmin read from the
accumulator) -- and
resolves every close call with the reference kernel's own arithmetic, so
either form's indices must equal, bit for bit, those of
  * the C restatement of the reference kernel (oracle.kmeans_assign), and
  * the reference's own GPU kernel hmlKmeansAssignCtrdSmem
    (include/hml_kmeans_kernel_template.h:19-90, built into oracle/_ref),
on random data, on data built to be close to ties (centroid pairs a few ulps
apart, duplicated centroids, points on the perpendicular bisector), on points
far from the origin (where ||x||^2 - 2 x.c cancels) and on a large case.
"""
import numpy as np
import pytest

import hiperml_b200 as hml
import oracle

pytestmark = pytest.mark.gpu


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


METHODS = [hml.KMEANS_TILED, hml.KMEANS_GEMM, hml.KMEANS_TENSOR]


def tensor_applies(d, k):
    return d >= 4 and d % 4 == 0 and d <= 64 and k <= 256


def skip_unless_applies(method, d, k):
    """The tensor-core form refuses shapes outside its range (checked here)."""
    if method == hml.KMEANS_TENSOR and not tensor_applies(d, k):
        with pytest.raises(hml.HmlError):
            hml.kmeans_assign(dev(np.zeros((4, d), np.float32)), dev(np.zeros((k, d), np.float32)),
                              method=method)
        pytest.skip("outside the tensor-core form's range (refusal checked)")


def ours(P, C, method=hml.KMEANS_AUTO):
    out, exact = hml.kmeans_assign(dev(P), dev(C), count_exact=True, method=method)
    return out.cpu().numpy().astype(np.uint32), exact


def clustered(rng, n, d, k, spread=0.3):
    C = rng.standard_normal((k, d)).astype(np.float32)
    lab = rng.integers(0, k, n)
    P = (C[lab] + spread * rng.standard_normal((n, d))).astype(np.float32)
    return P, C


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("d", [1, 3, 8, 16, 31, 32, 33, 64, 100, 300])
@pytest.mark.parametrize("k", [1, 2, 16, 64, 65, 130])
def test_matches_reference_arithmetic(cuda, method, d, k):
    """Dimensions around the tiled form's 32-wide stages, centroid counts
    around its 64-wide passes, point counts not a multiple of its 128-point
    blocks."""
    skip_unless_applies(method, d, k)
    rng = np.random.default_rng(d * 1000 + k)
    P, C = clustered(rng, 3001, d, k)
    got, _ = ours(P, C, method)
    np.testing.assert_array_equal(got, oracle.kmeans_assign(P, C))


def test_automatic_choice_and_edge_cases(cuda):
    import torch
    rng = np.random.default_rng(3)
    for d in (16, 256, 257, 500):
        P, C = clustered(rng, 700, d, 20)
        got, _ = ours(P, C)
        np.testing.assert_array_equal(got, oracle.kmeans_assign(P, C))
    # zero dimensions: every distance is 0, the first centroid wins
    for method in METHODS[:2]:
        out = hml.kmeans_assign(torch.zeros((50, 0), device="cuda"),
                                torch.zeros((7, 0), device="cuda"), method=method)
        assert int(out.abs().sum()) == 0
    # one point; no points
    P, C = clustered(rng, 1, 8, 9)
    for method in METHODS:
        np.testing.assert_array_equal(ours(P, C, method)[0], oracle.kmeans_assign(P, C))
        assert hml.kmeans_assign(torch.zeros((0, 8), device="cuda"), dev(C),
                                 method=method).numel() == 0
    with pytest.raises(hml.HmlError):
        hml.kmeans_assign(dev(P), dev(C), method=4)
    # the tensor-core form: 257 centroids, 68 dimensions, unaligned rows
    for shape in ((10, 8, 257), (10, 68, 9), (10, 6, 9)):
        with pytest.raises(hml.HmlError):
            hml.kmeans_assign(dev(np.zeros(shape[:2], np.float32)),
                              dev(np.zeros(shape[2:] + shape[1:2], np.float32)),
                              method=hml.KMEANS_TENSOR)
    import torch
    buf = torch.zeros(1 + 100 * 8, device="cuda")
    with pytest.raises(hml.HmlError):
        hml.kmeans_assign(buf[1:].view(100, 8), dev(np.zeros((9, 8), np.float32)),
                          method=hml.KMEANS_TENSOR)


@pytest.mark.parametrize("d,k", [(64, 250), (40, 256), (64, 160), (12, 256), (4, 1)])
def test_tensor_core_form_shapes(cuda, d, k):
    """The tensor-core form's kernels: the pipelined one (planes in shared
    memory) where two tile slots fit beside the centroids, the first one
    (planes in TMEM) beyond (64 dimensions with more than 160 centroids)."""
    rng = np.random.default_rng(d * 7 + k)
    P, C = clustered(rng, 5000, d, k)
    got, _ = ours(P, C, hml.KMEANS_TENSOR)
    np.testing.assert_array_equal(got, oracle.kmeans_assign(P, C))


@pytest.mark.parametrize("method", METHODS)
def test_non_finite_values(cuda, method):
    """NaN and infinite coordinates: the reference skips a NaN distance
    (`dist < minDist` is false) and keeps the first of equal ones."""
    rng = np.random.default_rng(4)
    P, C = clustered(rng, 2000, 12, 30)  # 12 dimensions: every form applies
    P[5, 3] = np.nan
    P[6, :] = np.inf
    P[7, 0] = -np.inf
    C[4, 2] = np.nan
    C[9, 1] = np.inf
    P[8] = np.float32(3e19)  # squares overflow to inf
    got, exact = ours(P, C, method)
    np.testing.assert_array_equal(got, oracle.kmeans_assign(P, C))
    assert exact >= 4


@pytest.mark.parametrize("method", METHODS)
def test_near_ties_duplicates_and_bisectors(cuda, method):
    rng = np.random.default_rng(7)
    d = 16
    base = rng.standard_normal((20, d)).astype(np.float32)
    # pairs a few ulps apart, exact duplicates, and the rest
    near = np.nextafter(base[:10], np.float32(np.inf)).astype(np.float32)
    C = np.concatenate([base, near, base[10:15]]).astype(np.float32)
    # points: on centroids, on bisectors of close pairs, and random
    mid = ((base[:10].astype(np.float64) + near.astype(np.float64)) / 2).astype(np.float32)
    bis = ((base[:10].astype(np.float64) + base[10:20].astype(np.float64)) / 2).astype(np.float32)
    P = np.concatenate([C, mid, bis, rng.standard_normal((4000, d)).astype(np.float32)])
    got, exact = ours(P, C, method)
    np.testing.assert_array_equal(got, oracle.kmeans_assign(P, C))
    assert exact >= 20  # the close calls went through the reference's arithmetic


@pytest.mark.parametrize("method", METHODS)
def test_far_from_origin(cuda, method):
    """A common offset of 1e3 makes ||x||^2 - 2 x.c cancel: most points need
    the exact comparison, and still agree."""
    rng = np.random.default_rng(8)
    P, C = clustered(rng, 5000, 24, 40, spread=0.5)
    P += np.float32(1e3)
    C += np.float32(1e3)
    got, exact = ours(P, C, method)
    np.testing.assert_array_equal(got, oracle.kmeans_assign(P, C))
    assert exact > 0


@pytest.mark.skipif(not oracle.ref_gpu_kmeans_available(),
                    reason="reference k-means kernel not built (make -C oracle refgpu)")
@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("d", [8, 16, 32, 64])
def test_matches_reference_gpu_kernel(cuda, method, d):
    import torch
    rng = np.random.default_rng(100 + d)
    P, C = clustered(rng, 200000, d, 64, spread=0.8)
    dP, dC = dev(P), dev(C)
    ref = torch.zeros(P.shape[0], dtype=torch.int32, device="cuda")
    oracle.ref_gpu_kmeans_assign(ref.data_ptr(), dP.data_ptr(), P.shape[0], dC.data_ptr(),
                                 C.shape[0], d)
    got, exact = hml.kmeans_assign(dP, dC, count_exact=True, method=method)
    torch.cuda.synchronize()
    assert torch.equal(got, ref), int((got != ref).sum())
    np.testing.assert_array_equal(got.cpu().numpy().astype(np.uint32)[:20000],
                                  oracle.kmeans_assign(P[:20000], C))


@pytest.mark.skipif(not oracle.ref_gpu_kmeans_available(),
                    reason="reference k-means kernel not built (make -C oracle refgpu)")
@pytest.mark.parametrize("method", METHODS)
def test_large_case_against_reference_gpu_kernel(cuda, method):
    """1M points, 32 dims, 256 centroids."""
    import torch
    n, d, k = 1 << 20, 32, 256
    P = torch.empty(n * d, device="cuda")
    hml.fill_random(P, 9, 0, 1)
    Cn = torch.empty(k * d, device="cuda")
    hml.fill_random(Cn, 9, 1, 1)
    P = P.view(n, d)
    C = Cn.view(k, d)
    ref = torch.zeros(n, dtype=torch.int32, device="cuda")
    oracle.ref_gpu_kmeans_assign(ref.data_ptr(), P.data_ptr(), n, C.data_ptr(), k, d)
    got = hml.kmeans_assign(P, C, method=method)
    torch.cuda.synchronize()
    assert torch.equal(got, ref), int((got != ref).sum())
    assert hml.device_error() == 0
