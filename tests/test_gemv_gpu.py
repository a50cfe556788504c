"""GEMV kernels against the oracle (GPU)."""
import numpy as np
import pytest

import hiperml_b200 as hml
import oracle
from hiperml_b200 import datagen as dg
from tests.golden_cases import load
from tests.gpu_util import assert_within_fp32_bound, to_dev, to_host

pytestmark = pytest.mark.gpu
META, ARR = load()


def run_gemv(order, trans, A_np, lda_pad, x_np, y_np, alpha, beta, variant=0, offset=0):
    """A_np is the logical M x N matrix; it is stored in `order` with a
    leading dimension padded by lda_pad and a base offset of `offset` floats."""
    import torch
    M, N = A_np.shape
    if order == hml.COL_MAJOR:
        lda = M + lda_pad
        store = torch.zeros(N * lda + offset, dtype=torch.float32, device="cuda")
        view = store[offset:offset + N * lda].view(N, lda)[:, :M]
        view.copy_(torch.from_numpy(np.ascontiguousarray(A_np.T)))
    else:
        lda = N + lda_pad
        store = torch.zeros(M * lda + offset, dtype=torch.float32, device="cuda")
        view = store[offset:offset + M * lda].view(M, lda)[:, :N]
        view.copy_(torch.from_numpy(A_np))
    base = store.data_ptr() + 4 * offset
    x = to_dev(x_np)
    y = to_dev(y_np)
    hml.sgemv_ex(order, trans, M, N, alpha, base, lda, x, beta, y, variant=variant)
    return to_host(y)


def expected(A, x, y, alpha, beta, trans):
    opA = A.T if trans else A
    D, absD = oracle.dgemm(opA, x.reshape(-1, 1), y.reshape(-1, 1), alpha, beta, with_abs=True)
    return D[:, 0], absD[:, 0]


SHAPES = [(1, 1), (7, 3), (128, 64), (129, 65), (1000, 37), (37, 1000), (4099, 129), (3, 5000)]


@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("trans", [0, 1])
@pytest.mark.parametrize("shape", SHAPES)
def test_gemv_layouts(cuda, order, trans, shape):
    M, N = shape
    A = dg.matrix(M, N, 101, 0, dg.NORMAL, order="C")
    P, Q = (N, M) if trans else (M, N)
    x = dg.fill(Q, 101, 1, dg.NORMAL)
    y = dg.fill(P, 101, 2, dg.UNIFORM)
    for alpha, beta in ((1.0, 0.0), (-0.75, 1.5)):
        for pad, off in ((0, 0), (1, 0), (0, 1)):
            got = run_gemv(order, trans, A, pad, x, y, alpha, beta, offset=off)
            D, absD = expected(A, x, y, alpha, beta, trans)
            assert_within_fp32_bound(got, D, absD, Q, what=f"{order}{trans}{shape}{pad}{off}")


@pytest.mark.parametrize("variant", [4, 8, 16, 32, 64, 128, 256])
def test_gemv_rows_variants(cuda, variant):
    M, N = 777, 3001
    A = dg.matrix(M, N, 102, 0, dg.UNIFORM, order="C")
    x = dg.fill(N, 102, 1)
    y = dg.fill(M, 102, 2)
    got = run_gemv(hml.ROW_MAJOR, hml.OP_N, A, 0, x, y, 1.0, 0.5, variant=variant)
    D, absD = expected(A, x, y, 1.0, 0.5, False)
    assert_within_fp32_bound(got, D, absD, N)


@pytest.mark.parametrize("variant", [1, 2, 3, 5, 8, 11, 16, 24, 64, 128, 256])
def test_gemv_cols_split(cuda, variant):
    """The column kernel with `variant` CTAs per 256-row tile (the last to
    finish sums the partials in a fixed order), ragged rows and columns."""
    M, N = 1531, 700
    A = dg.matrix(M, N, 103, 0, dg.UNIFORM, order="C")
    x = dg.fill(N, 103, 1)
    y = dg.fill(M, 103, 2)
    got = run_gemv(hml.COL_MAJOR, hml.OP_N, A, 0, x, y, 2.0, -1.0, variant=variant)
    D, absD = expected(A, x, y, 2.0, -1.0, False)
    assert_within_fp32_bound(got, D, absD, N)


def test_gemv_cols_split_repeatable(cuda):
    """Split partials are summed in a fixed order whatever order the CTAs finish
    in: repeated calls give identical bits, and the per-tile arrival counters
    are left ready for the next call (also after a call with another split)."""
    import torch
    M, N = 4099, 2048
    A = dg.matrix(M, N, 105, 0, dg.NORMAL, order="F")
    x = dg.fill(N, 105, 1, dg.NORMAL)
    Ad, xd = to_dev(A), to_dev(x)
    outs = []
    for variant in (8, 8, 5, 8, 1, 8):
        y = torch.zeros(M, device="cuda")
        hml.sgemv_ex(hml.COL_MAJOR, hml.OP_N, M, N, 1.0, Ad, M, xd, 0.0, y, variant=variant)
        torch.cuda.synchronize()
        outs.append((variant, y.cpu().numpy()))
    ref = [o for v, o in outs if v == 8]
    for o in ref[1:]:
        assert np.array_equal(o, ref[0])
    D, absD = expected(A, x, np.zeros(M, np.float32), 1.0, 0.0, False)
    for v, o in outs:
        assert_within_fp32_bound(o, D, absD, N, what=f"split {v}")


# Short-wide problems: y has few entries and A's rows are long.  Column
# layout (y = A x, A column-major): P <= 128 runs the 128-row tile with 8
# column phases, and up to 128 CTAs split the columns of one tile.  Row
# layout (y = A^T x): few long rows are split over several CTAs per row.
SHORT_WIDE = [(1, 5000), (3, 70001), (16, 100000), (64, 200000), (100, 30001), (128, 65536),
              (129, 40000), (255, 33333), (256, 65536), (512, 65536), (2048, 16384)]


@pytest.mark.parametrize("shape", SHORT_WIDE, ids=lambda s: f"{s[0]}x{s[1]}")
@pytest.mark.parametrize("layout", ["cols", "rows"])
def test_gemv_short_wide(cuda, shape, layout):
    import torch
    P, Q = shape
    rng = np.random.default_rng(P * 7 + Q)
    opA = rng.standard_normal((P, Q)).astype(np.float32)  # the logical op(A)
    x = rng.standard_normal(Q).astype(np.float32)
    y0 = rng.uniform(-1, 1, P).astype(np.float32)
    # cols: A = op(A) column-major, y = A x; rows: A = op(A)^T column-major
    # (Q x P), y = A^T x, whose rows are op(A)'s rows, contiguous
    if layout == "cols":
        store = torch.from_numpy(np.ascontiguousarray(opA.T)).cuda()  # columns contiguous
        args = (hml.COL_MAJOR, hml.OP_N, P, Q)
        lda = P
    else:
        store = torch.from_numpy(np.ascontiguousarray(opA)).cuda()    # rows contiguous
        args = (hml.COL_MAJOR, hml.OP_T, Q, P)
        lda = Q
    xd = to_dev(x)
    outs = []
    for _ in range(2):
        y = to_dev(y0)
        hml.sgemv_ex(*args, 1.5, store, lda, xd, -0.5, y)
        outs.append(to_host(y))
    assert np.array_equal(outs[0], outs[1])  # deterministic split reductions
    D, absD = oracle.dgemm(opA, x.reshape(-1, 1), y0.reshape(-1, 1), 1.5, -0.5,
                           with_abs=True)
    assert_within_fp32_bound(outs[0], D[:, 0], absD[:, 0], Q, what=f"{layout} {shape}")


@pytest.mark.parametrize("variant", [1, 7, 32, 128])
def test_gemv_cols_narrow_forced_splits(cuda, variant):
    """The 128-row tile with a forced split, odd P (ragged lanes) and a
    column count that the split does not divide."""
    P, Q = 77, 9999
    A = dg.matrix(P, Q, 106, 0, dg.UNIFORM, order="C")
    x = dg.fill(Q, 106, 1)
    y = dg.fill(P, 106, 2)
    got = run_gemv(hml.COL_MAJOR, hml.OP_N, A, 0, x, y, 1.0, 2.0, variant=variant)
    D, absD = expected(A, x, y, 1.0, 2.0, False)
    assert_within_fp32_bound(got, D, absD, Q)


@pytest.mark.parametrize("P,pad", [(2, 2), (4, 0), (5, 3), (8, 0), (30, 2), (61, 3), (64, 0),
                                   (97, 3), (128, 0)])
@pytest.mark.parametrize("variant", [0, 1, 3, 40, 256])
def test_gemv_short_kernel(cuda, P, pad, variant):
    """16-byte column layout with P <= 128 (LPC = 1..32 lanes per column,
    P % 4 != 0 leaves a partial last quad), leading dimension padded to a
    multiple of 4, forced and heuristic splits, ragged column count."""
    Q = 12347
    A = dg.matrix(P, Q, 107, 0, dg.NORMAL, order="C")
    x = dg.fill(Q, 107, 1, dg.NORMAL)
    y = dg.fill(P, 107, 2)
    outs = [run_gemv(hml.COL_MAJOR, hml.OP_N, A, pad, x, y, -1.0, 0.75, variant=variant)
            for _ in range(2)]
    assert np.array_equal(outs[0], outs[1])
    D, absD = expected(A, x, y, -1.0, 0.75, False)
    assert_within_fp32_bound(outs[0], D, absD, Q, what=f"P={P} split={variant}")


def test_beta_zero_does_not_read_y(cuda):
    import torch
    M, N = 300, 200
    A = dg.matrix(M, N, 104, 0, order="C")
    x = dg.fill(N, 104, 1)
    for order in (0, 1):
        y = torch.full((M,), float("nan"), device="cuda")
        Ad = to_dev(A if order == 1 else np.asfortranarray(A))
        lda = N if order == 1 else M
        hml.sgemv_ex(order, 0, M, N, 1.0, Ad, lda, to_dev(x), 0.0, y)
        assert torch.isfinite(y).all()


@pytest.mark.parametrize("case", META["sgemv"], ids=lambda c: c["name"])
def test_gemv_matches_reference_golden(cuda, case):
    """Our SGEMV vs the reference's hmlSgemvCpu output on the same inputs."""
    M, N = case["M"], case["N"]
    A = dg.matrix(M, N, case["seed"], 0, case["dist"], order="C")
    x = dg.fill(N, case["seed"], 1, case["dist"])
    y = dg.fill(M, case["seed"], 2, dg.UNIFORM)
    got = run_gemv(hml.ROW_MAJOR, hml.OP_N, A, 0, x, y, case["alpha"], case["beta"])
    D, absD = expected(A, x, y, case["alpha"], case["beta"], False)
    ref = ARR["sgemv_" + case["name"]]
    assert_within_fp32_bound(got, D, absD, N, what="ours")
    assert_within_fp32_bound(ref, D, absD, N, what="reference")
    # ours vs the reference's output directly: both within the bound of D
    assert np.all(np.abs(got.astype(np.float64) - ref) <= 4 * (N + 2) * 2.0 ** -24 * absD + 1e-37)


@pytest.mark.parametrize("kind", ["sgemv_n", "sgemv_t"])
def test_gemv_full_size_against_reference_golden(cuda, kind):
    """A 32768 x 4096 column-major N(0,1), seed 1: y = A x and y = A^T x,
    generated on the device and compared with the reference loop's outputs."""
    import torch
    c = [x for x in META["configs"] if x["kind"] == kind][0]
    M, N = 32768, 4096
    A = torch.empty(M * N, dtype=torch.float32, device="cuda")
    hml.fill_random(A, 1, 0, dg.NORMAL)
    Q = N if kind == "sgemv_n" else M
    x = torch.empty(Q, dtype=torch.float32, device="cuda")
    hml.fill_random(x, 1, 1, dg.NORMAL)
    P = M if kind == "sgemv_n" else N
    y = torch.zeros(P, dtype=torch.float32, device="cuda")
    hml.sgemv_ex(hml.COL_MAJOR, hml.OP_N if kind == "sgemv_n" else hml.OP_T, M, N, 1.0, A, M, x,
                 0.0, y)
    got = y.cpu().numpy().astype(np.float64)
    ref = ARR["cfg_" + kind + "_32768x4096"].astype(np.float64)
    n_op = kind == "sgemv_n"
    # FP64 answer and |A||x| on the GPU in double
    Am = A.view(N, M).t().double()  # logical 32768 x 4096
    opA = Am if n_op else Am.t()
    D = (opA @ x.double()).cpu().numpy()
    absD = (opA.abs() @ x.double().abs()).cpu().numpy()
    del Am, opA
    # ours and the reference loop each within the classical FP32 bound
    assert_within_fp32_bound(got, D, absD, Q, slack=1.0, what="ours")
    assert_within_fp32_bound(ref, D, absD, Q, slack=1.0, what="reference")
    assert abs(got.sum() - c["csum"]) <= 1e-5 * np.abs(ref).sum()
    # the product's own FP64 check agrees
    err = hml.error_fp64(hml.COL_MAJOR, hml.OP_N if n_op else hml.OP_T, hml.OP_N, P, 1, Q, 1.0,
                         A, M, x, Q, 0.0, None, y, P)
    assert err[0] < 1e-6 and err[2] <= (Q + 2) * 2.0 ** -24, err


def test_no_device_error_left(cuda):
    assert hml.device_error() == 0
