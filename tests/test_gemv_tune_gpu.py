"""The SGEMV autotuner (GPU): every variant of the kernel for the layout is
measured, the fastest is recorded, and hml_sgemv_ex / the SGEMM N = 1 route
/ hmlSgemv then run it, bit for bit the same as forcing that variant."""
import numpy as np
import pytest

import hiperml_b200 as hml
import oracle
from hiperml_b200 import datagen as dg
from hiperml_b200._lib import lib
from tests.gpu_util import assert_within_fp32_bound, to_dev, to_host

pytestmark = pytest.mark.gpu

ROW_VARIANTS = [4, 8, 16, 32, 64, 128, 256]
COL_VARIANTS = list(range(1, 17)) + [20, 24, 32, 48, 64, 96, 128, 192, 256]


def _store(A, order):
    """A (M x N, numpy) stored dense in `order`; returns (tensor, lda)."""
    import torch
    M, N = A.shape
    if order == hml.COL_MAJOR:
        return torch.from_numpy(np.ascontiguousarray(A.T)).cuda(), M
    return torch.from_numpy(np.ascontiguousarray(A)).cuda(), N


@pytest.mark.parametrize("order,trans,rows", [
    (hml.ROW_MAJOR, hml.OP_N, True),
    (hml.COL_MAJOR, hml.OP_N, False),
    (hml.COL_MAJOR, hml.OP_T, True),
    (hml.ROW_MAJOR, hml.OP_T, False),
])
def test_autotune_sgemv_records_fastest(cuda, order, trans, rows):
    M, N = (8192, 2048) if trans == hml.OP_N else (2048, 8192)
    hml.tune_clear()
    try:
        res = hml.autotune_sgemv(order, trans, M, N, reps=3)
        assert [v for v, _, _ in res] == (ROW_VARIANTS if rows else COL_VARIANTS)
        assert all(st == 0 and t > 0 for _, t, st in res), res
        best = min(res, key=lambda r: r[1])[0]
        assert hml.sgemv_select(order, trans, M, N) == best

        A = dg.matrix(M, N, 77, 0, dg.NORMAL, order="C")
        P, Q = (M, N) if trans == hml.OP_N else (N, M)
        x = dg.fill(Q, 77, 1, dg.NORMAL)
        y0 = dg.fill(P, 77, 2, dg.UNIFORM)
        dA, lda = _store(A, order)
        dx = to_dev(x)
        outs = []
        # variant=0 calls hml_sgemv_ex, which consults the table; then the
        # recorded variant forced through hml_sgemv_ex_variant
        for variant in (0, best):
            y = to_dev(y0)
            hml.sgemv_ex(order, trans, M, N, 0.5, dA, lda, dx, -1.25, y, variant=variant)
            outs.append(to_host(y))
        assert np.array_equal(outs[0], outs[1])
        opA = A.T if trans == hml.OP_T else A
        D, absD = oracle.dgemm(opA, x.reshape(-1, 1), y0.reshape(-1, 1), 0.5, -1.25,
                               with_abs=True)
        assert_within_fp32_bound(outs[0], D[:, 0], absD[:, 0], Q, what=f"tuned {best}")
    finally:
        hml.tune_clear()


def test_tuned_variant_serves_gemm_n1_and_host_path(cuda):
    """The SGEMM N = 1 route and hmlSgemv consult the same table."""
    import torch
    M, N = 8192, 2048
    hml.tune_clear()
    lib.hml_cfg_v1_clear()  # no reference v1 SGEMV rule overrides the table
    try:
        res = hml.autotune_sgemv(hml.ROW_MAJOR, hml.OP_N, M, N, reps=3)
        best = min(res, key=lambda r: r[1])[0]
        A = dg.matrix(M, N, 78, 0, dg.NORMAL, order="C")
        x = dg.fill(N, 78, 1, dg.NORMAL)
        dA, lda = _store(A, hml.ROW_MAJOR)
        dx = to_dev(x)
        y = torch.zeros(M, dtype=torch.float32, device="cuda")
        hml.sgemv_ex(hml.ROW_MAJOR, hml.OP_N, M, N, 1.0, dA, lda, dx, 0.0, y, variant=best)
        forced = to_host(y)
        # C (M x 1) = A (M x N) B (N x 1), row-major: B's one column is x
        c = torch.zeros(M, dtype=torch.float32, device="cuda")
        hml.sgemm_ex(hml.ROW_MAJOR, hml.OP_N, hml.OP_N, M, 1, N, 1.0, dA, lda, dx, 1, 0.0, c, 1)
        assert np.array_equal(to_host(c), forced)
        yh = np.zeros(M, np.float32)
        hml.hmlSgemv(yh, A, x, M, N, 1.0, 0.0)
        assert np.array_equal(yh, forced)
    finally:
        hml.tune_clear()

