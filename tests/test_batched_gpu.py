"""Batched SGEMM: many uneven problems in persistent launches (GPU).

Every problem of a batch is checked two ways: bit for bit against the
single-problem kernel run with the configuration the batch reports for it
(hml_batch_problem_config: the FP32 SIMT tile, or BF16X6 tensor-core tiles
for N > 8 with split_k = 1; the batched kernels share the tile arithmetic),
and against the FP64 oracle within the classical FP32 bound
gamma_{K+2} (|alpha||A||B| + |beta||C|)."""
import numpy as np
import pytest

import hiperml_b200 as hml
import oracle
from hiperml_b200 import datagen as dg
from hiperml_b200._lib import SgemmConfig, lib
from tests.gpu_util import assert_within_fp32_bound

pytestmark = pytest.mark.gpu

class Problem:
    """One problem with its own device buffers (storage order, ld padding and
    base offset chosen per problem)."""

    def __init__(self, order, ta, tb, M, N, K, alpha, beta, seed, pad, offset):
        import torch
        self.order, self.ta, self.tb = order, ta, tb
        self.M, self.N, self.K, self.alpha, self.beta = M, N, K, alpha, beta
        self.A = dg.matrix(K if ta else M, M if ta else K, seed, 0, dg.NORMAL, order="C")
        self.B = dg.matrix(N if tb else K, K if tb else N, seed, 1, dg.NORMAL, order="C")
        self.C0 = dg.matrix(M, N, seed, 2, dg.UNIFORM, order="C")
        self.pad, self.offset = pad, offset
        self.Ab, self.Ap, self.lda = self._store(self.A)
        self.Bb, self.Bp, self.ldb = self._store(self.B)
        self.Cb, self.Cp, self.ldc = self._store(self.C0)
        self.Cinit = self.Cb.clone()

    def _store(self, logical):
        import torch
        r, c = logical.shape
        if self.order == hml.COL_MAJOR:
            ld = max(1, r + self.pad)
            buf = torch.zeros(c * ld + self.offset + 4, device="cuda")
            buf[self.offset:self.offset + c * ld].view(c, ld)[:, :r].copy_(
                torch.from_numpy(np.ascontiguousarray(logical.T)))
        else:
            ld = max(1, c + self.pad)
            buf = torch.zeros(r * ld + self.offset + 4, device="cuda")
            buf[self.offset:self.offset + r * ld].view(r, ld)[:, :c].copy_(
                torch.from_numpy(logical))
        return buf, buf.data_ptr() + 4 * self.offset, ld

    def desc(self):
        return (self.ta, self.tb, self.M, self.N, self.K, self.alpha, self.Ap, self.lda, self.Bp,
                self.ldb, self.beta, self.Cp, self.ldc)

    def reset(self):
        self.Cb.copy_(self.Cinit)

    def result(self, buf=None):
        h = (self.Cb if buf is None else buf).cpu().numpy()[self.offset:]
        if self.order == hml.COL_MAJOR:
            return h[:self.N * self.ldc].reshape(self.N, self.ldc)[:, :self.M].T.copy()
        return h[:self.M * self.ldc].reshape(self.M, self.ldc)[:, :self.N].copy()

    def single(self):
        """The single-problem kernel with this problem's batched configuration."""
        import torch
        keep = self.Cb.clone()
        self.reset()
        hml.sgemm_ex(self.order, self.ta, self.tb, self.M, self.N, self.K, self.alpha, self.Ap,
                     self.lda, self.Bp, self.ldb, self.beta, self.Cp, self.ldc,
                     config=hml.batch_problem_config(self.order, self.desc()))
        torch.cuda.synchronize()
        out = self.result()
        self.Cb.copy_(keep)
        return out

    def check_fp64(self, got):
        D, absD = oracle.dgemm(self.A, self.B, self.C0, self.alpha, self.beta,
                               transA=bool(self.ta), transB=bool(self.tb), with_abs=True)
        assert_within_fp32_bound(got, D, absD, max(self.K, 1), what=f"batched {self}")

    def __repr__(self):
        return (f"P(order={self.order} ta={self.ta} tb={self.tb} M={self.M} N={self.N} K={self.K} "
                f"pad={self.pad} off={self.offset} a={self.alpha} b={self.beta})")


def random_batch(seed, count, Mmax, Nmax, Kmax, aligned):
    rng = np.random.default_rng(seed)
    probs = []
    for i in range(count):
        M = int(rng.integers(1, Mmax + 1))
        N = int(rng.integers(1, Nmax + 1))
        K = int(rng.integers(1, Kmax + 1))
        order = int(rng.integers(0, 2))
        ta, tb = int(rng.integers(0, 2)), int(rng.integers(0, 2))
        alpha = float(rng.choice([1.0, -0.75, 2.0]))
        beta = float(rng.choice([0.0, 1.0, 0.5]))
        if aligned:
            pad, offset = 0, 0  # natural dense storage
        else:
            pad, offset = int(rng.integers(0, 4)), int(rng.integers(0, 3))
        probs.append(Problem(order, ta, tb, M, N, K, alpha, beta, 1000 + seed * 977 + i, pad,
                             offset))
    return probs


def padded_batch(seed, count, Mmax, Nmax, Kmax):
    """All leading dimensions multiples of 4 floats and 16-byte bases: every
    problem takes the 16-byte copy path."""
    rng = np.random.default_rng(seed)
    probs = []
    for i in range(count):
        M = int(rng.integers(1, Mmax + 1))
        N = int(rng.integers(1, Nmax + 1))
        K = int(rng.integers(1, Kmax + 1))
        ta, tb = int(rng.integers(0, 2)), int(rng.integers(0, 2))
        p = Problem(hml.COL_MAJOR, ta, tb, M, N, K, 1.0, 0.0, 5000 + i, 0, 0)
        # rebuild with ld rounded up to a multiple of 4
        rows_a = K if ta else M
        p.pad = (-rows_a) % 4
        p.Ab, p.Ap, p.lda = p._store(p.A)
        p.pad = (-(N if tb else K)) % 4
        p.Bb, p.Bp, p.ldb = p._store(p.B)
        p.pad = (-M) % 4
        p.Cb, p.Cp, p.ldc = p._store(p.C0)
        p.Cinit = p.Cb.clone()
        probs.append(p)
    return probs


def run_plan(order, probs, graph=False):
    import torch
    with hml.BatchPlan(order, [p.desc() for p in probs]) as plan:
        if graph:
            plan.graph_launch()
        else:
            plan.run()
        torch.cuda.synchronize()
        info = plan.info()
    return info


@pytest.mark.parametrize("aligned", [True, False])
def test_batched_matches_single_kernel_bitwise(cuda, aligned):
    import torch
    probs = random_batch(1 if aligned else 2, 48, 600, 150, 300, aligned)
    # one batch per storage order (a batch has one order)
    for order in (hml.COL_MAJOR, hml.ROW_MAJOR):
        sub = [p for p in probs if p.order == order]
        info = run_plan(order, sub)
        assert info["tiles"] > 0 and info["ctas"] > 0
        assert hml.device_error() == 0
        for p in sub:
            got = p.result()
            ref = p.single()
            assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), p
            p.check_fp64(got)


def test_batched_16_byte_path_bitwise(cuda):
    probs = padded_batch(3, 40, 900, 130, 400)
    run_plan(hml.COL_MAJOR, probs)
    for p in probs:
        got = p.result()
        assert np.array_equal(got.view(np.uint32), p.single().view(np.uint32)), p
        p.check_fp64(got)


def test_graph_replay_and_queue_reset(cuda):
    """The queue resets itself at the end of each launch: every replay of the
    captured graph (and every plain run after it) redoes the whole batch."""
    import torch
    probs = padded_batch(4, 24, 700, 70, 200)
    for p in probs:
        p.beta = 1.0  # C accumulates: C = C0 + r * alpha * A B after r runs
    with hml.BatchPlan(hml.COL_MAJOR, [p.desc() for p in probs]) as plan:
        plan.graph_launch()
        plan.graph_launch()
        plan.run()
        torch.cuda.synchronize()
    for p in probs:
        got = p.result().astype(np.float64)
        D, absD = oracle.dgemm(p.A, p.B, p.C0, 3.0, 1.0, transA=bool(p.ta), transB=bool(p.tb),
                               with_abs=True)
        assert_within_fp32_bound(got, D, absD, p.K + 3, slack=4.0, what=repr(p))


def test_one_shot_equals_plan(cuda):
    import torch
    probs = random_batch(5, 20, 500, 100, 300, False)
    col = [p for p in probs if p.order == hml.COL_MAJOR]
    hml.sgemm_batched(hml.COL_MAJOR, [p.desc() for p in col])
    torch.cuda.synchronize()
    first = [p.result() for p in col]
    for p in col:
        p.reset()
    run_plan(hml.COL_MAJOR, col)
    for p, r in zip(col, first):
        assert np.array_equal(p.result().view(np.uint32), r.view(np.uint32)), p


def test_degenerate_problems(cuda):
    """K = 0 and alpha = 0 scale C by beta; empty problems are skipped."""
    import torch
    ps = [Problem(0, 0, 0, 300, 20, 0, 1.0, 0.5, 7, 0, 0),
          Problem(0, 1, 0, 200, 9, 50, 0.0, -2.0, 8, 0, 0),
          Problem(0, 0, 0, 0, 5, 10, 1.0, 0.0, 9, 0, 0),
          Problem(0, 0, 1, 129, 1, 70, 1.5, 0.0, 10, 1, 1)]
    run_plan(hml.COL_MAJOR, ps)
    np.testing.assert_array_equal(ps[0].result(), (np.float32(0.5) * ps[0].C0).astype(np.float32))
    np.testing.assert_array_equal(ps[1].result(), (np.float32(-2.0) * ps[1].C0).astype(np.float32))
    ps[3].check_fp64(ps[3].result())
    # an empty batch is a no-op
    with hml.BatchPlan(hml.COL_MAJOR, []) as plan:
        plan.run()
        plan.graph_launch()
        assert plan.info()["tiles"] == 0


def test_invalid_problem_reports_index(cuda):
    ps = [Problem(0, 0, 0, 64, 8, 32, 1.0, 0.0, 11, 0, 0)]
    d = [ps[0].desc(), (0, 0, 64, 8, 32, 1.0, ps[0].Ap, 10, ps[0].Bp, 32, 0.0, ps[0].Cp, 64)]
    with pytest.raises(hml.HmlError):
        hml.BatchPlan(hml.COL_MAJOR, d)
    assert b"batch problem 1" in lib.hml_last_error()


def test_benchmark_distribution_sample(cuda):
    """Problems drawn like the benchmark's batch (M log-uniform in
    [256, 16384], N uniform in 1..128, K log-uniform in [64, 4096], random
    transposes, N(0,1) entries), a subset small enough to check each one in
    FP64 on the GPU."""
    import torch
    rng = np.random.default_rng(3)
    descs, bufs = [], []
    shapes = []
    for i in range(40):
        M = int(np.exp(rng.uniform(np.log(256), np.log(16384))))
        N = int(rng.integers(1, 129))
        K = int(np.exp(rng.uniform(np.log(64), np.log(4096))))
        ta, tb = int(rng.integers(0, 2)), int(rng.integers(0, 2))
        A = torch.empty(M * K, device="cuda")
        B = torch.empty(K * N, device="cuda")
        C = torch.zeros(M * N, device="cuda")
        hml.fill_random(A, 3, 2 * i, dg.NORMAL)
        hml.fill_random(B, 3, 2 * i + 1, dg.NORMAL)
        lda = K if ta else M
        ldb = N if tb else K
        descs.append((ta, tb, M, N, K, 1.0, A, lda, B, ldb, 0.0, C, M))
        bufs.append((A, B, C))
        shapes.append((ta, tb, M, N, K, lda, ldb))
    with hml.BatchPlan(hml.COL_MAJOR, descs) as plan:
        plan.graph_launch()
        torch.cuda.synchronize()
    for (ta, tb, M, N, K, lda, ldb), (A, B, C) in zip(shapes, bufs):
        err = hml.error_fp64(0, ta, tb, M, N, K, 1.0, A, lda, B, ldb, 0.0, None, C, M)
        assert err[2] <= 2 * (K + 2) * 2.0 ** -24, (M, N, K, err)
