"""torch.ops.hml.* operators: registration and shapes on CPU (fake tensors),
results on the GPU."""
import numpy as np
import pytest
import torch

import hiperml_b200.torch_ops  # noqa: F401  (registers torch.ops.hml)
from tests.gpu_util import gamma


def test_ops_registered_with_fake_shapes():
    from torch._subclasses.fake_tensor import FakeTensorMode
    with FakeTensorMode():
        A = torch.empty(300, 40, device="cuda") if torch.cuda.is_available() else \
            torch.empty(300, 40)
        B = torch.empty(40, 7, device=A.device)
        C = torch.ops.hml.sgemm.default(A, B, 1.0)
        assert C.shape == (300, 7) and C.stride() == (1, 300)
        y = torch.ops.hml.sgemv.default(A, torch.empty(40, device=A.device), 2.0)
        assert y.shape == (300,)
        outs = torch.ops.hml.sgemm_batched.default([A, A.t()], [B, torch.empty(300, 3,
                                                                                 device=A.device)])
        assert [o.shape for o in outs] == [(300, 7), (40, 3)]


def _bound_check(got, A, B):
    exact = A.double() @ B.double()
    absb = A.double().abs() @ B.double().abs()
    err = (got.double() - exact).abs()
    K = A.shape[1]
    assert bool((err <= 2 * gamma(K + 2) * absb + 1e-30).all()), float((err / absb).max())


@pytest.mark.gpu
def test_sgemm_op_layouts(cuda):
    g = torch.Generator(device="cuda").manual_seed(1)
    for (M, N, K) in ((4096, 16, 4096), (1000, 130, 77), (33, 500, 64)):
        A = torch.randn(M, K, device="cuda", generator=g)
        B = torch.randn(K, N, device="cuda", generator=g)
        for a in (A, A.t().contiguous().t()):
            for b in (B, B.t().contiguous().t()):
                C = torch.ops.hml.sgemm(a, b)
                torch.cuda.synchronize()
                _bound_check(C, A, B)


@pytest.mark.gpu
def test_sgemv_and_batched_ops(cuda):
    g = torch.Generator(device="cuda").manual_seed(2)
    A = torch.randn(5000, 300, device="cuda", generator=g)
    x = torch.randn(300, device="cuda", generator=g)
    y = torch.ops.hml.sgemv(A, x, 1.0)
    _bound_check(y[:, None], A, x[:, None])
    As = [torch.randn(m, k, device="cuda", generator=g) for m, k in ((700, 64), (300, 2000), (9, 40))]
    Bs = [torch.randn(k, n, device="cuda", generator=g) for (m, k), n in
          zip(((700, 64), (300, 2000), (9, 40)), (5, 100, 12))]
    outs = torch.ops.hml.sgemm_batched(As, Bs)
    torch.cuda.synchronize()
    for C, A_, B_ in zip(outs, As, Bs):
        _bound_check(C, A_, B_)
