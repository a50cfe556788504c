"""Failure path of the bounded waits (GPU): a kernel waits on a barrier that
nothing completes; the wait gives up after its limit, the code lands in the
device error word, reading it clears it, and the device keeps working."""
import time

import numpy as np
import pytest

import hiperml_b200 as hml
import oracle
from hiperml_b200 import datagen as dg
from tests.gpu_util import assert_within_fp32_bound

pytestmark = pytest.mark.gpu


def test_expired_wait_is_reported_and_the_device_stays_usable(cuda):
    import torch
    hml.device_error()  # start clear
    t0 = time.time()
    hml.check_wait_limit()
    torch.cuda.synchronize()
    waited = time.time() - t0
    assert 1.5 < waited < 60, waited  # the 2 s limit, not a hang
    assert hml.device_error() == 1     # a tile that never landed
    assert hml.device_error() == 0     # reading cleared it
    # the context is intact: a split-BF16 and a SIMT GEMM still compute
    M, N, K = 700, 40, 900
    A = dg.matrix(M, K, 9, 0, order="F")
    B = dg.matrix(K, N, 9, 1, order="F")
    D, absD = oracle.dgemm(A, B, with_abs=True)
    for algo in (hml.ALGO_BF16X6, hml.ALGO_SIMT):
        cfg = hml.select_algo(0, 0, 0, M, N, K, algo)
        Ad = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
        Bd = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
        C = torch.zeros(N, M, device="cuda")
        hml.sgemm_ex(0, 0, 0, M, N, K, 1.0, Ad, M, Bd, K, 0.0, C, M, config=cfg)
        torch.cuda.synchronize()
        got = C.cpu().numpy().T
        e = oracle.rel_errors(got, D, absD)
        assert e["normwise"] < 2e-6, (algo, e)
    assert hml.device_error() == 0
