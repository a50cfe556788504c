"""Single calls captured in a CUDA graph by the caller (GPU): the split-BF16
path (B-splitting kernel, then the tensor-core kernel launched as its
programmatic dependent), the stream-K SIMT kernel and the column GEMV (both
with per-stream workspace and arrival counters) replay to the same bits as
the eager calls, also with new data in the same buffers."""
import numpy as np
import pytest

import hiperml_b200 as hml
from hiperml_b200 import datagen as dg
from hiperml_b200._lib import SgemmConfig

pytestmark = pytest.mark.gpu

CASES = [
    ("bf16x6", 2000, 48, 1500, SgemmConfig(hml.ALGO_BF16X6, 128, 64, 2, 4, 2)),
    ("tf32x3", 2000, 32, 1500, SgemmConfig(hml.ALGO_TF32X3, 128, 32, 1, 4, 1)),
    ("stream", 3000, 8, 2500, SgemmConfig(hml.ALGO_SIMT, 128, 8, 1, 4, 10)),
]


@pytest.mark.parametrize("name,M,N,K,cfg", CASES, ids=[c[0] for c in CASES])
def test_sgemm_call_replays_in_a_graph(cuda, name, M, N, K, cfg):
    import torch
    A = torch.empty(M * K, device="cuda")
    B = torch.empty(K * N, device="cuda")
    C = torch.zeros(M * N, device="cuda")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        def call():
            hml.sgemm_ex(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, C, M, stream=s, config=cfg)
        for seed in (1, 2):
            hml.fill_random(A, seed, 0, dg.UNIFORM, stream=s)
            hml.fill_random(B, seed, 1, dg.UNIFORM, stream=s)
            call()  # eager; also sizes the stream's workspace before capture
            s.synchronize()
            eager = C.clone()
            C.zero_()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s):
                call()
            for _ in range(2):
                g.replay()
                s.synchronize()
                assert torch.equal(C, eager), name
            del g
    assert hml.device_error() == 0


def test_gemv_call_replays_in_a_graph(cuda):
    import torch
    M, N = 4099, 3000
    A = torch.empty(M * N, device="cuda")
    x = torch.empty(N, device="cuda")
    y = torch.zeros(M, device="cuda")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        hml.fill_random(A, 3, 0, dg.NORMAL, stream=s)
        hml.fill_random(x, 3, 1, dg.NORMAL, stream=s)
        call = lambda: hml.sgemv_ex(0, 0, M, N, 1.0, A, M, x, 0.0, y, variant=8, stream=s)
        call()
        s.synchronize()
        eager = y.clone()
        y.zero_()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            call()
        for _ in range(3):
            g.replay()
            s.synchronize()
            assert torch.equal(y, eager)
        del g
