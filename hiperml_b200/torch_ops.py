"""PyTorch operators over the C ABI: ``torch.ops.hml.sgemm``,
``torch.ops.hml.sgemv`` and ``torch.ops.hml.sgemm_batched``.

They take FP32 CUDA tensors in place (no copies: any layout with one unit
stride per matrix is passed to the library as its storage order, transposes
and leading dimension), run on the current CUDA stream, and return new
tensors.  Fake (meta) implementations give shapes for tracing.
"""
from __future__ import annotations

from typing import List

import torch

from . import api


def _check(t: torch.Tensor, name: str) -> None:
    if t.dtype != torch.float32 or not t.is_cuda:
        raise TypeError(f"{name}: expected a float32 CUDA tensor")


def _layout(t: torch.Tensor):
    """(order, leading dimension) of a 2-D tensor with one unit stride."""
    r, c = t.shape
    s0, s1 = t.stride()
    if s1 == 1 or c == 1:
        return api.ROW_MAJOR, max(s0, c, 1)
    if s0 == 1 or r == 1:
        return api.COL_MAJOR, max(s1, r, 1)
    raise ValueError("each matrix needs one unit stride")


def _sgemm_into(A, B, C, alpha):
    M, K = A.shape
    N = B.shape[1]
    oc, ldc = _layout(C)

    def op(t):
        o, ld = _layout(t)
        return (api.OP_N if o == oc else api.OP_T), ld

    ta, lda = op(A)
    tb, ldb = op(B)
    return (ta, tb, M, N, K, alpha, A.data_ptr(), lda, B.data_ptr(), ldb, 0.0, C.data_ptr(), ldc,
            oc)


@torch.library.custom_op("hml::sgemm", mutates_args=())
def sgemm(A: torch.Tensor, B: torch.Tensor, alpha: float = 1.0) -> torch.Tensor:
    """alpha * A @ B (FP32, FP32-accurate: SIMT or split-BF16 BF16X6 as the
    library selects).  The result is column-major (stride (1, M))."""
    _check(A, "A")
    _check(B, "B")
    if A.dim() != 2 or B.dim() != 2 or A.shape[1] != B.shape[0]:
        raise ValueError("sgemm: shapes do not multiply")
    M, N = A.shape[0], B.shape[1]
    C = torch.empty((N, M), dtype=torch.float32, device=A.device).t()
    if M and N:
        ta, tb, M, N, K, al, a, lda, b, ldb, be, c, ldc, oc = _sgemm_into(A, B, C, alpha)
        api.sgemm_ex(oc, ta, tb, M, N, K, al, a, lda, b, ldb, be, c, ldc,
                     stream=torch.cuda.current_stream(A.device).cuda_stream)
    return C


@sgemm.register_fake
def _(A, B, alpha=1.0):
    return A.new_empty((B.shape[1], A.shape[0])).t()


@torch.library.custom_op("hml::sgemv", mutates_args=())
def sgemv(A: torch.Tensor, x: torch.Tensor, alpha: float = 1.0) -> torch.Tensor:
    """alpha * A @ x for a 2-D A and a 1-D contiguous x."""
    _check(A, "A")
    _check(x, "x")
    if A.dim() != 2 or x.dim() != 1 or A.shape[1] != x.shape[0] or x.stride(0) != 1:
        raise ValueError("sgemv: bad shapes")
    M, N = A.shape
    y = torch.empty(M, dtype=torch.float32, device=A.device)
    if M:
        order, lda = _layout(A)
        api.sgemv_ex(order, api.OP_N, M, N, alpha, A.data_ptr(), lda, x.data_ptr(), 0.0,
                     y.data_ptr(), stream=torch.cuda.current_stream(A.device).cuda_stream)
    return y


@sgemv.register_fake
def _(A, x, alpha=1.0):
    return A.new_empty((A.shape[0],))


@torch.library.custom_op("hml::sgemm_batched", mutates_args=())
def sgemm_batched(As: List[torch.Tensor], Bs: List[torch.Tensor]) -> List[torch.Tensor]:
    """[A_i @ B_i] for many uneven problems in one persistent launch
    (hml_sgemm_batched).  Results are column-major."""
    if len(As) != len(Bs):
        raise ValueError("sgemm_batched: list lengths differ")
    outs, descs = [], []
    for A, B in zip(As, Bs):
        _check(A, "A")
        _check(B, "B")
        if A.dim() != 2 or B.dim() != 2 or A.shape[1] != B.shape[0]:
            raise ValueError("sgemm_batched: shapes do not multiply")
        C = torch.empty((B.shape[1], A.shape[0]), dtype=torch.float32, device=A.device).t()
        outs.append(C)
        if C.numel() == 0:
            continue
        ta, tb, M, N, K, al, a, lda, b, ldb, be, c, ldc, oc = _sgemm_into(A, B, C, 1.0)
        # C is column-major, so every problem is expressed column-major
        descs.append((ta, tb, M, N, K, al, a, lda, b, ldb, be, c, ldc))
    if descs:
        api.sgemm_batched(api.COL_MAJOR, descs,
                          stream=torch.cuda.current_stream(As[0].device).cuda_stream)
    return outs


@sgemm_batched.register_fake
def _(As, Bs):
    return [A.new_empty((B.shape[1], A.shape[0])).t() for A, B in zip(As, Bs)]
