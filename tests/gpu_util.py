"""Helpers for the GPU parity tests: device copies of numpy operands and
the error bounds every parity check uses."""
import numpy as np

import oracle

U = 2.0 ** -24


def gamma(n):
    """Classical bound for n FP32 roundings (Higham, Lemma 3.1)."""
    return n * U / (1.0 - n * U)


def to_dev(a):
    """float32 CUDA tensor with the same memory order as the numpy array."""
    import torch
    a = np.asarray(a, np.float32)
    if a.ndim == 2 and a.flags["F_CONTIGUOUS"] and not a.flags["C_CONTIGUOUS"]:
        return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def to_host(t):
    import torch
    torch.cuda.synchronize()
    if t.dim() == 2 and t.stride(0) == 1 and t.stride(1) != 1:
        return np.ascontiguousarray(t.t().cpu().numpy()).T
    return t.cpu().numpy()


def assert_within_fp32_bound(got, exact, absbound, K, slack=2.0, what=""):
    """|got - exact| <= slack * gamma_{K+2} * (|alpha||A||B| + |beta||C|).
    Holds for any summation order; slack 2 also covers a second FP32 result
    (e.g. comparing two FP32 implementations through the FP64 value)."""
    got = np.asarray(got, np.float64)
    err = np.abs(got - exact)
    bound = slack * gamma(K + 2) * absbound
    bad = err > bound + 1e-37
    if bad.any():
        i = np.argwhere(bad)[0]
        raise AssertionError(f"{what}: |err| {err[tuple(i)]:.3e} > bound {bound[tuple(i)]:.3e} at {tuple(i)}"
                             f" ({bad.sum()} of {bad.size})")
    e = oracle.rel_errors(got, exact)
    assert e["normwise"] <= slack * gamma(K + 2), (what, e)
