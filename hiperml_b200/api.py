"""Python host side of the skinny SGEMM/SGEMV path.

Two layers, both thin over the C ABI (``include/hml_b200.h``):

* the reference's interface, same names and argument meaning as
  ``include/hml_sgemm.h`` / ``include/hml_sgemv.h`` of the reference:
  ``hmlSgemm(C, A, B, M, N, K, alpha, beta)`` etc. on host (numpy) arrays,
  row-major, C updated in place.  Where the reference prints and calls
  ``exit(1)`` these raise ``HmlError``.
* the device-pointer interface ``sgemm_ex`` / ``sgemv_ex`` (BLAS argument
  order, either storage order, transposes, leading dimensions, a stream),
  taking torch CUDA tensors or raw device addresses.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from ._lib import GemmDesc, SgemmConfig, SgemvTuneEntry, TuneEntry, check, lib

COL_MAJOR, ROW_MAJOR = 0, 1
OP_N, OP_T = 0, 1
ALGO_AUTO, ALGO_SIMT, ALGO_BF16X3, ALGO_BF16X6, ALGO_TF32X3, ALGO_FP16X3 = 0, 1, 2, 3, 4, 5


def _ptr(x) -> Optional[int]:
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    raise TypeError(f"cannot take a pointer of {type(x)}")


def _stream(stream) -> Optional[int]:
    if stream is None:
        try:
            import torch
            if torch.cuda.is_available():
                return torch.cuda.current_stream().cuda_stream
        except ImportError:
            pass
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _host_f32(a, name):
    if not isinstance(a, np.ndarray) or a.dtype != np.float32 or not a.flags["C_CONTIGUOUS"]:
        raise TypeError(f"{name} must be a C-contiguous float32 numpy array")
    return a


# ------------------------------------------------------ reference interface
def hmlSgemmKernelConfig(sgemmKernelConfigFileName: Optional[str]) -> None:
    """``hmlSgemmKernelConfig`` (reference src/hml_sgemm.cu:213-226)."""
    path = None if sgemmKernelConfigFileName is None else sgemmKernelConfigFileName.encode()
    check(lib.hml_config_file(0, path), "hmlSgemmKernelConfig")


def hmlSgemvKernelConfig(sgemvKernelConfigFileName: Optional[str]) -> None:
    """``hmlSgemvKernelConfig`` (reference src/hml_sgemv.cu:215-228)."""
    path = None if sgemvKernelConfigFileName is None else sgemvKernelConfigFileName.encode()
    check(lib.hml_config_file(1, path), "hmlSgemvKernelConfig")


def _host_sgemm(basic, C, A, B, M, N, K, alpha, beta, where):
    C = _host_f32(C, "C")
    A = _host_f32(A, "A")
    B = _host_f32(B, "B")
    if C.size < M * N or A.size < M * K or B.size < K * N:
        raise ValueError(f"{where}: arrays smaller than the M, N, K they are given with")
    check(lib.hml_host_sgemm(basic, C.ctypes.data, A.ctypes.data, B.ctypes.data, M, N, K,
                             alpha, beta), where)


def hmlSgemm(C, A, B, M, N, K, alpha, beta) -> None:
    """C = alpha*A*B + beta*C, host arrays, row-major, C updated in place
    (reference src/hml_sgemm.cu:120-211)."""
    _host_sgemm(0, C, A, B, M, N, K, alpha, beta, "hmlSgemm")


def hmlSgemmBasic(C, A, B, M, N, K, alpha, beta) -> None:
    """Same with the default configuration (reference src/hml_sgemm.cu:39-113)."""
    _host_sgemm(1, C, A, B, M, N, K, alpha, beta, "hmlSgemmBasic")


def _host_sgemv(basic, y, A, x, M, N, alpha, beta, where):
    y = _host_f32(y, "y")
    A = _host_f32(A, "A")
    x = _host_f32(x, "x")
    if y.size < M or A.size < M * N or x.size < N:
        raise ValueError(f"{where}: arrays smaller than the M, N they are given with")
    check(lib.hml_host_sgemv(basic, y.ctypes.data, A.ctypes.data, x.ctypes.data, M, N,
                             alpha, beta), where)


def hmlSgemv(y, A, x, M, N, alpha, beta) -> None:
    """y = alpha*A*x + beta*y, host arrays, A row-major M x N
    (reference src/hml_sgemv.cu:125-213)."""
    _host_sgemv(0, y, A, x, M, N, alpha, beta, "hmlSgemv")


def hmlSgemvBasic(y, A, x, M, N, alpha, beta) -> None:
    """Same with the default kernel (reference src/hml_sgemv.cu:38-118)."""
    _host_sgemv(1, y, A, x, M, N, alpha, beta, "hmlSgemvBasic")


# ---------------------------------------------------- device-pointer layer
def sgemm_ex(order, transA, transB, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc,
             stream=None, config: Optional[SgemmConfig] = None) -> None:
    """``hml_sgemm_ex`` / ``hml_sgemm_ex_config`` on device memory."""
    s = _stream(stream)
    if config is None:
        st = lib.hml_sgemm_ex(order, transA, transB, M, N, K, alpha, _ptr(A), lda, _ptr(B), ldb,
                              beta, _ptr(C), ldc, s)
    else:
        st = lib.hml_sgemm_ex_config(order, transA, transB, M, N, K, alpha, _ptr(A), lda,
                                     _ptr(B), ldb, beta, _ptr(C), ldc, ctypes.byref(config), s)
    check(st, "hml_sgemm_ex")


def sgemv_ex(order, trans, M, N, alpha, A, lda, x, beta, y, stream=None, variant=0) -> None:
    """``hml_sgemv_ex`` on device memory (``variant`` forces a kernel shape)."""
    s = _stream(stream)
    if variant:
        st = lib.hml_sgemv_ex_variant(order, trans, M, N, alpha, _ptr(A), lda, _ptr(x), beta,
                                      _ptr(y), variant, s)
    else:
        st = lib.hml_sgemv_ex(order, trans, M, N, alpha, _ptr(A), lda, _ptr(x), beta, _ptr(y), s)
    check(st, "hml_sgemv_ex")


def _blas_view(t):
    """(order, ld) of a 2-D torch tensor that is column- or row-major dense
    along one dimension."""
    r, c = t.shape
    s0, s1 = t.stride()
    if s0 == 1 and (s1 >= max(1, r) or c == 1):
        return COL_MAJOR, max(1, s1 if c > 1 else r)
    if s1 == 1 and (s0 >= max(1, c) or r == 1):
        return ROW_MAJOR, max(1, s0 if r > 1 else c)
    raise ValueError("tensor must have one unit stride")


def sgemm(A, B, C=None, alpha=1.0, beta=0.0, config=None, stream=None):
    """C = alpha*A@B + beta*C for FP32 CUDA tensors of either storage order.
    Returns C (allocated column-major when not given)."""
    import torch
    M, K = A.shape
    K2, N = B.shape
    if K != K2:
        raise ValueError("inner dimensions differ")
    if C is None:
        C = torch.empty((N, M), dtype=torch.float32, device=A.device).t()
        beta = 0.0
    oc, ldc = _blas_view(C)
    # express A and B in C's storage order, transposing as needed
    def op(t):
        o, ld = _blas_view(t)
        return (OP_N if o == oc else OP_T), ld
    ta, lda = op(A)
    tb, ldb = op(B)
    sgemm_ex(oc, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, stream=stream,
             config=config)
    return C


def select(order, transA, transB, M, N, K) -> SgemmConfig:
    c = SgemmConfig()
    check(lib.hml_sgemm_select(order, transA, transB, M, N, K, ctypes.byref(c)), "hml_sgemm_select")
    return c


def select_algo(order, transA, transB, M, N, K, algo) -> SgemmConfig:
    """The heuristic configuration of one algorithm family."""
    c = SgemmConfig()
    check(lib.hml_sgemm_select_algo(order, transA, transB, M, N, K, algo, ctypes.byref(c)),
          "hml_sgemm_select_algo")
    return c


def configs():
    """The autotuner's configuration space."""
    out = []
    for i in range(lib.hml_sgemm_num_configs()):
        c = SgemmConfig()
        check(lib.hml_sgemm_get_config(i, ctypes.byref(c)), "hml_sgemm_get_config")
        out.append(c)
    return out


def config_check(order, transA, transB, M, N, K, lda, ldb, ldc, config) -> int:
    return lib.hml_sgemm_config_check(order, transA, transB, M, N, K, lda, ldb, ldc,
                                      ctypes.byref(config))


def fill_random(t, seed: int, stream_id: int, dist: int = 0, stream=None) -> None:
    """Fill a float32 CUDA tensor with the SplitMix64 stream of
    ``hiperml_b200.datagen`` (storage order)."""
    check(lib.hml_fill_random(_ptr(t), t.numel(), seed, stream_id, dist, _stream(stream)),
          "hml_fill_random")


def error_fp64(order, transA, transB, M, N, K, alpha, A, lda, B, ldb, beta, C0, C, ldc,
               stream=None):
    """FP64 check on the GPU: (normwise, rms, componentwise, max|C64|)."""
    err = (ctypes.c_double * 4)()
    check(lib.hml_sgemm_error_fp64(order, transA, transB, M, N, K, alpha, _ptr(A), lda, _ptr(B),
                                   ldb, beta, _ptr(C0), _ptr(C), ldc, err, _stream(stream)),
          "hml_sgemm_error_fp64")
    return tuple(err)


KMEANS_AUTO, KMEANS_TILED, KMEANS_GEMM, KMEANS_TENSOR = 0, 1, 2, 3


def kmeans_assign(points, centroids, out=None, stream=None, count_exact=False,
                  method=KMEANS_AUTO):
    """Nearest-centroid index of every point (``hml_kmeans_assign_ex``):
    points (n x d) and centroids (k x d) are row-major float32 CUDA tensors;
    returns an int32 tensor of n indices (the reference kernel's, bit for
    bit), and with ``count_exact`` also the number of points whose candidates
    were resolved with the reference's own arithmetic.  ``method``: 0 = the
    library's choice, 1 = the tiled SIMT form with the argmin fused, 2 = the
    SGEMM form (products through HBM), 3 = the tensor-core form (TF32X3
    products in TMEM, the argmin read from the accumulator; 4 <= d <= 64 with
    d a multiple of 4, at most 256 centroids)."""
    import torch
    n, d = points.shape
    k, d2 = centroids.shape
    if d != d2:
        raise ValueError("points and centroids differ in dimension")
    if not (points.is_contiguous() and centroids.is_contiguous()):
        raise ValueError("points and centroids must be row-major contiguous")
    if out is None:
        out = torch.empty(n, dtype=torch.int32, device=points.device)
    cnt = torch.zeros(1, dtype=torch.int32, device=points.device) if count_exact else None
    check(lib.hml_kmeans_assign_ex(_ptr(points), n, d, _ptr(centroids), k, _ptr(out), method,
                                   _ptr(cnt) if cnt is not None else None, _stream(stream)),
          "hml_kmeans_assign_ex")
    if count_exact:
        return out, int(cnt.item())
    return out


def device_error() -> int:
    code = ctypes.c_int()
    check(lib.hml_device_error(ctypes.byref(code)), "hml_device_error")
    return code.value


def check_wait_limit(stream=None) -> None:
    """``hml_check_wait_limit``: a kernel whose bounded wait expires."""
    check(lib.hml_check_wait_limit(_stream(stream)), "hml_check_wait_limit")


# ------------------------------------------------------------- autotuning
MATH_FP32, MATH_FAST = 0, 1


def autotune(order, transA, transB, M, N, K, families=0, reps=5, stream=None):
    """Measure the configuration space on this shape (``hml_autotune_sgemm``).
    Returns a list of (SgemmConfig, time_us, status); the fastest allowed
    configuration is recorded in the library's tuned table."""
    cap = lib.hml_sgemm_num_configs()
    ents = (TuneEntry * cap)()
    n = ctypes.c_int()
    st = lib.hml_autotune_sgemm(order, transA, transB, M, N, K, families, reps, ents, cap,
                                ctypes.byref(n), _stream(stream))
    check(st, "hml_autotune_sgemm")
    return [(ents[i].config, ents[i].time_us, ents[i].status) for i in range(n.value)]


def autotune_sgemv(order, trans, M, N, reps=5, stream=None):
    """Measure every variant of the SGEMV kernel for this layout on an M x N
    problem (``hml_autotune_sgemv``).  Returns a list of (variant, time_us,
    status); the fastest is recorded in the library's tuned table."""
    ents = (SgemvTuneEntry * 32)()
    n = ctypes.c_int()
    st = lib.hml_autotune_sgemv(order, trans, M, N, reps, ents, 32, ctypes.byref(n),
                                _stream(stream))
    check(st, "hml_autotune_sgemv")
    return [(ents[i].variant, ents[i].time_us, ents[i].status) for i in range(n.value)]


def sgemv_select(order, trans, M, N, lda=None) -> int:
    """The variant ``hml_sgemv_ex`` runs this problem with: the tuned table's,
    or 0 when the heuristic decides (``hml_sgemv_select``)."""
    if lda is None:
        lda = max(1, M if order == COL_MAJOR else N)
    v = ctypes.c_int()
    check(lib.hml_sgemv_select(order, trans, M, N, lda, ctypes.byref(v)), "hml_sgemv_select")
    return v.value


def tune_save(path: str) -> None:
    check(lib.hml_tune_save(path.encode()), "hml_tune_save")


def tune_load(path: str) -> int:
    n = ctypes.c_int()
    check(lib.hml_tune_load(path.encode(), ctypes.byref(n)), "hml_tune_load")
    return n.value


def tune_clear() -> None:
    check(lib.hml_tune_clear(), "hml_tune_clear")


def set_math_mode(mode: int) -> None:
    check(lib.hml_set_math_mode(mode), "hml_set_math_mode")


# ----------------------------------------------------------------- batched
def gemm_descs(problems):
    """ctypes array of ``hml_gemm_desc`` from tuples
    (transA, transB, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc); A, B, C
    are device pointers (ints) or CUDA tensors."""
    arr = (GemmDesc * max(1, len(problems)))()
    for i, (ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc) in enumerate(problems):
        arr[i] = GemmDesc(ta, tb, M, N, K, lda, ldb, ldc, alpha, beta, _ptr(A), _ptr(B), _ptr(C))
    return arr


class BatchPlan:
    """``hml_batch_plan``: a batch of SGEMMs run by one persistent launch."""

    def __init__(self, order, problems):
        self._descs = gemm_descs(problems)
        h = ctypes.c_void_p()
        check(lib.hml_batch_plan_create(order, self._descs, len(problems), ctypes.byref(h)),
              "hml_batch_plan_create")
        self._h = h

    def run(self, stream=None):
        check(lib.hml_batch_plan_run(self._h, _stream(stream)), "hml_batch_plan_run")

    def graph_launch(self, stream=None):
        check(lib.hml_batch_plan_graph_launch(self._h, _stream(stream)),
              "hml_batch_plan_graph_launch")

    def info(self):
        t, c = ctypes.c_int(), ctypes.c_int()
        f, b = ctypes.c_double(), ctypes.c_double()
        check(lib.hml_batch_plan_info(self._h, ctypes.byref(t), ctypes.byref(c), ctypes.byref(f),
                                      ctypes.byref(b)), "hml_batch_plan_info")
        return {"tiles": t.value, "ctas": c.value, "flops": f.value, "bytes": b.value}

    def close(self):
        if self._h:
            lib.hml_batch_plan_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_problem_config(order, problem) -> SgemmConfig:
    """``hml_batch_problem_config``: the configuration a batch runs this
    problem (one descriptor tuple, as for ``BatchPlan``) with."""
    descs = gemm_descs([problem])
    c = SgemmConfig()
    check(lib.hml_batch_problem_config(order, descs, ctypes.byref(c)), "hml_batch_problem_config")
    return c


def sgemm_batched(order, problems, stream=None):
    """``hml_sgemm_batched``: one-shot batch, stream ordered."""
    descs = gemm_descs(problems)
    check(lib.hml_sgemm_batched(order, descs, len(problems), _stream(stream)), "hml_sgemm_batched")
