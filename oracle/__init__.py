"""CPU oracle for the skinny SGEMM/SGEMV path -- TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker.  The product
library (``hiperml_b200``) never imports, links or runs anything here.

Two native libraries back it (built by ``oracle/Makefile``):

* ``_build/libhml_oracle.so`` -- the C restatement (``hml_oracle.c``):
  FP32 row-major loops with the reference's exact summation order
  (``apps/gemm/hml_sgemm_main.cu:260-292``, ``apps/gemv/hml_sgemv_main.cu:254-283``),
  the double checksum (``apps/gemm/hml_sgemm_main.cu:294-305``) and a
  multithreaded FP64 GEMM over arbitrary strides.
* ``_ref/libhml_ref_cpu.so`` -- the reference's own ``hmlSgemmCpu`` /
  ``hmlSgemvCpu`` / ``hmlComputeCsum`` / ``hmlComputeYsum`` compiled from its
  unmodified sources.  It pins the restatement bit for bit.
* ``_ref/libhml_ref_gpu_{sgemm,sgemv}.so`` -- the reference's own GPU kernel
  repositories and selectors, compiled from its unmodified sources with the
  texture stand-in of ``ref_gpu_compat.h`` (``make -C oracle refgpu``): the
  GPU baseline and a second parity target.
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_c_float_p = ctypes.POINTER(ctypes.c_float)
_c_double_p = ctypes.POINTER(ctypes.c_double)

_lib = None
_ref = None


def _load(path):
    if not os.path.exists(path):
        raise OSError(f"oracle library missing: {path} (run `make -C oracle`)")
    return ctypes.CDLL(path)


def lib():
    global _lib
    if _lib is None:
        L = _load(os.path.join(_HERE, "_build", "libhml_oracle.so"))
        L.oracle_sgemm_rm_f32.argtypes = [_c_float_p, _c_float_p, _c_float_p,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_float, ctypes.c_float]
        L.oracle_sgemm_rm_f32.restype = None
        L.oracle_sgemm_rm_f32_mt.argtypes = L.oracle_sgemm_rm_f32.argtypes + [ctypes.c_int]
        L.oracle_sgemm_rm_f32_mt.restype = ctypes.c_int
        L.oracle_sgemv_rm_f32.argtypes = [_c_float_p, _c_float_p, _c_float_p,
                                          ctypes.c_int, ctypes.c_int,
                                          ctypes.c_float, ctypes.c_float]
        L.oracle_sgemv_rm_f32.restype = None
        L.oracle_csum.argtypes = [_c_float_p, ctypes.c_int, ctypes.c_int]
        L.oracle_csum.restype = ctypes.c_double
        i64 = ctypes.c_int64
        L.oracle_dgemm_strided.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_double, _c_float_p, i64, i64,
                                           _c_float_p, i64, i64, ctypes.c_double,
                                           _c_float_p, i64, i64, _c_double_p,
                                           _c_double_p, ctypes.c_int]
        L.oracle_dgemm_strided.restype = ctypes.c_int
        L.oracle_kmeans_assign.argtypes = [_c_float_p, ctypes.c_int64, ctypes.c_int, _c_float_p,
                                           ctypes.c_int, ctypes.POINTER(ctypes.c_uint32)]
        L.oracle_kmeans_assign.restype = None
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(os.path.join(_HERE, "_ref", "libhml_ref_cpu.so"))


def ref():
    """The reference's own CPU loops (C++ linkage, mangled names)."""
    global _ref
    if _ref is None:
        R = _load(os.path.join(_HERE, "_ref", "libhml_ref_cpu.so"))
        f = getattr(R, "_Z11hmlSgemmCpuPfPKfS1_iiiff")
        f.argtypes = [_c_float_p, _c_float_p, _c_float_p, ctypes.c_int,
                      ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float]
        f.restype = None
        g = getattr(R, "_Z11hmlSgemvCpuPfPKfS1_iiff")
        g.argtypes = [_c_float_p, _c_float_p, _c_float_p, ctypes.c_int,
                      ctypes.c_int, ctypes.c_float, ctypes.c_float]
        g.restype = None
        cs = getattr(R, "_Z14hmlComputeCsumPfii")
        cs.argtypes = [_c_float_p, ctypes.c_int, ctypes.c_int]
        cs.restype = ctypes.c_double
        ys = getattr(R, "_Z14hmlComputeYsumPfi")
        ys.argtypes = [_c_float_p, ctypes.c_int]
        ys.restype = ctypes.c_double
        R.sgemm_cpu, R.sgemv_cpu, R.csum, R.ysum = f, g, cs, ys
        _ref = R
    return _ref


_ref_gpu = {}


def ref_gpu_available() -> bool:
    return all(os.path.exists(os.path.join(_HERE, "_ref", f"libhml_ref_gpu_{k}.so"))
               for k in ("sgemm", "sgemv"))


def ref_gpu(kind):
    """The reference's own GPU kernels and selectors (kind 'sgemm' or
    'sgemv'), built from its sources by `make -C oracle refgpu`; entry points
    of oracle/ref_gpu_harness.cu on device pointers (ints)."""
    if kind not in _ref_gpu:
        L = _load(os.path.join(_HERE, "_ref", f"libhml_ref_gpu_{kind}.so"))
        vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        ip = ctypes.POINTER(ctypes.c_int)
        if kind == "sgemm":
            L.ref_gpu_sgemm_config.argtypes = [ctypes.c_char_p]
            L.ref_gpu_sgemm_select.argtypes = [i, i, i, ip, ip, ip]
            L.ref_gpu_sgemm.argtypes = [vp, vp, vp, i, i, i, f, f, i, ctypes.POINTER(f)]
        else:
            L.ref_gpu_sgemv_config.argtypes = [ctypes.c_char_p]
            L.ref_gpu_sgemv_select.argtypes = [i, i, ip, ip, ip]
            L.ref_gpu_sgemv.argtypes = [vp, vp, vp, i, i, f, f, i, ctypes.POINTER(f)]
        _ref_gpu[kind] = L
    return _ref_gpu[kind]


def ref_gpu_sgemm(C, A, B, M, N, K, alpha, beta, reps=1):
    """hmlSgemm's kernel on device pointers (row-major); returns ms per launch."""
    ms = ctypes.c_float()
    with _QuietStderr():
        rc = ref_gpu("sgemm").ref_gpu_sgemm(C, A, B, M, N, K, alpha, beta, reps, ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError(f"reference SGEMM kernel: CUDA status {rc}")
    return ms.value


def ref_gpu_sgemv(y, A, x, M, N, alpha, beta, reps=1):
    """hmlSgemv's kernel on device pointers (A row-major M x N)."""
    ms = ctypes.c_float()
    with _QuietStderr():
        rc = ref_gpu("sgemv").ref_gpu_sgemv(y, A, x, M, N, alpha, beta, reps, ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError(f"reference SGEMV kernel: CUDA status {rc}")
    return ms.value


def ref_gpu_select(kind, *shape):
    """(is_const, grid, block) of the kernel the loaded rules pick."""
    c = ctypes.c_int()
    g = (ctypes.c_int * 3)()
    b = (ctypes.c_int * 3)()
    fn = ref_gpu(kind).ref_gpu_sgemm_select if kind == "sgemm" else \
        ref_gpu(kind).ref_gpu_sgemv_select
    with _QuietStderr():
        rc = fn(*shape, ctypes.byref(c), g, b)
    if rc != 0:
        raise RuntimeError("reference selector: no rules loaded")
    return bool(c.value), tuple(g), tuple(b)


def ref_gpu_load_rules(kind, path):
    """hmlSgemmKernelConfigReadFile / hmlSgemvKernelConfigReadFile."""
    fn = ref_gpu(kind).ref_gpu_sgemm_config if kind == "sgemm" else \
        ref_gpu(kind).ref_gpu_sgemv_config
    with _QuietStderr():
        rc = fn(str(path).encode())
    if rc != 0:
        raise RuntimeError(f"reference {kind} rules not loaded from {path}")


def _fp(a):
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_c_float_p)


class _QuietStderr:
    """Silences fd 2 while the reference loops print their timing lines."""

    def __enter__(self):
        sys.stderr.flush()
        self._saved = os.dup(2)
        self._null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self._null, 2)

    def __exit__(self, *exc):
        os.dup2(self._saved, 2)
        os.close(self._saved)
        os.close(self._null)


# ---------------------------------------------------------------- restatement
def sgemm_rm_f32(A, B, C=None, alpha=1.0, beta=0.0, threads=1):
    """Row-major NN SGEMM with the reference loop's rounding (hml_oracle.c)."""
    A = np.ascontiguousarray(A, np.float32)
    B = np.ascontiguousarray(B, np.float32)
    M, K = A.shape
    K2, N = B.shape
    assert K == K2
    out = np.zeros((M, N), np.float32) if C is None else np.array(C, np.float32, order="C")
    if threads > 1:
        lib().oracle_sgemm_rm_f32_mt(_fp(out), _fp(A), _fp(B), M, N, K, alpha, beta, threads)
    else:
        lib().oracle_sgemm_rm_f32(_fp(out), _fp(A), _fp(B), M, N, K, alpha, beta)
    return out


def sgemv_rm_f32(A, x, y=None, alpha=1.0, beta=0.0):
    A = np.ascontiguousarray(A, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    M, N = A.shape
    out = np.zeros(M, np.float32) if y is None else np.array(y, np.float32)
    lib().oracle_sgemv_rm_f32(_fp(out), _fp(A), _fp(x), M, N, alpha, beta)
    return out


def csum(C):
    C = np.ascontiguousarray(C, np.float32)
    M = C.shape[0]
    N = C.shape[1] if C.ndim == 2 else 1
    return lib().oracle_csum(_fp(C), M, N)


def dgemm(A, B, C=None, alpha=1.0, beta=0.0, transA=False, transB=False,
          with_abs=False, threads=None):
    """FP64 C = alpha*op(A)@op(B) + beta*C on float32 numpy arrays of any
    memory order.  Returns (D, absD or None) as float64 (M, N) arrays."""
    A = np.asarray(A, np.float32)
    B = np.asarray(B, np.float32)
    opA = A.T if transA else A
    opB = B.T if transB else B
    M, K = opA.shape
    K2, N = opB.shape
    assert K == K2
    isz = 4
    sam, sak = opA.strides[0] // isz, opA.strides[1] // isz
    sbk, sbn = opB.strides[0] // isz, opB.strides[1] // isz
    # the C routine wants non-negative strides from a base pointer
    for s in (sam, sak, sbk, sbn):
        assert s >= 0
    D = np.empty((N, M), np.float64)  # column-major (M, N) buffer
    absD = np.empty((N, M), np.float64) if with_abs else None
    if C is not None and beta != 0.0:
        C = np.asarray(C, np.float32)
        scm, scn = C.strides[0] // isz, C.strides[1] // isz
        cptr = C.ctypes.data_as(_c_float_p)
    else:
        scm = scn = 0
        cptr = None
    if threads is None:
        threads = os.cpu_count() or 1
    rc = lib().oracle_dgemm_strided(
        M, N, K, float(alpha), opA.ctypes.data_as(_c_float_p), sam, sak,
        opB.ctypes.data_as(_c_float_p), sbk, sbn, float(beta), cptr, scm, scn,
        D.ctypes.data_as(_c_double_p),
        absD.ctypes.data_as(_c_double_p) if absD is not None else None, threads)
    assert rc == 0
    return D.T, (absD.T if absD is not None else None)


# ------------------------------------------------------------- the reference
def ref_sgemm_cpu(A, B, C=None, alpha=1.0, beta=0.0):
    """The reference's hmlSgemmCpu (apps/gemm/hml_sgemm_main.cu:260-292)."""
    A = np.ascontiguousarray(A, np.float32)
    B = np.ascontiguousarray(B, np.float32)
    M, K = A.shape
    _, N = B.shape
    out = np.zeros((M, N), np.float32) if C is None else np.array(C, np.float32, order="C")
    with _QuietStderr():
        ref().sgemm_cpu(_fp(out), _fp(A), _fp(B), M, N, K, alpha, beta)
    return out


def ref_sgemv_cpu(A, x, y=None, alpha=1.0, beta=0.0):
    """The reference's hmlSgemvCpu (apps/gemv/hml_sgemv_main.cu:254-283)."""
    A = np.ascontiguousarray(A, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    M, N = A.shape
    out = np.zeros(M, np.float32) if y is None else np.array(y, np.float32)
    with _QuietStderr():
        ref().sgemv_cpu(_fp(out), _fp(A), _fp(x), M, N, alpha, beta)
    return out


def ref_csum(C):
    C = np.ascontiguousarray(C, np.float32)
    if C.ndim == 1:
        return ref().ysum(_fp(C), C.shape[0])
    return ref().csum(_fp(C), C.shape[0], C.shape[1])


def kmeans_assign(points, centroids):
    """Nearest-centroid index per point with the reference kernel's
    arithmetic (hml_oracle.c: oracle_kmeans_assign)."""
    P = np.ascontiguousarray(points, np.float32)
    C = np.ascontiguousarray(centroids, np.float32)
    out = np.zeros(P.shape[0], np.uint32)
    lib().oracle_kmeans_assign(_fp(P), P.shape[0], P.shape[1], _fp(C), C.shape[0],
                               out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    return out


def ref_gpu_kmeans_available() -> bool:
    return os.path.exists(os.path.join(_HERE, "_ref", "libhml_ref_gpu_kmeans.so"))


def ref_gpu_kmeans_assign(asg, rows, n, ctrds, k, d, reps=1):
    """The reference's hmlKmeansAssignCtrdSmem on device pointers (ints);
    returns ms per launch."""
    if "kmeans" not in _ref_gpu:
        L = _load(os.path.join(_HERE, "_ref", "libhml_ref_gpu_kmeans.so"))
        vp, u = ctypes.c_void_p, ctypes.c_uint32
        L.ref_gpu_kmeans_assign.argtypes = [vp, vp, u, vp, u, u, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_float)]
        _ref_gpu["kmeans"] = L
    ms = ctypes.c_float()
    rc = _ref_gpu["kmeans"].ref_gpu_kmeans_assign(asg, rows, n, ctrds, k, d, reps,
                                                  ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError(f"reference k-means kernel: CUDA status {rc}")
    return ms.value


def rel_errors(approx, exact, absbound=None):
    """Error metrics used by every parity check in this repository.

    * ``normwise``  = max|approx-exact| / max|exact|
    * ``rms``       = ||approx-exact||_2 / ||exact||_2
    * ``compwise``  = max |approx-exact| / (|A||B|)_ij (needs absbound)
    """
    approx = np.asarray(approx, np.float64)
    exact = np.asarray(exact, np.float64)
    d = np.abs(approx - exact)
    den = np.max(np.abs(exact)) if exact.size else 0.0
    out = {
        "normwise": float(d.max() / den) if den > 0 else float(d.max() if d.size else 0.0),
        "rms": float(np.sqrt((d ** 2).sum()) / max(np.sqrt((exact ** 2).sum()), 1e-300)),
    }
    if absbound is not None:
        ab = np.asarray(absbound, np.float64)
        with np.errstate(divide="ignore", invalid="ignore"):
            r = np.where(ab > 0, d / ab, 0.0)
        out["compwise"] = float(r.max()) if r.size else 0.0
    return out
