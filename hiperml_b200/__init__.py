"""hiperml_b200 -- HiperML's skinny SGEMM/SGEMV path rebuilt for NVIDIA B200.

The compute lives in ``libhml_b200.so`` (hand-written sm_100a CUDA behind
the C ABI of ``include/hml_b200.h``); this package is its Python host side.
Importing it fails when the library has not been built: there is no CPU
fallback for any entry point.
"""
from ._lib import HmlError, SgemmConfig, lib  # noqa: F401  (loads the .so)
from .api import (  # noqa: F401
    ALGO_AUTO, ALGO_BF16X3, ALGO_BF16X6, ALGO_FP16X3, ALGO_SIMT, ALGO_TF32X3, COL_MAJOR, OP_N, OP_T, ROW_MAJOR,
    check_wait_limit, config_check, configs, device_error, error_fp64, fill_random, hmlSgemm,
    hmlSgemmBasic,
    hmlSgemmKernelConfig, hmlSgemv, hmlSgemvBasic, hmlSgemvKernelConfig, select, select_algo, sgemm,
    sgemm_ex, sgemv_ex, autotune, autotune_sgemv, sgemv_select, tune_save, tune_load, tune_clear,
    set_math_mode, MATH_FP32, MATH_FAST, BatchPlan, gemm_descs, sgemm_batched, batch_problem_config,
    kmeans_assign, KMEANS_AUTO, KMEANS_TILED, KMEANS_GEMM, KMEANS_TENSOR)

__version__ = lib.hml_version().decode()
