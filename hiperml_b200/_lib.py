"""ctypes binding of ``libhml_b200.so`` (the C ABI in ``include/hml_b200.h``).

The library is built in-tree by ``make -C hiperml_b200/csrc`` (or
``__graft_entry__.build()``).  Importing this module without it raises
``ImportError``: there is no fallback implementation of any entry point.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhml_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `make -C {os.path.join(_HERE, 'csrc')} -j` "
        "(the SGEMM/SGEMV path has no CPU fallback)")

lib = ctypes.CDLL(LIB_PATH)

c_int, c_float, c_double, c_void_p = ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_void_p
c_size_t, c_uint64, c_char_p = ctypes.c_size_t, ctypes.c_uint64, ctypes.c_char_p
c_int_p = ctypes.POINTER(ctypes.c_int)


class SgemmConfig(ctypes.Structure):
    """``hml_sgemm_config``."""
    _fields_ = [("algo", ctypes.c_int32), ("tile_m", ctypes.c_int32), ("tile_n", ctypes.c_int32),
                ("split_k", ctypes.c_int32), ("stages", ctypes.c_int32), ("variant", ctypes.c_int32)]

    def as_tuple(self):
        return (self.algo, self.tile_m, self.tile_n, self.split_k, self.stages, self.variant)

    def __repr__(self):
        names = {0: "AUTO", 1: "SIMT", 2: "BF16X3", 3: "BF16X6", 4: "TF32X3", 5: "FP16X3"}
        return (f"SgemmConfig({names.get(self.algo, self.algo)}, {self.tile_m}x{self.tile_n}, "
                f"split_k={self.split_k}, stages={self.stages}, variant={self.variant})")


class TuneEntry(ctypes.Structure):
    """``hml_tune_entry``."""
    _fields_ = [("config", SgemmConfig), ("time_us", ctypes.c_float), ("status", ctypes.c_int32)]


class SgemvTuneEntry(ctypes.Structure):
    """``hml_sgemv_tune_entry``."""
    _fields_ = [("variant", ctypes.c_int32), ("time_us", ctypes.c_float),
                ("status", ctypes.c_int32)]


class GemmDesc(ctypes.Structure):
    """``hml_gemm_desc``: one problem of a batch (device pointers)."""
    _fields_ = [("transA", ctypes.c_int32), ("transB", ctypes.c_int32), ("M", ctypes.c_int32),
                ("N", ctypes.c_int32), ("K", ctypes.c_int32), ("lda", ctypes.c_int32),
                ("ldb", ctypes.c_int32), ("ldc", ctypes.c_int32), ("alpha", ctypes.c_float),
                ("beta", ctypes.c_float), ("A", ctypes.c_void_p), ("B", ctypes.c_void_p),
                ("C", ctypes.c_void_p)]


class PredictorOptions(ctypes.Structure):
    """``hml_predictor_options``."""
    _fields_ = [("epochs", ctypes.c_int32), ("batch", ctypes.c_int32), ("lr", ctypes.c_float),
                ("weight_decay", ctypes.c_float), ("target_clip", ctypes.c_float),
                ("seed", ctypes.c_uint64)]


_SIGS = {
    "hml_status_string": (c_char_p, [c_int]),
    "hml_version": (c_char_p, []),
    "hml_last_error": (c_char_p, []),
    "hml_sgemm_ex": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int, c_float, c_void_p, c_int,
                             c_void_p, c_int, c_float, c_void_p, c_int, c_void_p]),
    "hml_sgemm_ex_config": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int, c_float, c_void_p,
                                    c_int, c_void_p, c_int, c_float, c_void_p, c_int,
                                    ctypes.POINTER(SgemmConfig), c_void_p]),
    "hml_sgemm_select": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int,
                                 ctypes.POINTER(SgemmConfig)]),
    "hml_sgemm_select_algo": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int, c_int,
                                      ctypes.POINTER(SgemmConfig)]),
    "hml_sgemm_config_check": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_int,
                                       c_int, ctypes.POINTER(SgemmConfig)]),
    "hml_sgemm_num_configs": (c_int, []),
    "hml_sgemm_get_config": (c_int, [c_int, ctypes.POINTER(SgemmConfig)]),
    "hml_sgemm_config_index": (c_int, [ctypes.POINTER(SgemmConfig)]),
    "hml_sgemv_ex": (c_int, [c_int, c_int, c_int, c_int, c_float, c_void_p, c_int, c_void_p,
                             c_float, c_void_p, c_void_p]),
    "hml_sgemv_ex_variant": (c_int, [c_int, c_int, c_int, c_int, c_float, c_void_p, c_int,
                                     c_void_p, c_float, c_void_p, c_int, c_void_p]),
    "hml_host_sgemm": (c_int, [c_int, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_float,
                               c_float]),
    "hml_host_sgemv": (c_int, [c_int, c_void_p, c_void_p, c_void_p, c_int, c_int, c_float,
                               c_float]),
    "hml_config_file": (c_int, [c_int, c_char_p]),
    "hml_cfg_v1_load": (c_int, [c_int, c_char_p, c_int_p]),
    "hml_cfg_v1_sgemm_rule": (c_int, [c_int, c_int, c_int_p, c_int_p]),
    "hml_cfg_v1_sgemv_rule": (c_int, [c_int, c_int_p, c_int_p, c_int_p]),
    "hml_cfg_v1_clear": (None, []),
    "hml_cfg_v1_save": (c_int, [c_int, c_char_p]),
    "hml_sgemm_v1_config": (c_int, [c_int, c_int, c_int, ctypes.POINTER(SgemmConfig)]),
    "hml_fill_random": (c_int, [c_void_p, c_size_t, c_uint64, c_uint64, c_int, c_void_p]),
    "hml_kmeans_assign": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int, c_void_p, c_void_p]),
    "hml_kmeans_assign_ex": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int, c_void_p, c_int,
                                     c_void_p, c_void_p]),
    "hml_sgemm_error_fp64": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int, c_float, c_void_p,
                                     c_int, c_void_p, c_int, c_float, c_void_p, c_void_p, c_int,
                                     ctypes.POINTER(c_double), c_void_p]),
    "hml_device_error": (c_int, [c_int_p]),
    "hml_check_wait_limit": (c_int, [c_void_p]),
    "hml_release_resources": (c_int, []),
    "hml_launch_count": (c_uint64, []),
    "hml_autotune_sgemm": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int, ctypes.c_uint32,
                                   c_int, ctypes.POINTER(TuneEntry), c_int, c_int_p, c_void_p]),
    "hml_autotune_sgemv": (c_int, [c_int, c_int, c_int, c_int, c_int,
                                   ctypes.POINTER(SgemvTuneEntry), c_int, c_int_p, c_void_p]),
    "hml_sgemv_select": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int_p]),
    "hml_tune_save": (c_int, [c_char_p]),
    "hml_tune_load": (c_int, [c_char_p, c_int_p]),
    "hml_tune_clear": (c_int, []),
    "hml_tune_size": (c_int, []),
    "hml_set_math_mode": (c_int, [c_int]),
    "hml_batch_plan_create": (c_int, [c_int, ctypes.POINTER(GemmDesc), c_int,
                                      ctypes.POINTER(c_void_p)]),
    "hml_batch_plan_run": (c_int, [c_void_p, c_void_p]),
    "hml_batch_plan_graph_launch": (c_int, [c_void_p, c_void_p]),
    "hml_batch_plan_info": (c_int, [c_void_p, c_int_p, c_int_p, ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_double)]),
    "hml_batch_plan_destroy": (c_int, [c_void_p]),
    "hml_sgemm_batched": (c_int, [c_int, ctypes.POINTER(GemmDesc), c_int, c_void_p]),
    "hml_batch_problem_config": (c_int, [c_int, ctypes.POINTER(GemmDesc),
                                         ctypes.POINTER(SgemmConfig)]),
    "hml_predictor_train": (c_int, [c_int, c_void_p, c_void_p, c_int, ctypes.POINTER(SgemmConfig),
                                    c_int, ctypes.POINTER(PredictorOptions), c_void_p]),
    "hml_predictor_loss_grad": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_int,
                                        c_void_p, c_void_p]),
    "hml_predictor_predict_batch": (c_int, [c_int, c_void_p, c_int, c_void_p]),
    "hml_predictor_save": (c_int, [c_char_p]),
    "hml_predictor_load": (c_int, [c_char_p]),
    "hml_predictor_clear": (c_int, []),
    "hml_predictor_outputs": (c_int, []),
    "hml_predictor_params": (c_int, [c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "hml_predictor_features": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int, c_void_p]),
}

for _name, (_res, _args) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


def bind(name, restype, argtypes):
    """Declare a further entry point (used by modules that add to the ABI)."""
    f = getattr(lib, name)
    f.restype = restype
    f.argtypes = argtypes
    return f


class HmlError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        msg = lib.hml_status_string(status).decode()
        extra = lib.hml_last_error().decode()
        super().__init__(f"{where}: {msg}" + (f" ({extra})" if extra else ""))


def check(status: int, where: str) -> None:
    if status != 0:
        raise HmlError(status, where)
