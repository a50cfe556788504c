"""Generates the golden vectors in this directory from the reference itself.

Run in the development container (where the reference tree and the prebuilt
``oracle/_ref/libhml_ref_cpu.so`` exist):

    python tests/golden/make_golden.py

Inputs are not stored: every case records the (seed, stream, distribution,
storage order) of ``hiperml_b200.datagen`` that regenerates them.  Outputs
are those of the reference's own CPU verification loops ``hmlSgemmCpu`` /
``hmlSgemvCpu`` (apps/gemm/hml_sgemm_main.cu:260-292,
apps/gemv/hml_sgemv_main.cu:254-283) compiled from its sources, together with
the reference checksum ``hmlComputeCsum`` / ``hmlComputeYsum``.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from hiperml_b200 import datagen as dg  # noqa: E402  (pure numpy module)

# name, M, N, K, alpha, beta, seed, dist  (row-major, the reference's layout)
SGEMM = [
    ("k_lt_16", 37, 5, 19, 0.7, -1.3, 11, dg.UNIFORM),
    ("n16_k96", 128, 16, 96, 1.0, 0.0, 12, dg.UNIFORM),
    ("ragged", 300, 40, 333, 1.5, 0.5, 13, dg.UNIFORM),
    ("n_gt_96", 129, 100, 50, -1.0, 1.0, 14, dg.NORMAL),
    ("unit", 1, 1, 1, 2.0, 0.0, 15, dg.UNIFORM),
    ("k1", 5, 3, 1, 1.0, 0.25, 16, dg.UNIFORM),
    ("m1", 1, 7, 64, 1.0, 0.0, 17, dg.UNIFORM),
    ("n1", 257, 1, 129, 1.0, 0.0, 18, dg.UNIFORM),
    ("loguniform", 200, 24, 512, 1.0, 0.0, 19, dg.LOGUNIFORM),
    ("tall_n8", 2048, 8, 1000, 1.0, 0.0, 20, dg.UNIFORM),
]

# name, M, N, alpha, beta, seed, dist (row-major y = alpha*A*x + beta*y)
SGEMV = [
    ("small", 37, 19, 0.5, 2.0, 31, dg.UNIFORM),
    ("one_col", 1000, 1, 1.0, 0.0, 32, dg.UNIFORM),
    ("one_row", 1, 1000, 1.0, 0.0, 33, dg.UNIFORM),
    ("ragged", 513, 257, -1.0, 1.0, 34, dg.NORMAL),
    ("wide", 64, 5000, 1.0, 0.0, 35, dg.NORMAL),
]


def sgemm_inputs(M, N, K, seed, dist):
    A = dg.matrix(M, K, seed, 0, dist, order="C")
    B = dg.matrix(K, N, seed, 1, dist, order="C")
    C = dg.matrix(M, N, seed, 2, dg.UNIFORM, order="C")
    return A, B, C


def sgemv_inputs(M, N, seed, dist):
    A = dg.matrix(M, N, seed, 0, dist, order="C")
    x = dg.fill(N, seed, 1, dist)
    y = dg.fill(M, seed, 2, dg.UNIFORM)
    return A, x, y


def main():
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/libhml_ref_cpu.so missing: run `make -C oracle` first")
    arrays = {}
    meta = {"sgemm": [], "sgemv": [], "configs": []}
    for name, M, N, K, al, be, seed, dist in SGEMM:
        A, B, C = sgemm_inputs(M, N, K, seed, dist)
        out = oracle.ref_sgemm_cpu(A, B, C, al, be)
        arrays[f"sgemm_{name}"] = out
        meta["sgemm"].append(dict(name=name, M=M, N=N, K=K, alpha=al, beta=be, seed=seed,
                                  dist=dist, csum=oracle.ref_csum(out)))
    for name, M, N, al, be, seed, dist in SGEMV:
        A, x, y = sgemv_inputs(M, N, seed, dist)
        out = oracle.ref_sgemv_cpu(A, x, y, al, be)
        arrays[f"sgemv_{name}"] = out
        meta["sgemv"].append(dict(name=name, M=M, N=N, alpha=al, beta=be, seed=seed, dist=dist,
                                  csum=oracle.ref_csum(out)))
    # Skinny SGEMM, column-major M=4096, N=16, K=4096, A and B uniform[-1,1],
    # seed 0 (A stream 0, B stream 1).  The reference is row-major only: its
    # loop runs on the exact row-major copies of the same logical matrices.
    A = dg.matrix(4096, 4096, 0, 0, dg.UNIFORM, order="F")
    B = dg.matrix(4096, 16, 0, 1, dg.UNIFORM, order="F")
    out = oracle.ref_sgemm_cpu(np.ascontiguousarray(A), np.ascontiguousarray(B), None, 1.0, 0.0)
    arrays["cfg_sgemm_4096x16x4096"] = out
    meta["configs"].append(dict(name="sgemm_4096x16x4096", kind="sgemm", M=4096, N=16, K=4096,
                                seed=0, dist=dg.UNIFORM, order="col", csum=oracle.ref_csum(out)))
    # SGEMV on column-major A 32768 x 4096, N(0,1), seed 1 (A stream 0,
    # x stream 1 with the length op(A) needs).
    A = dg.matrix(32768, 4096, 1, 0, dg.NORMAL, order="F")
    x_n = dg.fill(4096, 1, 1, dg.NORMAL)
    x_t = dg.fill(32768, 1, 1, dg.NORMAL)
    y_n = oracle.ref_sgemv_cpu(np.ascontiguousarray(A), x_n, None, 1.0, 0.0)  # y = A x
    # y = A^T x: the column-major storage is the row-major 4096 x 32768 A^T
    At = A.T
    assert At.flags["C_CONTIGUOUS"]
    y_t = oracle.ref_sgemv_cpu(At, x_t, None, 1.0, 0.0)
    arrays["cfg_sgemv_n_32768x4096"] = y_n
    arrays["cfg_sgemv_t_32768x4096"] = y_t
    meta["configs"].append(dict(name="sgemv_n_32768x4096", kind="sgemv_n", M=32768, N=4096,
                                seed=1, dist=dg.NORMAL, order="col", csum=oracle.ref_csum(y_n)))
    meta["configs"].append(dict(name="sgemv_t_32768x4096", kind="sgemv_t", M=32768, N=4096,
                                seed=1, dist=dg.NORMAL, order="col", csum=oracle.ref_csum(y_t)))
    np.savez_compressed(os.path.join(HERE, "reference_outputs.npz"), **arrays)
    with open(os.path.join(HERE, "reference_outputs.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print("wrote", len(arrays), "arrays")


if __name__ == "__main__":
    main()
