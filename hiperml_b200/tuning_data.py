"""Measured tuning data for the configuration predictor.

The predictor learns from what the autotuner (``hml_autotune_sgemm``)
measures: for each sampled problem shape, the median device time of every
configuration of the library's space (-1 where a configuration cannot run the
shape).  This module draws the shapes and runs the measurements; the result
is an ``.npz`` file with

    shapes   int64 [n, 5]   M, N, K, transA, transB (column-major storage)
    times_us float32 [n, C] measured time per configuration, -1 = not run
    configs  int32 [C, 6]   the configuration space (algo, tile_m, tile_n,
                            split_k, stages, variant), column order of times_us
    device   str

Usage (on the GPU):  python -m hiperml_b200.tuning_data OUT.npz --count 5000

It also writes the B200 tuned table shipped beside the library
(``data/tuned_b200.txt``, the counterpart of the reference's per-GPU .cfg
files): the autotuner's measured best configuration, among the FP32-accurate
families, for each of the library's reference workload shapes:

    python -m hiperml_b200.tuning_data --table hiperml_b200/data/tuned_b200.txt

The table also holds the measured best SGEMV variant of the reference
workloads' SGEMV shapes (``hml_autotune_sgemv``); ``--gemv-only`` re-measures
just those and keeps the SGEMM records.
"""
from __future__ import annotations

import argparse
import time

import numpy as np

# Shape distribution: M, N, K log-uniform in [1, 65536] x [1, 256] x
# [16, 16384], transposes Bernoulli(0.5).
M_RANGE, N_RANGE, K_RANGE = (1, 65536), (1, 256), (16, 16384)


def _log_uniform(rng, lo, hi, n):
    v = np.exp(rng.uniform(np.log(lo), np.log(hi + 1), n))
    return np.clip(np.floor(v), lo, hi).astype(np.int64)


def sample_shapes(count: int, seed: int) -> np.ndarray:
    """`count` shapes (M, N, K, transA, transB) from the distribution above,
    leaving out GEMV shapes (min(M, N) == 1, served by the GEMV kernels, where
    no configuration applies): draws are repeated until `count` remain."""
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < count:
        n = 2 * (count - len(out)) + 16
        M = _log_uniform(rng, *M_RANGE, n)
        N = _log_uniform(rng, *N_RANGE, n)
        K = _log_uniform(rng, *K_RANGE, n)
        ta = rng.integers(0, 2, n)
        tb = rng.integers(0, 2, n)
        for i in range(n):
            if min(M[i], N[i]) > 1:
                out.append((M[i], N[i], K[i], ta[i], tb[i]))
                if len(out) == count:
                    break
    return np.asarray(out, dtype=np.int64)


def config_table() -> np.ndarray:
    from . import api
    return np.asarray([c.as_tuple() for c in api.configs()], dtype=np.int32)


def measure(shapes: np.ndarray, reps: int = 3, deadline: float | None = None,
            progress=None, families: int = 0) -> np.ndarray:
    """Autotunes every shape (the algorithm families of the bitmask, 0 = all).
    Returns times_us [n, C]; configurations outside the families are -1, and
    rows of shapes not reached before `deadline` (time.time()) stay NaN."""
    from . import api
    cfgs = config_table()
    index = {tuple(c): i for i, c in enumerate(cfgs)}
    times = np.full((len(shapes), len(cfgs)), np.nan, dtype=np.float32)
    for r, (M, N, K, ta, tb) in enumerate(shapes):
        if deadline is not None and time.time() > deadline:
            break
        ents = api.autotune(api.COL_MAJOR, int(ta), int(tb), int(M), int(N), int(K),
                            families=families, reps=reps)
        row = np.full(len(cfgs), -1.0, dtype=np.float32)
        for c, t, st in ents:
            if st == 0 and t > 0:
                row[index[c.as_tuple()]] = t
        times[r] = row
        api.tune_clear()  # the dataset, not the tuned table, keeps the results
        if progress is not None:
            progress(r)
    return times


# The reference workloads' SGEMM shapes (M, N, K, transA, transB), column-major:
# the skinny 4096 x 16 x 4096 case, the M=65536, K=4096 precision sweep and the
# square 8192^3 case, and the skinny ones again in the reference's own
# row-major storage.
TABLE_SHAPES = ((4096, 16, 4096, 0, 0), (65536, 8, 4096, 0, 0), (65536, 32, 4096, 0, 0),
                (65536, 64, 4096, 0, 0), (65536, 128, 4096, 0, 0), (8192, 8192, 8192, 0, 0),
                # the same problems as the reference's row-major hmlSgemm stores
                # them (column-major op(A) = A^T, op(B) = B^T: A K-contiguous)
                (4096, 16, 4096, 1, 1), (65536, 8, 4096, 1, 1), (65536, 32, 4096, 1, 1),
                (65536, 64, 4096, 1, 1), (65536, 128, 4096, 1, 1))


# The reference workloads' SGEMV shapes (order, trans, M, N): the column-major
# 32768 x 4096 A applied as A x (column kernel) and as A^T x (row kernel).
GEMV_TABLE_SHAPES = ((0, 0, 32768, 4096), (0, 1, 32768, 4096))


def make_gemv_records(shapes=GEMV_TABLE_SHAPES, reps: int = 9) -> None:
    """Autotunes the SGEMV variants of each shape into the current table."""
    from . import api
    for (order, trans, M, N) in shapes:
        ents = api.autotune_sgemv(order, trans, M, N, reps=reps)
        t, v = min((t, v) for v, t, st in ents if st == 0 and t > 0)
        print(f"SGEMV order={order} trans={trans} M={M} N={N}: variant {v} {t:.1f} us "
              f"(all: {[(v, round(t, 1)) for v, t, _ in ents]})", flush=True)


def make_table(path, shapes=TABLE_SHAPES, reps: int = 5, gemv_only: bool = False) -> None:
    """Autotunes each shape over the FP32-accurate families (SIMT, BF16X6) and
    each SGEMV shape, and saves the resulting tuned table.  gemv_only: keep
    the SGEMM records of the table already at `path` and re-measure only the
    SGEMV ones."""
    from . import api
    api.tune_clear()
    if gemv_only:
        api.tune_load(str(path))
    else:
        fams = (1 << api.ALGO_SIMT) | (1 << api.ALGO_BF16X6)
        for (M, N, K, ta, tb) in shapes:
            ents = api.autotune(api.COL_MAJOR, ta, tb, M, N, K, families=fams, reps=reps)
            best = min(((t, c) for c, t, st in ents if st == 0 and t > 0), key=lambda e: e[0])
            print(f"M={M} N={N} K={K} ta={ta} tb={tb}: {best[1]} {best[0]:.1f} us", flush=True)
    make_gemv_records()
    api.tune_save(str(path))


def save(path, shapes, times, cfgs, device):
    np.savez_compressed(path, shapes=shapes, times_us=times.astype(np.float32), configs=cfgs,
                        device=np.asarray(device))


def load(path):
    d = np.load(path, allow_pickle=False)
    return {k: d[k] for k in d.files}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("out", nargs="?")
    ap.add_argument("--table", default=None,
                    help="write the tuned table of the reference workload shapes to this file")
    ap.add_argument("--gemv-only", action="store_true",
                    help="with --table: keep the file's SGEMM records, re-measure the SGEMV ones")
    ap.add_argument("--count", type=int, default=5000)
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--max-seconds", type=float, default=3000.0)
    ap.add_argument("--save-every", type=int, default=250)
    ap.add_argument("--families", type=int, default=0,
                    help="bitmask of algorithm families to measure (1 << hml_algo; 0 = all)")
    ap.add_argument("--merge", default=None,
                    help="existing dataset: its shapes are re-measured for --families only "
                         "and its other columns kept")
    args = ap.parse_args(argv)
    if args.table:
        make_table(args.table, gemv_only=args.gemv_only)
        return 0
    if not args.out:
        ap.error("OUT.npz is required")
    import torch
    base = load(args.merge) if args.merge else None
    shapes = base["shapes"] if base is not None else sample_shapes(args.count, args.seed)
    cfgs = config_table()
    fam_cols = (np.ones(len(cfgs), bool) if args.families == 0
                else ((1 << cfgs[:, 0]) & args.families) != 0)
    if base is not None and not np.array_equal(base["configs"], cfgs):
        # the space has grown or changed: keep the old columns of the
        # configurations still in it; every other column must be measured
        col = {tuple(c): i for i, c in enumerate(base["configs"])}
        old_t = base["times_us"]
        mapped = np.full((len(shapes), len(cfgs)), np.nan, dtype=np.float32)
        for j, c in enumerate(cfgs):
            i = col.get(tuple(c))
            if i is not None:
                mapped[:, j] = old_t[:, i]
            elif not fam_cols[j]:
                raise SystemExit(f"--merge: configuration {tuple(c)} is new; "
                                 "measure its family (--families)")
        base = dict(base, times_us=mapped, configs=cfgs)
    device = torch.cuda.get_device_name(0)
    deadline = time.time() + args.max_seconds
    t0 = time.time()
    # measure in blocks so partial results are saved (with --merge, a shape
    # not reached before the deadline is left out rather than kept stale)
    times = np.full((len(shapes), len(cfgs)), np.nan, dtype=np.float32)
    for b0 in range(0, len(shapes), args.save_every):
        blk = measure(shapes[b0:b0 + args.save_every], reps=args.reps, deadline=deadline,
                      families=args.families)
        if base is not None:
            done_blk = ~np.isnan(blk[:, 0])
            old = base["times_us"][b0:b0 + len(blk)]
            blk = np.where(fam_cols[None, :] | ~done_blk[:, None], blk, old)
        times[b0:b0 + len(blk)] = blk
        done = ~np.isnan(times[:, 0])
        save(args.out, shapes[done], times[done], cfgs, device)
        print(f"{done.sum()} shapes measured, {time.time() - t0:.0f} s", flush=True)
        if time.time() > deadline:
            break
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
