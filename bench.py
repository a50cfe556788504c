"""Benchmark of the skinny SGEMM/SGEMV path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload sweep|c1|gemv_n|gemv_t|square|batched]

Default workload ("sweep"): the skinny SGEMM precision sweep, C = A * B
column-major with M = 65536, K = 4096 and N in {8, 32, 64, 128}, A and B
uniform[-1, 1] from seed 0 (synthetic, generated on the device by the
library's SplitMix64 stream).  One step = the four GEMMs, each through
hml_sgemm_ex with the library's own configuration choice.  A is 1 GiB
(> the 126 MB L2), so no L2 flush is needed between steps.

The JSON line reports useful TFLOPS (2*M*N*K per GEMM), the roofline of the
dominant kernel (its algorithmic bytes, A and B read once and C written once,
over its event-timed duration against the measured HBM copy rate), an
end-to-end figure through the host-pointer C ABI (hml_host_sgemm, pinned host
buffers, copies inside the timed region), the reference's CPU loop as a CPU
baseline, the SM clocks sampled during the timed region and the number of
library kernel launches in it.  With the default workload it also carries
``workloads``: one short measured entry for each of the other configurations
(c1 with L2 flushed, both SGEMV forms, the square 8192^3 problem, the
log-uniform sweep, the sweep forced onto FP32 SIMT, the batched 1024-problem
plan against separate calls, and the configuration predictor's regret).

With torchrun (N > 1) every rank runs the same per-GPU workload on its own
data (weak scaling: the GEMMs are independent row blocks of a larger
problem, so there is no data-path collective); the timing is the max over
ranks.  --impl reference times the reference's own CPU implementation
(hmlSgemmCpu from oracle/_ref) on a bounded sample on rank 0.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "skinny SGEMM TFLOPS & % roofline: split-BF16 TC vs FP32 SIMT at FP32 accuracy"
UNIT = "TFLOPS"

SWEEP_M, SWEEP_K, SWEEP_N = 65536, 4096, (8, 32, 64, 128)
SIMT_PEAK_NOMINAL = 148 * 128 * 2 * 1.965e-3  # TFLOP/s: 148 SMs x 128 FMA lanes x 2 x 1.965 GHz
ALGO_NAMES = {1: "simt", 2: "bf16x3", 3: "bf16x6", 4: "tf32x3", 5: "fp16x3"}
ALGO_CODES = {"auto": None, "simt": 1, "bf16x3": 2, "bf16x6": 3, "tf32x3": 4, "fp16x3": 5}
# BF16-product equivalents of one useful multiply-add per split form (a TF32
# product runs at half the BF16 rate)
PRODUCTS = {2: 3, 3: 6, 4: 6, 5: 3}
# the least tensor work that gives FP32-level accuracy: a 3-product split
# (hi*hi + hi*lo + lo*hi); the problem's tensor roofline uses it
MIN_PRODUCTS = 3


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sweep",
                    choices=["sweep", "c1", "gemv_n", "gemv_t", "square", "batched"])
    ap.add_argument("--algo", default="auto", choices=list(ALGO_CODES),
                    help="force one algorithm family (default: the library's choice)")
    ap.add_argument("--dist", default="uniform", choices=["uniform", "loguniform"],
                    help="sweep/c1/square inputs: uniform[-1,1] or log-uniform 1e-3..1e3")
    ap.add_argument("--rows", type=int, default=None,
                    help="sweep workload: M other than 65536 (small cases for profiler captures)")
    ap.add_argument("--only-n", type=int, default=None,
                    help="sweep workload: run only this N (profiler captures)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-workloads", action="store_true",
                    help="default workload: leave out the per-configuration entries")
    return ap.parse_args()


def load_datagen():
    """hiperml_b200/datagen.py as a stand-alone module (pure numpy): the
    reference arm draws its inputs with it without importing the package,
    which would load the library."""
    path = os.path.join(ROOT, "hiperml_b200", "datagen.py")
    spec = importlib.util.spec_from_file_location("hml_datagen_standalone", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


# ------------------------------------------------------------------ peaks
def peaks():
    p = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0,
         "source": "fallback"}
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            m = json.load(f)
        for k in ("hbm_gbs", "bf16_tflops", "bf16_tflops_sustained"):
            if k in m:
                p[k] = float(m[k])
        p["source"] = "measured"
    return p


def traffic_table():
    """Per-launch DRAM bytes of the dominant kernels from committed ncu
    summaries (profiles/traffic.json), keyed by workload name."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while running."""

    REASONS = {
        0x0000000000000001: "gpu_idle", 0x0000000000000002: "applications_clocks_setting",
        0x0000000000000004: "sw_power_cap", 0x0000000000000008: "hw_slowdown",
        0x0000000000000010: "sync_boost", 0x0000000000000020: "sw_thermal_slowdown",
        0x0000000000000040: "hw_thermal_slowdown", 0x0000000000000080: "hw_power_brake_slowdown",
        0x0000000000000100: "display_clock_setting",
    }

    def __init__(self, index=0, period=0.01):
        self.samples, self.reasons = [], set()
        self.max_mhz = None
        self.period = period
        self._stop = threading.Event()
        self.ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:  # noqa: BLE001  (NVML unavailable: report no clocks)
            self.ok = False

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                mask = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for bit, name in self.REASONS.items():
                    if mask & bit and name != "gpu_idle":
                        self.reasons.add(name)
            except Exception:  # noqa: BLE001
                pass
            time.sleep(self.period)

    def __enter__(self):
        if self.ok:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *exc):
        if self.ok:
            self._stop.set()
            self._t.join()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                    "samples": len(self.samples)}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


# ------------------------------------------------------------- workloads
def workload_problems(name, rows=None, only_n=None):
    """List of (kind, M, N, K) problems making one step."""
    if name == "sweep":
        return [("sgemm", rows or SWEEP_M, n, SWEEP_K) for n in SWEEP_N
                if only_n is None or n == only_n]
    if name == "c1":
        return [("sgemm", 4096, 16, 4096)]
    if name == "gemv_n":
        return [("gemv_n", 32768, 1, 4096)]
    if name == "gemv_t":
        return [("gemv_t", 32768, 1, 4096)]
    if name == "square":
        return [("sgemm", 8192, 8192, 8192)]
    if name == "batched":
        return [("sgemm", M, N, K) for (_ta, _tb, M, N, K) in batch_shapes()]
    raise ValueError(name)


BATCH_COUNT, BATCH_SEED = 1024, 3


def batch_shapes(count=BATCH_COUNT, seed=BATCH_SEED):
    """The batched workload: `count` problems (transA, transB, M, N, K) with
    M log-uniform in [256, 16384], N uniform in 1..128, K log-uniform in
    [64, 4096] and Bernoulli(0.5) transposes, drawn from numpy's PCG64 with
    the given seed."""
    import numpy as np
    rng = np.random.default_rng(seed)
    M = np.exp(rng.uniform(np.log(256), np.log(16384), count)).astype(np.int64)
    N = rng.integers(1, 129, count)
    K = np.exp(rng.uniform(np.log(64), np.log(4096), count)).astype(np.int64)
    ta = rng.integers(0, 2, count)
    tb = rng.integers(0, 2, count)
    return [(int(ta[i]), int(tb[i]), int(M[i]), int(N[i]), int(K[i])) for i in range(count)]


def flops_of(kind, M, N, K):
    return 2.0 * M * N * K if kind == "sgemm" else 2.0 * M * K


def bytes_of(kind, M, N, K):
    """Algorithmic bytes: A and B read once, C written once (beta = 0)."""
    if kind == "sgemm":
        return 4.0 * (M * K + K * N + M * N)
    P = M if kind == "gemv_n" else K
    Q = K if kind == "gemv_n" else M
    return 4.0 * (M * K + Q + P)


DIST_DESC = {"uniform": "uniform[-1,1]", "loguniform": "log-uniform magnitude 1e-3..1e3, random sign"}


def config_desc(name, dist="uniform"):
    """The workload, identical in both arms' JSON lines."""
    if name == "sweep":
        return {"workload": f"skinny SGEMM C=A*B col-major, M={SWEEP_M}, K={SWEEP_K}, "
                            f"N in {list(SWEEP_N)} (one step = the 4 GEMMs)",
                "M": SWEEP_M, "K": SWEEP_K, "N": list(SWEEP_N), "alpha": 1.0, "beta": 0.0,
                "layout": "column-major NN", "inputs": f"{DIST_DESC[dist]}, seed 0",
                "l2": "A is 1 GiB per GEMM (> 126 MB L2): inputs larger than L2, no flush"}
    if name == "c1":
        return {"workload": "skinny SGEMM col-major M=4096, N=16, K=4096", "M": 4096, "N": 16,
                "K": 4096, "inputs": f"{DIST_DESC[dist]}, seed 0",
                "l2": "L2 flushed (256 MiB write) before every step"}
    if name in ("gemv_n", "gemv_t"):
        return {"workload": f"SGEMV y={'A' if name == 'gemv_n' else 'A^T'}*x, A 32768x4096 "
                            "col-major", "inputs": "N(0,1), seed 1",
                "l2": "A is 512 MiB (> L2): no flush"}
    if name == "batched":
        return {"workload": f"batched: {BATCH_COUNT} independent FP32 GEMMs C=op(A)op(B), "
                            "col-major, one persistent graph-captured launch",
                "M": "log-uniform [256, 16384]", "N": "uniform {1..128}",
                "K": "log-uniform [64, 4096]", "trans": "Bernoulli(0.5) each",
                "alpha": 1.0, "beta": 0.0, "count": BATCH_COUNT,
                "shapes_seed": BATCH_SEED, "inputs": "N(0,1), seed 3",
                "storage": "leading dimensions rounded up to 4 floats, 256-byte aligned bases",
                "l2": "about 15 GB of operands per step (> 126 MB L2): no flush"}
    return {"workload": "square SGEMM 8192^3 col-major", "inputs": f"{DIST_DESC[dist]}, seed 0",
            "l2": "compute bound; inputs 256 MiB each"}


# -------------------------------------------------------------- reference
def cpu_reference_sample(problems, seconds=10.0, threads=None):
    """Times the reference's own hmlSgemmCpu / hmlSgemvCpu (oracle/_ref, or
    the C restatement when the reference build is absent) on row slices of
    each problem, on all host cores (one independent row block per thread).
    Returns (TFLOPS, cores, kind, sample description, seconds timed, passes)."""
    import ctypes
    from concurrent.futures import ThreadPoolExecutor

    import numpy as np

    import oracle
    dg = load_datagen()

    cores = threads or os.cpu_count() or 1
    kind = "reference" if oracle.ref_available() else "port"
    if kind == "reference":
        R = oracle.ref()
        f_gemm, f_gemv = R.sgemm_cpu, R.sgemv_cpu
    else:
        L = oracle.lib()
        f_gemm, f_gemv = L.oracle_sgemm_rm_f32, L.oracle_sgemv_rm_f32
    fp = ctypes.POINTER(ctypes.c_float)
    # row slices of each problem: rows chosen so that one pass takes ~seconds
    rows_per_thread = 8
    jobs = []
    for (k, M, N, K) in problems:
        # operands: the logical matrices' row-major copies (exact transposes)
        A = dg.fill(cores * rows_per_thread * K, 0, 0).reshape(cores * rows_per_thread, K)
        if k == "sgemm":
            B = dg.fill(K * N, 0, 1).reshape(K, N)
            jobs.append((k, A, B, N, K))
        else:
            x = dg.fill(K, 1, 1)
            jobs.append((k, A, x, 1, K))

    def run_block(args):
        k, A, B, N, K, r0, r1 = args
        a = A[r0:r1]
        if k == "sgemm":
            C = np.zeros((r1 - r0, N), np.float32)
            f_gemm(C.ctypes.data_as(fp), a.ctypes.data_as(fp), B.ctypes.data_as(fp), r1 - r0, N,
                   K, 1.0, 0.0)
        else:
            y = np.zeros(r1 - r0, np.float32)
            f_gemv(y.ctypes.data_as(fp), a.ctypes.data_as(fp), B.ctypes.data_as(fp), r1 - r0, K,
                   1.0, 0.0)

    total_flops, elapsed, passes = 0.0, 0.0, 0
    with oracle._QuietStderr(), ThreadPoolExecutor(cores) as ex:
        t_end = time.perf_counter() + seconds
        while True:
            for (k, A, B, N, K) in jobs:
                work = [(k, A, B, N, K, t * rows_per_thread, (t + 1) * rows_per_thread)
                        for t in range(cores)]
                t0 = time.perf_counter()
                list(ex.map(run_block, work))
                elapsed += time.perf_counter() - t0
                total_flops += flops_of(k, cores * rows_per_thread, N, K)
            passes += 1
            if time.perf_counter() > t_end:
                break
    desc = (f"{passes} pass(es) over {cores * rows_per_thread} rows of each problem "
            f"({', '.join(f'{k} M={M} N={N} K={K}' for (k, M, N, K) in problems)}), "
            f"one row block per thread, {elapsed:.1f} s")
    return total_flops / elapsed / 1e12, cores, kind, desc, elapsed, passes


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    problems = workload_problems(args.workload)
    if args.workload == "batched":
        # the reference has no batched form: its callers loop over hmlSgemm,
        # here over its CPU loop, on the first 64 problems of the batch
        problems = problems[:64]
    per_step = max(1.0, 120.0 / max(1, args.steps + args.warmup))
    per_step = min(per_step, 10.0)
    vals, secs = [], []
    cores = kind = desc = None
    for i in range(args.warmup + args.steps):
        v, cores, kind, desc, el, _ = cpu_reference_sample(problems, seconds=per_step)
        if i >= args.warmup:
            vals.append(v)
            secs.append(el)
    value = statistics.median(vals)
    step_flops = sum(flops_of(*p) for p in problems)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        # what one timed step actually ran: a bounded row sample of the
        # workload (the full workload at this rate is reported beside it)
        "ms_per_step": statistics.mean(secs) * 1e3,
        "ms_per_step_kind": "timed CPU sample per step (bounded row slices of the workload)",
        "ms_per_full_workload_at_sample_rate": step_flops / (value * 1e12) * 1e3,
        "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_desc(args.workload),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# -------------------------------------------------------------------- ours
class Ctx:
    """Device, stream and process-group state of one rank."""

    def __init__(self):
        import torch
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist_on = self.world > 1
        if self.dist_on:
            import datetime

            import torch.distributed as dist
            torch.cuda.set_device(self.local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        self.dev = torch.device("cuda", self.local)
        torch.cuda.set_device(self.dev)
        self.stream = torch.cuda.current_stream()

    def barrier(self):
        if self.dist_on:
            import torch.distributed as dist
            dist.barrier()

    def close(self):
        if self.dist_on:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


def measure_gemms(ctx, problems, algo, dist, steps, warmup, flush_l2, clocks=None,
                  err_check=True):
    """Runs `problems` (one step) `warmup` + `steps` times through
    hml_sgemm_ex / hml_sgemv_ex and times them with CUDA events on the
    launching stream.  Returns a dict with the step time (max over ranks),
    per-problem times and configurations, launch counts and FP64 errors."""
    import torch

    import hiperml_b200 as hml
    from hiperml_b200 import datagen as dg
    from hiperml_b200.dist import max_over_ranks

    dev, stream, rank = ctx.dev, ctx.stream, ctx.rank
    dist_code = {"uniform": dg.UNIFORM, "loguniform": dg.LOGUNIFORM}[dist]
    bufs = []
    Ashared = None
    for (k, M, N, K) in problems:
        if k == "sgemm":
            if Ashared is None or Ashared.numel() != M * K:
                Ashared = torch.empty(M * K, dtype=torch.float32, device=dev)
                hml.fill_random(Ashared, 0 + rank * 1000, 0, dist_code)
            B = torch.empty(K * N, dtype=torch.float32, device=dev)
            hml.fill_random(B, 0 + rank * 1000, 1, dist_code)
            C = torch.zeros(M * N, dtype=torch.float32, device=dev)
            cfg = hml.select(0, 0, 0, M, N, K) if algo is None else \
                hml.select_algo(0, 0, 0, M, N, K, algo)
            bufs.append((k, M, N, K, Ashared, B, C, cfg))
        else:
            A = torch.empty(M * K, dtype=torch.float32, device=dev)
            hml.fill_random(A, 1 + rank * 1000, 0, dg.NORMAL)
            Q = K if k == "gemv_n" else M
            P = M if k == "gemv_n" else K
            x = torch.empty(Q, dtype=torch.float32, device=dev)
            hml.fill_random(x, 1 + rank * 1000, 1, dg.NORMAL)
            y = torch.zeros(P, dtype=torch.float32, device=dev)
            bufs.append((k, M, N, K, A, x, y, None))
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev) if flush_l2 else None

    def launch(item):
        k, M, N, K, A, B, C, cfg = item
        if k == "sgemm":
            hml.sgemm_ex(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, C, M, stream=stream,
                         config=cfg if algo is not None else None)
        elif k == "gemv_n":
            hml.sgemv_ex(0, 0, M, K, 1.0, A, M, B, 0.0, C, stream=stream)
        else:
            hml.sgemv_ex(0, 1, M, K, 1.0, A, M, B, 0.0, C, stream=stream)

    n_items = len(bufs)
    ev = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(n_items)] for _ in range(steps)]

    def step(i=None):
        if flush is not None:
            flush.fill_(float(i or 0))  # 256 MiB write: nothing of the operands stays in L2
        for j, item in enumerate(bufs):
            if i is not None:
                ev[i][j][0].record(stream)
            launch(item)
            if i is not None:
                ev[i][j][1].record(stream)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    if hml.device_error() != 0:
        raise RuntimeError("device wait expired during warm-up")
    ctx.barrier()
    torch.cuda.synchronize()
    launches0 = hml.lib.hml_launch_count()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    sampler = clocks if clocks is not None else ClockSampler(ctx.local, period=1.0)
    with sampler:
        t0.record(stream)
        for i in range(steps):
            step(i)
        t1.record(stream)
        torch.cuda.synchronize()
    launches = hml.lib.hml_launch_count() - launches0
    ctx.barrier()
    elapsed_ms = t0.elapsed_time(t1)
    per_kernel_ms = [statistics.mean(ev[i][j][0].elapsed_time(ev[i][j][1]) for i in range(steps))
                     for j in range(n_items)]
    if flush is not None:
        # the flush is outside the measured GEMM events; time only the GEMMs
        elapsed_ms = sum(sum(ev[i][j][0].elapsed_time(ev[i][j][1]) for j in range(n_items))
                         for i in range(steps))
    elapsed_ms = max_over_ranks(elapsed_ms, dev)
    if hml.device_error() != 0:
        raise RuntimeError("device wait expired in the timed region")
    per_shape = []
    for j, (k, M, N, K, A, B, C, cfg) in enumerate(bufs):
        entry = {"kind": k, "M": M, "N": N, "K": K, "ms": per_kernel_ms[j],
                 "tflops": flops_of(k, M, N, K) / (per_kernel_ms[j] * 1e-3) / 1e12,
                 "gbs": bytes_of(k, M, N, K) / (per_kernel_ms[j] * 1e-3) / 1e9,
                 "config": repr(cfg) if cfg is not None else "gemv"}
        if k == "sgemm" and rank == 0 and err_check:
            err = hml.error_fp64(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, None, C, M)
            entry["max_rel_err_fp64"] = err[0]
            entry["rms_rel_err_fp64"] = err[1]
            entry["compwise_err_fp64"] = err[2]
        per_shape.append(entry)
    step_flops = sum(flops_of(k, M, N, K) for (k, M, N, K, *_r) in bufs)
    return {"bufs": bufs, "elapsed_ms": elapsed_ms, "per_kernel_ms": per_kernel_ms,
            "launches": launches, "per_shape": per_shape, "step_flops": step_flops,
            "value": step_flops * steps * ctx.world / (elapsed_ms * 1e-3) / 1e12,
            "ms_per_step": elapsed_ms / steps}


def roofline_of(kind, M, N, K, cfg, ms, key, pk):
    """Roofline of one kernel launch, set by the problem, not by the form that
    runs it.  Its memory floor is the algorithmic bytes (A and B read once, C
    written once) at the measured HBM copy rate; its compute floor is the
    useful 2MNK at the sustained BF16 tensor peak divided by MIN_PRODUCTS
    (the least tensor work that keeps FP32-level accuracy).  The larger floor
    bounds it: `frac` = that floor over the measured launch time.  Every
    skinny and GEMV shape is HBM-bound; the square 8192^3 problem is
    tensor-bound.  tensor_pipe_frac reports the tensor-pipe work the running
    split form does (its BF16 products per useful multiply-add) against the
    sustained BF16 peak."""
    alg_bytes = bytes_of(kind, M, N, K)
    alg_flops = flops_of(kind, M, N, K)
    s = ms * 1e-3
    ai = alg_flops / alg_bytes
    tensor_peak = pk["bf16_tflops_sustained"]
    useful_cap = tensor_peak / MIN_PRODUCTS  # TFLOP/s of useful work at the tensor peak
    hbm_time = alg_bytes / (pk["hbm_gbs"] * 1e9)
    tensor_time = alg_flops / (useful_cap * 1e12)
    roof = {"bound": "hbm", "achieved": alg_bytes / s / 1e9, "peak": pk["hbm_gbs"],
            "unit": "GB/s", "frac": alg_bytes / s / 1e9 / pk["hbm_gbs"],
            "traffic": traffic_table().get(key), "kernel": key,
            "alg_bytes_per_launch": alg_bytes, "alg_flops_per_launch": alg_flops,
            "ms_per_launch": ms, "peak_source": pk["source"], "arith_intensity": ai}
    if kind == "sgemm" and tensor_time > hbm_time:
        roof.update({"bound": "tensor", "achieved": alg_flops / s / 1e12, "peak": useful_cap,
                     "unit": f"TFLOP/s (useful 2MNK; peak = sustained BF16 / {MIN_PRODUCTS})",
                     "frac": alg_flops / s / 1e12 / useful_cap})
    if cfg is not None and cfg.algo in PRODUCTS:
        products = PRODUCTS[cfg.algo]
        roof["tensor_pipe_frac"] = alg_flops * products / s / 1e12 / tensor_peak
        roof["tensor_products_per_mac"] = products
    if cfg is not None and cfg.algo == 1:
        roof["simt_fp32_tflops"] = alg_flops / s / 1e12
        roof["simt_fp32_peak_nominal"] = SIMT_PEAK_NOMINAL
        roof["simt_fp32_frac_nominal"] = alg_flops / s / 1e12 / SIMT_PEAK_NOMINAL
    return roof


def kernel_key(workload, kind, M, N, K, cfg):
    return f"{workload}:{kind}:{M}x{N}x{K}:{ALGO_NAMES.get(cfg.algo, 'gemv') if cfg else 'gemv'}"


def workload_entry(ctx, name, algo=None, dist="uniform", steps=10, warmup=3):
    """One short measured entry of a non-headline configuration."""
    problems = workload_problems(name)
    r = measure_gemms(ctx, problems, algo, dist, steps, warmup, flush_l2=(name == "c1"))
    pk = peaks()
    dom = max(range(len(r["bufs"])), key=lambda j: r["per_kernel_ms"][j])
    k, M, N, K, *_x, cfg = r["bufs"][dom]
    roof = roofline_of(k, M, N, K, cfg, r["per_kernel_ms"][dom],
                       kernel_key(name, k, M, N, K, cfg), pk)
    errs = [e for e in r["per_shape"] if "max_rel_err_fp64" in e]
    step_bytes = sum(bytes_of(k, M, N, K) for (k, M, N, K, *_r) in r["bufs"])
    out = {"workload": name, "config": config_desc(name, dist),
           "selection": "automatic" if algo is None else f"forced {ALGO_NAMES[algo]}",
           "steps": steps, "warmup": warmup, "ms_per_step": r["ms_per_step"],
           "tflops": r["value"] / ctx.world,
           "gbs": step_bytes / (r["ms_per_step"] * 1e-3) / 1e9,
           "roofline": {kk: roof[kk] for kk in ("bound", "achieved", "peak", "unit", "frac",
                                                "kernel", "tensor_pipe_frac")
                        if kk in roof},
           "per_shape": r["per_shape"]}
    if errs:
        out["max_rel_err_fp64"] = max(e["max_rel_err_fp64"] for e in errs)
        out["compwise_err_fp64"] = max(e["compwise_err_fp64"] for e in errs)
    return out


def predictor_entry(ctx, live_shapes=4, live_reps=3):
    """Regret of the shipped configuration predictor: on the 1000 held-out
    shapes of the measured dataset (exhaustive autotune times), against the
    best fixed configuration and the built-in heuristic; and live, on a few
    unseen shapes autotuned now over the FP32-accurate families."""
    import numpy as np

    import hiperml_b200 as hml
    from hiperml_b200 import predictor as pr
    from hiperml_b200 import tuning_data as td
    if not (os.path.exists(pr.DATASET) and os.path.exists(pr.MODEL)):
        return {"workload": "predictor", "unavailable": "no shipped dataset or network"}
    d = td.load(pr.DATASET)
    shapes, times, cfgs = d["shapes"], d["times_us"], d["configs"]
    n_tr = min(4000, int(0.8 * len(shapes)))
    te = slice(n_tr, None)
    hml.tune_clear()
    pr.load(pr.MODEL)
    t0 = time.perf_counter()
    pred = pr.predict_batch(shapes[te])
    r_pred = pr.summarize(pr.regret(times[te], pred, cfgs))
    fixed = pr.best_fixed_config(times[:n_tr], cfgs)
    r_fixed = pr.summarize(pr.regret(times[te], np.full(len(pred), fixed), cfgs))
    live = []
    cfg_t = [tuple(int(x) for x in c) for c in cfgs]
    for (M, N, K, ta, tb) in td.sample_shapes(live_shapes, 4242):
        j = pr.predict_batch(np.array([[M, N, K, ta, tb]]))[0]
        ents = hml.autotune(0, int(ta), int(tb), int(M), int(N), int(K),
                            families=(1 << hml.ALGO_SIMT) | (1 << hml.ALGO_BF16X6), reps=live_reps)
        t = {c.as_tuple(): us for c, us, st in ents if st == 0 and us > 0}
        if cfg_t[j] in t:
            live.append({"shape": [int(M), int(N), int(K), int(ta), int(tb)],
                         "regret": t[cfg_t[j]] / min(t.values()) - 1.0})
    hml.tune_clear()
    pr.clear()
    heur = pr.heuristic_choices(shapes[te], cfgs)
    r_heur = pr.summarize(pr.regret(times[te], heur, cfgs))
    # the library's defaults back (the shipped tuned table and network) for
    # the entries measured after this one
    hml.tune_load(os.path.join(os.path.dirname(hml.__file__), "data", "tuned_b200.txt"))
    pr.load(pr.MODEL)
    return {"workload": "predictor",
            "config": {"dataset": "5000 shapes (M,N,K log-uniform [1,65536]x[1,256]x[16,16384], "
                                  "random transposes), each autotuned over the configuration "
                                  "space on a B200; network trained on the first 4000",
                       "held_out": int(len(pred))},
            "held_out_regret": r_pred, "fixed_default_regret": r_fixed,
            "heuristic_regret": r_heur,
            "live_regret": live,
            "live_regret_mean": (float(np.mean([x["regret"] for x in live])) if live else None),
            "seconds": time.perf_counter() - t0}


def reference_gpu_entry(ctx, reps=3):
    """The reference's own GPU kernels (its kernel repositories and selectors
    compiled from its sources into oracle/_ref, K40 rules loaded) against
    this library on the same row-major problems, kernel time only (CUDA
    events, operands on the device; L2 flushed before each launch of the
    4096 x 16 x 4096 problem, whose A fits in it).  The reference's
    host-pointer API refuses problems with M*K or N*K >= 2^27 (its texture
    limit, src/hml_sgemm.cu:146-149, src/hml_sgemv.cu:150); its kernels run
    them here through the texture stand-in, and such shapes are marked."""
    import tempfile

    import numpy as np
    import torch

    import hiperml_b200 as hml
    import oracle
    from hiperml_b200 import datagen as dg
    if not oracle.ref_gpu_available():
        return {"workload": "reference_gpu",
                "unavailable": "oracle/_ref GPU libraries not built (make -C oracle refgpu)"}
    rules = dict(np.load(os.path.join(ROOT, "tests", "golden", "cfg_rules.npz")))
    with tempfile.TemporaryDirectory() as d:
        for kind in ("sgemm", "sgemv"):
            rows = rules[f"hml_{kind}_k40"]
            path = os.path.join(d, f"{kind}.cfg")
            with open(path, "w") as f:
                f.write(f"#{kind.upper()} smart kernel config file v1.0\n")
                for r in rows:
                    f.write((f"{r[0]} {r[1]} : {r[2]} {r[3]}\n" if kind == "sgemm"
                             else f"{r[0]} : {r[1]} {r[2]} {r[3]}\n"))
            oracle.ref_gpu_load_rules(kind, path)
    dev, stream = ctx.dev, ctx.stream
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    out = []

    def ours_ms(fn, n, flush_l2):
        evs = []
        for _ in range(n + 1):
            if flush_l2:
                flush.fill_(1.0)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            evs.append((a, b))
        torch.cuda.synchronize()
        return statistics.median(a.elapsed_time(b) for a, b in evs[1:])

    def ref_ms(fn, n, flush_l2):
        times = []
        for _ in range(n + 1):
            if flush_l2:
                flush.fill_(1.0)
                torch.cuda.synchronize()
            times.append(fn())
        return statistics.median(times[1:])

    for (M, N, K) in [(4096, 16, 4096)] + [(SWEEP_M, n, SWEEP_K) for n in SWEEP_N]:
        A = torch.empty(M * K, device=dev)
        B = torch.empty(K * N, device=dev)
        hml.fill_random(A, 0, 0, dg.UNIFORM)
        hml.fill_random(B, 0, 1, dg.UNIFORM)
        Cr = torch.zeros(M * N, device=dev)
        Co = torch.zeros(M * N, device=dev)
        fl = M * K * 4 < 126e6
        t_ref = ref_ms(lambda: oracle.ref_gpu_sgemm(Cr.data_ptr(), A.data_ptr(), B.data_ptr(), M, N,
                                                    K, 1.0, 0.0, 1), reps, fl)
        t_ours = ours_ms(lambda: hml.sgemm_ex(hml.ROW_MAJOR, 0, 0, M, N, K, 1.0, A, K, B, N, 0.0,
                                              Co, N, stream=stream), reps, fl)
        torch.cuda.synchronize()
        diff = float((Cr - Co).abs().max() / Co.abs().max())
        err_ref = hml.error_fp64(hml.ROW_MAJOR, 0, 0, M, N, K, 1.0, A, K, B, N, 0.0, None, Cr, N)
        err_ours = hml.error_fp64(hml.ROW_MAJOR, 0, 0, M, N, K, 1.0, A, K, B, N, 0.0, None, Co, N)
        is_const, grid, block = oracle.ref_gpu_select("sgemm", M, N, K)
        out.append({"kind": "sgemm", "M": M, "N": N, "K": K, "layout": "row-major NN",
                    "reference_ms": t_ref, "ours_ms": t_ours, "speedup": t_ref / t_ours,
                    "reference_tflops": flops_of("sgemm", M, N, K) / (t_ref * 1e-3) / 1e12,
                    "reference_kernel": {"const_k": is_const, "grid": grid, "block": block},
                    "beyond_reference_texture_limit": M * K >= 1 << 27,
                    "max_rel_diff": diff, "reference_max_rel_err_fp64": err_ref[0],
                    "ours_max_rel_err_fp64": err_ours[0], "l2_flushed": fl})
        del A, B, Cr, Co
    for (M, N, form) in ((32768, 4096, "y = A x"), (4096, 32768, "y = A^T x")):
        # row-major M x N: the two forms of the 32768 x 4096 column-major GEMV
        A = torch.empty(M * N, device=dev)
        x = torch.empty(N, device=dev)
        hml.fill_random(A, 1, 0, dg.NORMAL)
        hml.fill_random(x, 1, 1, dg.NORMAL)
        yr = torch.zeros(M, device=dev)
        yo = torch.zeros(M, device=dev)
        t_ref = ref_ms(lambda: oracle.ref_gpu_sgemv(yr.data_ptr(), A.data_ptr(), x.data_ptr(), M, N,
                                                    1.0, 0.0, 1), reps, False)
        t_ours = ours_ms(lambda: hml.sgemv_ex(hml.ROW_MAJOR, hml.OP_N, M, N, 1.0, A, N, x, 0.0, yo,
                                              stream=stream), reps, False)
        torch.cuda.synchronize()
        diff = float((yr - yo).abs().max() / yo.abs().max())
        # y = A x as an M x 1 x N GEMM, row-major
        err_ref = hml.error_fp64(hml.ROW_MAJOR, 0, 0, M, 1, N, 1.0, A, N, x, 1, 0.0, None, yr, 1)
        err_ours = hml.error_fp64(hml.ROW_MAJOR, 0, 0, M, 1, N, 1.0, A, N, x, 1, 0.0, None, yo, 1)
        out.append({"kind": "sgemv", "M": M, "N": N, "form": form, "layout": "row-major",
                    "reference_max_rel_err_fp64": err_ref[0], "ours_max_rel_err_fp64": err_ours[0],
                    "reference_kernel": "basic (N > 1024): its unsynchronised warp reduction "
                                        "gives wrong sums on B200",
                    "reference_ms": t_ref, "ours_ms": t_ours, "speedup": t_ref / t_ours,
                    "reference_gbs": bytes_of("gemv_n", M, 1, N) / (t_ref * 1e-3) / 1e9,
                    "beyond_reference_texture_limit": M * N >= 1 << 27, "max_rel_diff": diff})
        del A, x, yr, yo
    return {"workload": "reference_gpu", "rules": "shipped K40 .cfg (config/hml_sgemm_k40.cfg, "
                                                   "config/hml_sgemv_k40.cfg)",
            "shapes": out}


def kmeans_entry(ctx, reps=5):
    """The k-means assignment step (hml_kmeans_assign_ex: the dot products as
    one skinny GEMM, an exact argmin) in each of its forms -- tiled (the
    argmin fused into a register-tiled SIMT GEMM), SGEMM (the products
    through HBM, then a pick kernel) and tensor-core (TF32X3 products in
    TMEM, the argmin read from the accumulator) -- against the reference's own assignment
    kernel hmlKmeansAssignCtrdSmem (oracle/_ref; up to 64 dimensions, as in
    the reference), 1M points, N(0,1), kernel time with CUDA events, and
    whether the index arrays are equal."""
    import torch

    import hiperml_b200 as hml
    import oracle
    from hiperml_b200 import datagen as dg

    def timed(fn):
        evs = []
        for i in range(reps + 2):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(ctx.stream)
            fn()
            b.record(ctx.stream)
            evs.append((a, b))
        torch.cuda.synchronize()
        return statistics.median(a.elapsed_time(b) for a, b in evs[2:])

    out = []
    for (n, d, k) in ((1 << 20, 32, 64), (1 << 20, 32, 256), (1 << 20, 64, 128),
                      (1 << 20, 128, 64), (1 << 20, 256, 64)):
        P = torch.empty(n * d, device=ctx.dev)
        C = torch.empty(k * d, device=ctx.dev)
        hml.fill_random(P, 11, 0, dg.NORMAL)
        hml.fill_random(C, 11, 1, dg.NORMAL)
        P, C = P.view(n, d), C.view(k, d)
        got = torch.empty(n, dtype=torch.int32, device=ctx.dev)
        entry = {"points": n, "dims": d, "clusters": k}
        results = {}
        forms = [("tiled", hml.KMEANS_TILED), ("gemm", hml.KMEANS_GEMM)]
        if d % 4 == 0 and d <= 64 and k <= 256:
            forms.append(("tensor", hml.KMEANS_TENSOR))
        for name, method in forms + [("auto", hml.KMEANS_AUTO)]:
            t = timed(lambda: hml.kmeans_assign(P, C, out=got, stream=ctx.stream, method=method))
            entry[f"{name}_ms"] = t
            results[name] = got.clone()
        t_ours = entry["auto_ms"]
        entry.update({"ours_points_per_s": n / (t_ours * 1e-3),
                      "gemm_tflops": 2.0 * n * d * k / (t_ours * 1e-3) / 1e12,
                      "forms_equal": all(bool(torch.equal(results[f], results["tiled"]))
                                         for f, _ in forms)})
        _, exact = hml.kmeans_assign(P, C, count_exact=True)
        entry["points_resolved_exactly"] = exact
        if oracle.ref_gpu_kmeans_available() and d in (4, 8, 16, 32, 64):
            ref = torch.zeros(n, dtype=torch.int32, device=ctx.dev)
            oracle.ref_gpu_kmeans_assign(ref.data_ptr(), P.data_ptr(), n, C.data_ptr(), k, d, 1)
            t_ref = oracle.ref_gpu_kmeans_assign(ref.data_ptr(), P.data_ptr(), n, C.data_ptr(), k,
                                                 d, reps)
            torch.cuda.synchronize()
            entry.update({"reference_ms": t_ref, "speedup": t_ref / t_ours,
                          "indices_equal": bool(torch.equal(results["auto"], ref))})
        out.append(entry)
        del P, C, got, results
    return {"workload": "kmeans_assign",
            "config": {"data": "points and centroids N(0,1), seed 11", "layout": "row-major",
                       "reference": "hmlKmeansAssignCtrdSmem built from the reference's header "
                                    "(dimensions up to 64, its limit)"},
            "shapes": out}


def run_ours(args):
    import torch

    import hiperml_b200 as hml
    from hiperml_b200.dist import max_over_ranks

    ctx = Ctx()
    algo = ALGO_CODES[args.algo]
    problems = workload_problems(args.workload, args.rows, args.only_n)
    clocks = ClockSampler(ctx.local)
    r = measure_gemms(ctx, problems, algo, args.dist, args.steps, args.warmup,
                      flush_l2=(args.workload == "c1"), clocks=clocks)
    bufs = r["bufs"]
    pk = peaks()
    # dominant kernel = longest per-launch time
    dom = max(range(len(bufs)), key=lambda j: r["per_kernel_ms"][j])
    k, M, N, K, *_x, dcfg = bufs[dom]
    roof = roofline_of(k, M, N, K, dcfg, r["per_kernel_ms"][dom],
                       kernel_key(args.workload, k, M, N, K, dcfg), pk)

    # ---- end to end through the host-pointer C ABI (pinned host buffers)
    e2e = None
    if not args.no_e2e and all(b[0] == "sgemm" for b in bufs):
        e2e_steps = max(1, min(args.steps, 5))
        hosts = []
        for (k_, M_, N_, K_, A, B, C, cfg) in bufs:
            hA = A.cpu().pin_memory() if not hosts or hosts[-1][0].numel() != A.numel() \
                else hosts[-1][0]
            hB = B.cpu().pin_memory()
            hC = torch.empty(M_ * N_, dtype=torch.float32).pin_memory()
            hosts.append((hA, hB, hC, M_, N_, K_))

        # column-major C = A B  ==  row-major C^T = B^T A^T : hmlSgemm(C, B, A, N, M, K)
        def e2e_step():
            from hiperml_b200._lib import check
            for (hA, hB, hC, M_, N_, K_) in hosts:
                check(hml.lib.hml_host_sgemm(0, hC.data_ptr(), hB.data_ptr(), hA.data_ptr(),
                                             N_, M_, K_, 1.0, 0.0), "hml_host_sgemm")
        e2e_step()
        ctx.barrier()
        ts = time.perf_counter()
        for _ in range(e2e_steps):
            e2e_step()
        te = time.perf_counter() - ts
        te = max_over_ranks(te, ctx.dev)
        h2d = sum(4 * (M_ * K_ + K_ * N_) for (_, _, _, M_, N_, K_) in hosts)
        d2h = sum(4 * M_ * N_ for (_, _, _, M_, N_, K_) in hosts)
        e2e = {"value": r["step_flops"] * e2e_steps * ctx.world / te / 1e12, "unit": UNIT,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "api": "hml_host_sgemm (reference-facing hmlSgemm ABI), pinned host buffers",
               "steps": e2e_steps}
        del hosts

    cpu = None
    if not args.no_cpu_baseline and ctx.rank == 0 and ctx.world == 1:
        v, cores, kind, desc, _, _ = cpu_reference_sample(
            [(k_, M_, N_, K_) for (k_, M_, N_, K_, *_r) in bufs], seconds=10.0)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": desc}

    # ---- the other configurations, one short entry each (default run on one
    # GPU only: with several ranks the rank-0 entries would hold the others at
    # the closing barrier)
    workloads = None
    if (args.workload == "sweep" and not args.no_workloads and args.rows is None
            and args.only_n is None and algo is None and args.dist == "uniform"
            and ctx.world == 1):
        del bufs
        r.pop("bufs")
        torch.cuda.empty_cache()
        workloads = []
        for name, a, dist_ in (("c1", None, "uniform"), ("gemv_n", None, "uniform"),
                               ("gemv_t", None, "uniform"), ("square", None, "uniform"),
                               ("square", None, "loguniform"), ("sweep", None, "loguniform"),
                               ("sweep", 1, "uniform")):
            workloads.append(workload_entry(ctx, name, a, dist_))
            torch.cuda.empty_cache()
        simt = workloads[-1]
        workloads.append({"workload": "split_over_simt",
                          "sweep_speedup": r["value"] / (simt["tflops"] * ctx.world),
                          "per_n_speedup": {
                              str(s["N"]): simt["per_shape"][i]["ms"] / r["per_shape"][i]["ms"]
                              for i, s in enumerate(r["per_shape"])}})
        workloads.append(batched_entry(ctx, steps=10, warmup=3))
        torch.cuda.empty_cache()
        if ctx.rank == 0:
            workloads.append(predictor_entry(ctx))
            workloads.append(reference_gpu_entry(ctx))
            workloads.append(kmeans_entry(ctx))

    if ctx.rank == 0:
        line = {
            "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": ctx.world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": r["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_desc(args.workload, args.dist),
            "run": {"parallelism": f"independent per-GPU problems x{ctx.world}",
                    "selection": ("the library's automatic choice: the B200 tuned table "
                                  "shipped as data/tuned_b200.txt (autotuner-measured), "
                                  "else the learned predictor" if algo is None else
                                  f"forced family {args.algo}: the library's heuristic "
                                  "configuration of that family"),
                    **({"rows_override": args.rows} if args.rows else {}),
                    **({"only_n": args.only_n} if args.only_n else {})},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
            "clocks": clocks.summary(), "gpu_launches": int(r["launches"]),
            "per_shape": r["per_shape"],
        }
        if workloads is not None:
            line["workloads"] = workloads
        print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def batched_entry(ctx, steps, warmup, clocks=None, with_e2e=False):
    """The batched workload: one persistent launch (replayed from a CUDA
    graph) per step, against the same 1024 problems as separate calls."""
    import numpy as np  # noqa: F401
    import torch

    import hiperml_b200 as hml
    from hiperml_b200 import datagen as dg
    from hiperml_b200.dist import max_over_ranks

    dev, stream, rank, world = ctx.dev, ctx.stream, ctx.rank, ctx.world
    shapes = batch_shapes()
    r4 = lambda x: (x + 3) // 4 * 4
    a64 = lambda x: (x + 63) // 64 * 64
    layout = []  # (ta, tb, M, N, K, lda, ldb, ldc, offA, offB, offC)
    oa = ob = oc = 0
    for (ta, tb, M, N, K) in shapes:
        lda = r4(K if ta else M)
        ldb = r4(N if tb else K)
        ldc = r4(M)
        layout.append((ta, tb, M, N, K, lda, ldb, ldc, oa, ob, oc))
        oa += a64(lda * (M if ta else K))
        ob += a64(ldb * (K if tb else N))
        oc += a64(ldc * N)
    poolA = torch.empty(oa, dtype=torch.float32, device=dev)
    poolB = torch.empty(ob, dtype=torch.float32, device=dev)
    poolC = torch.zeros(oc, dtype=torch.float32, device=dev)
    hml.fill_random(poolA, BATCH_SEED + rank * 1000, 0, dg.NORMAL)
    hml.fill_random(poolB, BATCH_SEED + rank * 1000, 1, dg.NORMAL)
    pa, pb, pc = poolA.data_ptr(), poolB.data_ptr(), poolC.data_ptr()
    descs = [(ta, tb, M, N, K, 1.0, pa + 4 * oa_, lda, pb + 4 * ob_, ldb, 0.0, pc + 4 * oc_, ldc)
             for (ta, tb, M, N, K, lda, ldb, ldc, oa_, ob_, oc_) in layout]
    plan = hml.BatchPlan(hml.COL_MAJOR, descs)
    info = plan.info()

    for _ in range(warmup):
        plan.graph_launch(stream)
    torch.cuda.synchronize()
    ctx.barrier()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(steps)]
    launches0 = hml.lib.hml_launch_count()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    sampler = clocks if clocks is not None else ClockSampler(ctx.local, period=1.0)
    with sampler:
        t0.record(stream)
        for i in range(steps):
            evs[i][0].record(stream)
            plan.graph_launch(stream)
            evs[i][1].record(stream)
        t1.record(stream)
        torch.cuda.synchronize()
    launches = hml.lib.hml_launch_count() - launches0
    ctx.barrier()
    elapsed_ms = t0.elapsed_time(t1)
    per_launch_ms = statistics.mean(a.elapsed_time(b) for a, b in evs)
    elapsed_ms = max_over_ranks(elapsed_ms, dev)
    step_flops = info["flops"]
    value = step_flops * steps * world / (elapsed_ms * 1e-3) / 1e12

    # ---- accuracy on a sample of problems (FP64 on the GPU)
    errs = []
    if rank == 0:
        for (ta, tb, M, N, K, lda, ldb, ldc, oa_, ob_, oc_) in layout[:: max(1, len(layout) // 16)]:
            e = hml.error_fp64(0, ta, tb, M, N, K, 1.0, pa + 4 * oa_, lda, pb + 4 * ob_, ldb, 0.0,
                               None, pc + 4 * oc_, ldc)
            errs.append(e)

    # ---- the same problems as 1024 separate calls (device pointers)
    def separate(config_of):
        reps = max(1, min(steps, 3))
        cfgs = [config_of(d) for d in descs]
        for d, c in zip(descs, cfgs):  # warm-up
            hml.sgemm_ex(0, d[0], d[1], d[2], d[3], d[4], 1.0, d[6], d[7], d[8], d[9], 0.0, d[11],
                         d[12], stream=stream, config=c)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            for d, c in zip(descs, cfgs):
                hml.sgemm_ex(0, d[0], d[1], d[2], d[3], d[4], 1.0, d[6], d[7], d[8], d[9], 0.0,
                             d[11], d[12], stream=stream, config=c)
        b.record(stream)
        torch.cuda.synchronize()
        return step_flops * reps / (a.elapsed_time(b) * 1e-3) / 1e12

    sep_simt = separate(lambda d: hml.select_algo(0, d[0], d[1], d[2], d[3], d[4], hml.ALGO_SIMT))
    sep_auto = separate(lambda d: None)

    # ---- end to end: pinned host operands copied in, one graph launch,
    # every C copied back
    e2e = None
    if with_e2e:
        hA = poolA.cpu().pin_memory()
        hB = poolB.cpu().pin_memory()
        hC = torch.empty(poolC.numel(), dtype=torch.float32).pin_memory()
        reps = max(1, min(steps, 2))

        def e2e_step():
            poolA.copy_(hA, non_blocking=True)
            poolB.copy_(hB, non_blocking=True)
            plan.graph_launch(stream)
            hC.copy_(poolC, non_blocking=True)
            torch.cuda.synchronize()

        e2e_step()
        ts = time.perf_counter()
        for _ in range(reps):
            e2e_step()
        te = (time.perf_counter() - ts) / reps
        te = max_over_ranks(te, dev)
        e2e = {"value": step_flops * world / te / 1e12, "unit": UNIT,
               "h2d_bytes_per_step": 4 * (poolA.numel() + poolB.numel()),
               "d2h_bytes_per_step": 4 * poolC.numel(),
               "api": "hml_batch_plan_graph_launch, operands from pinned host memory", "steps": reps}
        del hA, hB, hC

    pk = peaks()
    alg_bytes = info["bytes"]
    dom_s = per_launch_ms * 1e-3
    roof = {"bound": "hbm", "achieved": alg_bytes / dom_s / 1e9, "peak": pk["hbm_gbs"],
            "unit": "GB/s", "frac": alg_bytes / dom_s / 1e9 / pk["hbm_gbs"],
            "traffic": traffic_table().get("batched"),
            "kernel": "batch plan (tc_batch_kernel<32|64|128> + batched_kernel + split_b_batch_kernel)",
            "alg_bytes_per_launch": alg_bytes, "alg_flops_per_launch": step_flops,
            "ms_per_launch": per_launch_ms, "peak_source": pk["source"],
            "useful_tflops": step_flops / dom_s / 1e12,
            "note": ("one graph launch of the whole plan: BF16X6 tensor-core tiles for N > 8 "
                     "and FP32 SIMT tiles for N <= 8; achieved = the plan's algorithmic bytes "
                     "over its event-timed duration")}
    plan.close()
    return {"workload": "batched", "value": value, "elapsed_ms": elapsed_ms,
            "ms_per_step": elapsed_ms / steps, "steps": steps, "warmup": warmup,
            "tflops": value / world, "launches": launches, "roofline": roof, "e2e": e2e,
            "config": config_desc("batched"),
            "batch": {"tiles": info["tiles"], "ctas": info["ctas"],
                      "separate_simt_calls_tflops": sep_simt,
                      "separate_auto_calls_tflops": sep_auto,
                      "speedup_vs_separate_simt": value / world / sep_simt,
                      "speedup_vs_separate_auto": value / world / sep_auto,
                      "max_rel_err_fp64_sample": max(e[0] for e in errs) if errs else None,
                      "max_compwise_err_fp64_sample": max(e[2] for e in errs) if errs else None}}


def run_batched(args):
    ctx = Ctx()
    clocks = ClockSampler(ctx.local)
    b = batched_entry(ctx, args.steps, args.warmup, clocks=clocks, with_e2e=not args.no_e2e)
    cpu = None
    if not args.no_cpu_baseline and ctx.rank == 0 and ctx.world == 1:
        sample = [("sgemm", M, N, K) for (_ta, _tb, M, N, K) in batch_shapes()[:64]]
        v, cores, kind, desc, _, _ = cpu_reference_sample(sample, seconds=10.0)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": kind,
               "sample": "first 64 problems of the batch: " + desc}
    if ctx.rank == 0:
        line = {
            "metric": METRIC, "value": b["value"], "unit": UNIT, "n_gpus": ctx.world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": b["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_desc("batched"),
            "run": {"parallelism": f"independent per-GPU batches x{ctx.world}"},
            "roofline": b["roofline"], "cpu_baseline": cpu, "e2e": b["e2e"],
            "clocks": clocks.summary(), "gpu_launches": int(b["launches"]),
            "batch": b["batch"],
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batched":
        return run_batched(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
