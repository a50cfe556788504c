"""Benchmark of the skinny SGEMM/SGEMV path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload sweep|c1|gemv_n|gemv_t|square]

Default workload ("sweep"): the skinny SGEMM precision sweep, C = A * B
column-major with M = 65536, K = 4096 and N in {8, 32, 64, 128}, A and B
uniform[-1, 1] from seed 0 (synthetic, generated on the device by the
library's SplitMix64 stream).  One step = the four GEMMs, each through
hml_sgemm_ex with the library's own configuration choice.  A is 1 GiB
(> the 126 MB L2), so no L2 flush is needed between steps.

The JSON line reports useful TFLOPS (2*M*N*K per GEMM), the roofline of the
dominant kernel, an end-to-end figure through the host-pointer C ABI
(hml_host_sgemm, pinned host buffers, copies inside the timed region), the
reference's CPU loop as a CPU baseline, the SM clocks sampled during the
timed region and the number of library kernel launches in it.

With torchrun (N > 1) every rank runs the same per-GPU workload on its own
data (weak scaling: the GEMMs are independent row blocks of a larger
problem, so there is no data-path collective); the timing is the max over
ranks.  --impl reference times the reference's own CPU implementation
(hmlSgemmCpu from oracle/_ref) on a bounded sample on rank 0.
"""
from __future__ import annotations

import argparse
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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sweep",
                    choices=["sweep", "c1", "gemv_n", "gemv_t", "square", "batched"])
    ap.add_argument("--algo", default="auto", choices=["auto", "simt", "bf16x3", "bf16x6", "tf32x3"],
                    help="force one algorithm family (default: the library's choice)")
    ap.add_argument("--rows", type=int, default=None,
                    help="sweep workload: M other than 65536 (small cases for profiler captures)")
    ap.add_argument("--only-n", type=int, default=None,
                    help="sweep workload: run only this N (profiler captures)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    return ap.parse_args()


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


def config_desc(name):
    if name == "sweep":
        return {"workload": f"skinny SGEMM C=A*B col-major, M={SWEEP_M}, K={SWEEP_K}, "
                            f"N in {list(SWEEP_N)} (one step = the 4 GEMMs)",
                "M": SWEEP_M, "K": SWEEP_K, "N": list(SWEEP_N), "alpha": 1.0, "beta": 0.0,
                "layout": "column-major NN", "inputs": "uniform[-1,1], seed 0",
                "l2": "A is 1 GiB per GEMM (> 126 MB L2): inputs larger than L2, no flush"}
    if name == "c1":
        return {"workload": "skinny SGEMM col-major M=4096, N=16, K=4096", "M": 4096, "N": 16,
                "K": 4096, "inputs": "uniform[-1,1], seed 0",
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
    return {"workload": "square SGEMM 8192^3 col-major", "inputs": "uniform[-1,1], seed 0",
            "l2": "compute bound; inputs 256 MiB each"}


# -------------------------------------------------------------- reference
def cpu_reference_sample(problems, seconds=10.0, threads=None):
    """Times the reference's own hmlSgemmCpu / hmlSgemvCpu (oracle/_ref, or
    the C restatement when the reference build is absent) on row slices of
    each problem, on all host cores (one independent row block per thread).
    Returns (TFLOPS, cores, kind, sample description)."""
    import ctypes
    from concurrent.futures import ThreadPoolExecutor

    import numpy as np

    import oracle
    from hiperml_b200 import datagen as dg

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
    return total_flops / elapsed / 1e12, cores, kind, desc


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
    vals = []
    cores = kind = desc = None
    for i in range(args.warmup + args.steps):
        v, cores, kind, desc = cpu_reference_sample(problems, seconds=per_step)
        if i >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    step_flops = sum(flops_of(*p) for p in problems)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "sample_problems": len(problems),
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": step_flops / (value * 1e12) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_desc(args.workload),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# -------------------------------------------------------------------- ours
def run_ours(args):
    import torch

    import hiperml_b200 as hml
    from hiperml_b200 import datagen as dg
    from hiperml_b200.dist import max_over_ranks

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist_on = world > 1
    if dist_on:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()

    problems = workload_problems(args.workload, args.rows, args.only_n)
    algo = {"auto": None, "simt": 1, "bf16x3": 2, "bf16x6": 3, "tf32x3": 4}[args.algo]

    # ---- device operands (one A shared by the sweep's GEMMs)
    bufs = []
    Ashared = None
    for (k, M, N, K) in problems:
        if k == "sgemm":
            if Ashared is None or Ashared.numel() != M * K:
                Ashared = torch.empty(M * K, dtype=torch.float32, device=dev)
                hml.fill_random(Ashared, 0 + rank * 1000, 0, dg.UNIFORM)
            B = torch.empty(K * N, dtype=torch.float32, device=dev)
            hml.fill_random(B, 0 + rank * 1000, 1, dg.UNIFORM)
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
    flush = None
    if args.workload == "c1":
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB

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
           for _ in range(n_items)] for _ in range(args.steps)]

    def step(i=None):
        if flush is not None:
            flush.fill_(float(i or 0))
        for j, item in enumerate(bufs):
            if i is not None:
                ev[i][j][0].record(stream)
            launch(item)
            if i is not None:
                ev[i][j][1].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if hml.device_error() != 0:
        raise RuntimeError("device wait expired during warm-up")

    if dist_on:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = hml.lib.hml_launch_count()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        t0.record(stream)
        for i in range(args.steps):
            step(i)
        t1.record(stream)
        torch.cuda.synchronize()
    launches = hml.lib.hml_launch_count() - launches0
    if dist_on:
        dist.barrier()
    elapsed_ms = t0.elapsed_time(t1)
    per_kernel_ms = [statistics.mean(ev[i][j][0].elapsed_time(ev[i][j][1]) for i in
                                     range(args.steps)) for j in range(n_items)]
    if flush is not None:
        # the flush is outside the measured GEMM events; time only the GEMMs
        elapsed_ms = sum(sum(ev[i][j][0].elapsed_time(ev[i][j][1]) for j in range(n_items))
                         for i in range(args.steps))
    elapsed_ms = max_over_ranks(elapsed_ms, dev)
    if hml.device_error() != 0:
        raise RuntimeError("device wait expired in the timed region")

    step_flops = sum(flops_of(k, M, N, K) for (k, M, N, K, *_rest) in bufs)
    value = step_flops * args.steps * world / (elapsed_ms * 1e-3) / 1e12
    pk = peaks()
    # dominant kernel = longest per-launch time
    dom = max(range(n_items), key=lambda j: per_kernel_ms[j])
    k, M, N, K, *_ = bufs[dom]
    alg_bytes = bytes_of(k, M, N, K)
    alg_flops = flops_of(k, M, N, K)
    dom_s = per_kernel_ms[dom] * 1e-3
    dcfg = bufs[dom][7]
    algo_names = {1: "simt", 2: "bf16x3", 3: "bf16x6", 4: "tf32x3"}
    key = f"{args.workload}:{k}:{M}x{N}x{K}:{algo_names.get(dcfg.algo, 'gemv') if dcfg else 'gemv'}"
    traffic = traffic_table().get(key)
    ai = alg_flops / alg_bytes
    roof = {"bound": "hbm", "achieved": alg_bytes / dom_s / 1e9, "peak": pk["hbm_gbs"],
            "unit": "GB/s", "frac": alg_bytes / dom_s / 1e9 / pk["hbm_gbs"],
            "traffic": traffic, "kernel": key, "alg_bytes_per_launch": alg_bytes,
            "alg_flops_per_launch": alg_flops, "ms_per_launch": per_kernel_ms[dom],
            "peak_source": pk["source"], "arith_intensity": ai}
    if dcfg is not None and dcfg.algo in (2, 3, 4):
        ridge = pk["bf16_tflops_sustained"] * 1e12 / (pk["hbm_gbs"] * 1e9)
        # tensor work in BF16-product units: a TF32 product runs at half the
        # BF16 rate, so TF32X3's three count as six
        products = {2: 3, 3: 6, 4: 6}[dcfg.algo]
        if ai * products > ridge:
            tc = alg_flops * products / dom_s / 1e12
            roof.update({"bound": "tensor", "achieved": tc, "peak": pk["bf16_tflops_sustained"],
                         "unit": "TFLOP/s", "frac": tc / pk["bf16_tflops_sustained"]})
    if dcfg is not None and dcfg.algo == 1:
        # SIMT FP32: nominal 148 SMs x 128 FMA lanes x 2 x 1.965 GHz
        roof["simt_fp32_tflops"] = alg_flops / dom_s / 1e12
        roof["simt_fp32_peak_nominal"] = 148 * 128 * 2 * 1.965e-3

    per_shape = []
    for j, (k, M, N, K, A, B, C, cfg) in enumerate(bufs):
        entry = {"kind": k, "M": M, "N": N, "K": K, "ms": per_kernel_ms[j],
                 "tflops": flops_of(k, M, N, K) / (per_kernel_ms[j] * 1e-3) / 1e12,
                 "gbs": bytes_of(k, M, N, K) / (per_kernel_ms[j] * 1e-3) / 1e9,
                 "config": repr(cfg) if cfg is not None else "gemv"}
        if k == "sgemm" and rank == 0:
            err = hml.error_fp64(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, None, C, M)
            entry["max_rel_err_fp64"] = err[0]
            entry["rms_rel_err_fp64"] = err[1]
            entry["compwise_err_fp64"] = err[2]
        per_shape.append(entry)

    # ---- end to end through the host-pointer C ABI (pinned host buffers)
    e2e = None
    if not args.no_e2e and all(b[0] == "sgemm" for b in bufs):
        e2e_steps = max(1, min(args.steps, 5))
        hosts = []
        for (k, M, N, K, A, B, C, cfg) in bufs:
            hA = A.cpu().pin_memory() if not hosts or hosts[-1][0].numel() != A.numel() else hosts[-1][0]
            hB = B.cpu().pin_memory()
            hC = torch.empty(M * N, dtype=torch.float32).pin_memory()
            hosts.append((hA, hB, hC, M, N, K))
        # column-major C = A B  ==  row-major C^T = B^T A^T : hmlSgemm(C, B, A, N, M, K)
        def e2e_step():
            for (hA, hB, hC, M, N, K) in hosts:
                from hiperml_b200._lib import check
                check(hml.lib.hml_host_sgemm(0, hC.data_ptr(), hB.data_ptr(), hA.data_ptr(),
                                             N, M, K, 1.0, 0.0), "hml_host_sgemm")
        e2e_step()
        if dist_on:
            dist.barrier()
        ts = time.perf_counter()
        for _ in range(e2e_steps):
            e2e_step()
        te = time.perf_counter() - ts
        te = max_over_ranks(te, dev)
        h2d = sum(4 * (M * K + K * N) for (_, _, _, M, N, K) in hosts)
        d2h = sum(4 * M * N for (_, _, _, M, N, K) in hosts)
        e2e = {"value": step_flops * e2e_steps * world / te / 1e12, "unit": UNIT,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "api": "hml_host_sgemm (reference-facing hmlSgemm ABI), pinned host buffers",
               "steps": e2e_steps}

    cpu = None
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        v, cores, kind, desc = cpu_reference_sample([(k, M, N, K) for (k, M, N, K, *_r) in bufs],
                                                    seconds=10.0)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": desc}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(config_desc(args.workload),
                           parallelism=f"independent per-GPU problems x{world}",
                           selection=("the library's automatic choice: the B200 tuned table "
                                      "shipped as data/tuned_b200.txt (autotuner-measured), "
                                      "else the learned predictor" if algo is None else
                                      f"forced family {args.algo}: the library's heuristic "
                                      "configuration of that family"),
                           **({"rows_override": args.rows} if args.rows else {}),
                           **({"only_n": args.only_n} if args.only_n else {})),
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
            "clocks": clocks.summary(), "gpu_launches": int(launches),
            "per_shape": per_shape,
        }
        print(json.dumps(line), flush=True)
    if dist_on:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_batched(args):
    """The batched workload: one persistent launch (replayed from a CUDA
    graph) per step, against the same 1024 problems as separate calls."""
    import numpy as np
    import torch

    import hiperml_b200 as hml
    from hiperml_b200 import datagen as dg
    from hiperml_b200.dist import max_over_ranks

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist_on = world > 1
    if dist_on:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()

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

    for _ in range(args.warmup):
        plan.graph_launch(stream)
    torch.cuda.synchronize()
    if dist_on:
        dist.barrier()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    launches0 = hml.lib.hml_launch_count()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        t0.record(stream)
        for i in range(args.steps):
            evs[i][0].record(stream)
            plan.graph_launch(stream)
            evs[i][1].record(stream)
        t1.record(stream)
        torch.cuda.synchronize()
    launches = hml.lib.hml_launch_count() - launches0
    if dist_on:
        dist.barrier()
    elapsed_ms = t0.elapsed_time(t1)
    per_launch_ms = statistics.mean(a.elapsed_time(b) for a, b in evs)
    elapsed_ms = max_over_ranks(elapsed_ms, dev)
    step_flops = info["flops"]
    value = step_flops * args.steps * world / (elapsed_ms * 1e-3) / 1e12

    # ---- accuracy on a sample of problems (FP64 on the GPU)
    errs = []
    if rank == 0:
        for (ta, tb, M, N, K, lda, ldb, ldc, oa_, ob_, oc_) in layout[:: max(1, len(layout) // 16)]:
            e = hml.error_fp64(0, ta, tb, M, N, K, 1.0, pa + 4 * oa_, lda, pb + 4 * ob_, ldb, 0.0,
                               None, pc + 4 * oc_, ldc)
            errs.append(e)

    # ---- the same problems as 1024 separate calls (device pointers)
    def separate(config_of):
        reps = max(1, min(args.steps, 3))
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
    if not args.no_e2e:
        hA = poolA.cpu().pin_memory()
        hB = poolB.cpu().pin_memory()
        hC = torch.empty(poolC.numel(), dtype=torch.float32).pin_memory()
        reps = max(1, min(args.steps, 2))

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
            "simt_fp32_tflops": step_flops / dom_s / 1e12,
            "simt_fp32_peak_nominal": 148 * 128 * 2 * 1.965e-3,
            "note": ("one graph launch of the whole plan: BF16X6 tensor-core tiles for N > 8 "
                     "(tc_batch_kernel<128,3> dominates) and FP32 SIMT tiles for N <= 8; "
                     "achieved = the plan's algorithmic bytes over its event-timed duration")}

    cpu = None
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        sample = [("sgemm", M, N, K) for (_ta, _tb, M, N, K) in shapes[:64]]
        v, cores, kind, desc = cpu_reference_sample(sample, seconds=10.0)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": kind,
               "sample": "first 64 problems of the batch: " + desc}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(config_desc("batched"),
                           parallelism=f"independent per-GPU batches x{world}"),
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
            "clocks": clocks.summary(), "gpu_launches": int(launches),
            "batch": {"tiles": info["tiles"], "ctas": info["ctas"],
                      "separate_simt_calls_tflops": sep_simt,
                      "separate_auto_calls_tflops": sep_auto,
                      "speedup_vs_separate_simt": value / world / sep_simt,
                      "max_rel_err_fp64_sample": max(e[0] for e in errs) if errs else None,
                      "max_compwise_err_fp64_sample": max(e[2] for e in errs) if errs else None},
        }
        print(json.dumps(line), flush=True)
    plan.close()
    if dist_on:
        dist.barrier()
        dist.destroy_process_group()
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
