#!/usr/bin/env python
"""Headline benchmark: DGEMM TFLOP/s at FP64 accuracy, 8192^3, Ozaki-INT8 vs native FP64 on B200.

Workload (the reference's dgemm contract, routines/dgemm/dgemm.h:9): row-major C = alpha*A*B + beta*C,
M = N = K = 8192, alpha = 1.5, beta = 0.5, entries u*2^e with u ~ U[-1,1) and e ~ U{-phi..phi}
(phi = 0 by default), C0 from the same law; seeded synthetic data generated on the device.

One step = one full DGEMM through the Ozaki-II CRT form (exponent and residue passes, tcgen05 INT8
products of the residues, FP64 reconstruction with the alpha/beta epilogue). The modulus count is the
smallest whose measured componentwise error |C - C_exact| / (|alpha||A||B| + |beta||C0|) on sampled
rows is no worse than the native FP64 path's on the same rows (C_exact from the library's compensated
Dot2 reference of those rows, computed on the device); that selection runs before the timed region.
The native FP64 tensor-core kernel, cuBLAS DGEMM and the Ozaki slice form are timed alongside, and
the other BASELINE configurations (exponent spreads 8 and 32, the tall and long-K shapes with scaled
rows and columns, the 512-problem grouped set) are reported as extra keys of the same line.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: replicas only (each rank runs its own 8192^3 problem; no data exchange), weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np
import statistics
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "DGEMM TFLOP/s at FP64 accuracy, 8192^3: Ozaki-INT8 vs native FP64 on 1 B200"
UNIT = "TFLOP/s"
SEED = 1234


WORKLOADS = ("square", "tall", "longk")


def workload(args):
    """(M, N, K, alpha, beta, row/column scale exponent bound, description) of the selected workload."""
    if args.workload == "tall":
        return 65536, 64, 4096, 1.0, 0.0, 64, "dgemm 65536x64x4096, rows/cols scaled 2^U{-64..64}"
    if args.workload == "longk":
        return 2048, 2048, 65536, 1.0, 0.0, 64, "dgemm 2048x2048x65536, rows/cols scaled 2^U{-64..64}"
    n = args.size
    return n, n, n, 1.5, 0.5, 0, f"dgemm {n}^3 alpha=1.5 beta=0.5 phi={args.phi}"


def reduce_max(x: float, dist=None, device="cpu") -> float:
    """The largest of every rank's x (timings are reported as the slowest rank's)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(flop_per_rank: float, world: int, ms_per_step: float) -> float:
    """Whole-job TFLOP/s of `world` replicas, each doing flop_per_rank per step, timed by the slowest."""
    return world * flop_per_rank / (ms_per_step * 1e-3) / 1e12


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0)))


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            pass
    return {}


def profile_traffic(name: str):
    """DRAM bytes per launch recorded in a committed ncu summary (profiles/<name>.txt), or None."""
    p = ROOT / "profiles" / f"{name}.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("dram_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """SM clock, power and clock-event reasons of one GPU, read through NVML every 2 ms by a
    background thread while the timed region runs (reading only; no setting is changed)."""

    REASONS = (("hw_slowdown", "nvmlClocksThrottleReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksThrottleReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksThrottleReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksThrottleReasonSwPowerCap"),
               ("hw_power_brake_slowdown", "nvmlClocksThrottleReasonHwPowerBrakeSlowdown"))

    def __init__(self, device: int, period_s: float = 0.002):
        self.device = device
        self.period = period_s
        self.rows = []
        self.error = None
        self.thread = None
        self.stop = None

    def _loop(self):
        import pynvml as nv

        h = nv.nvmlDeviceGetHandleByIndex(self.device)
        self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        masks = [(name, getattr(nv, attr)) for name, attr in self.REASONS]
        while True:
            sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
            bits = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
            self.rows.append((sm, pw, [name for name, m in masks if bits & m]))
            if self.stop.wait(self.period):
                break

    def __enter__(self):
        import threading

        try:
            import pynvml as nv

            nv.nvmlInit()
            self.stop = threading.Event()
            self.thread = threading.Thread(target=self._loop, daemon=True)
            self.thread.start()
            t0 = time.perf_counter()
            while not self.rows and time.perf_counter() - t0 < 2.0:  # the first sample precedes the work
                time.sleep(0.001)
        except Exception as e:  # no NVML on this machine
            self.error = f"NVML unavailable: {e}"
        return self

    def __exit__(self, *exc):
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=5)

    def summary(self) -> dict:
        if self.error or not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [self.error or "no samples"]}
        loaded = [r for r in self.rows if r[1] > 200.0] or self.rows
        reasons = sorted({x for r in self.rows for x in r[2]})
        return {"sm_mhz": statistics.median(r[0] for r in loaded), "sm_mhz_min": min(r[0] for r in loaded),
                "sm_max_mhz": self.max_mhz, "power_w_max": max(r[1] for r in self.rows),
                "samples": len(self.rows), "source": "NVML, 2 ms", "reasons": reasons}


# ------------------------------------------------------------------------------------------------
# CPU legs (the oracle appears only here: the CPU baseline and the reference arm)
# ------------------------------------------------------------------------------------------------
def cpu_baseline_blocked(M: int, N: int, K: int, rows: int, phi: int, smax: int, threads: int) -> dict:
    """Host blocked FP64 DGEMM on the first `rows` rows of the workload (A rows x K times K x N)."""
    import oracle

    oracle.build()
    rows = min(rows, M)
    A = oracle.fill(rows, K, 1, phi, SEED)
    B = oracle.fill(K, N, 2, phi, SEED)
    C0 = oracle.fill(rows, N, 3, phi, SEED)
    if smax > 0:
        oracle.scale_rows(A, SEED, 4, smax)
        oracle.scale_cols(B, SEED, 5, smax)
    t0 = time.perf_counter()
    oracle.dgemm_blocked(A, B, C0, 1.5, 0.5, threads)
    dt = time.perf_counter() - t0
    flop = 2.0 * rows * N * K
    return {"value": flop / dt / 1e12, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"host blocked FP64 DGEMM (oracle/oracle_blocked.c) on {rows} of {M} rows of the "
                      f"{M}x{N}x{K} problem ({flop:.3g} flop, {dt:.2f} s wall on {threads} threads)"}


_REF_STATE = {}


def _ref_init(shm_name: str, N: int, phi: int):
    import ctypes
    from multiprocessing import shared_memory

    import numpy as np
    import oracle

    shm = shared_memory.SharedMemory(name=shm_name)
    _REF_STATE["shm"] = shm
    _REF_STATE["B"] = np.ndarray((N, N), dtype=np.float64, buffer=shm.buf)
    R = oracle.ref_lib()
    if R is not None:
        _REF_STATE["fn"] = R.ref_dgemm_host
        _REF_STATE["kind"] = "reference"
    else:
        _REF_STATE["fn"] = oracle.lib().oracle_dgemm_naive
        _REF_STATE["kind"] = "port"
    _REF_STATE["N"] = N
    _REF_STATE["phi"] = phi


def _ref_rows(row0: int, rows: int):
    import numpy as np
    import oracle

    N, phi = _REF_STATE["N"], _REF_STATE["phi"]
    A = np.empty((rows, N))
    C = np.empty((rows, N))
    # rows row0.. of A and C0 of the full problem (same generator indices as the device fill)
    full_a = oracle.fill(1, (row0 + rows) * N, 1, phi, SEED).reshape(-1, N)[row0:row0 + rows]
    full_c = oracle.fill(1, (row0 + rows) * N, 3, phi, SEED).reshape(-1, N)[row0:row0 + rows]
    A[:] = full_a
    C[:] = full_c
    B = _REF_STATE["B"]
    t0 = time.perf_counter()
    _REF_STATE["fn"](A.ctypes.data, B.ctypes.data, C.ctypes.data, rows, N, N, 1.5, 0.5)
    return time.perf_counter() - t0, _REF_STATE["kind"]


def run_reference(args) -> None:
    """The reference's own CPU implementation of the path (routines/dgemm/dgemm.cpp:122-133, built
    from its sources into oracle/_ref; the oracle restatement if that build is absent), on all host
    cores (one process per core, each running the reference loop on its own rows)."""
    rank, world, _ = env_rank()
    if rank != 0:
        return
    import multiprocessing as mp
    from multiprocessing import shared_memory

    import numpy as np
    import oracle

    oracle.build()
    N = args.size
    cores = len(os.sched_getaffinity(0))
    B = oracle.fill(N, N, 2, args.phi, SEED)
    shm = shared_memory.SharedMemory(create=True, size=B.nbytes)
    try:
        np.ndarray(B.shape, dtype=np.float64, buffer=shm.buf)[:] = B
        del B
        ctx = mp.get_context("spawn")
        rows_per_proc = 1
        with ctx.Pool(cores, initializer=_ref_init, initargs=(shm.name, N, args.phi)) as pool:
            times = []
            kind = "reference"
            for step in range(args.warmup + args.steps):
                t0 = time.perf_counter()
                res = pool.starmap(_ref_rows, [(i * rows_per_proc, rows_per_proc) for i in range(cores)])
                dt = time.perf_counter() - t0
                kind = res[0][1]
                if step >= args.warmup:
                    times.append(dt)
        flops = 2.0 * cores * rows_per_proc * N * N
        ms = 1e3 * sum(times) / len(times)
        value = flops / (ms * 1e-3) / 1e12
        sample = (f"{cores * rows_per_proc} rows of the {N}^3 problem per step ({flops:.3g} flop), "
                  f"reference loop dgemm.cpp:122-133, one process per core")
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
                "config": {"workload": f"dgemm {N}^3 alpha=1.5 beta=0.5 phi={args.phi}", "M": N, "N": N, "K": N,
                           "sample_rows_per_step": cores * rows_per_proc},
                "impl": "reference",
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
    finally:
        shm.close()
        shm.unlink()


# ------------------------------------------------------------------------------------------------
# GPU arm
# ------------------------------------------------------------------------------------------------
def dot2_reference(lt, torch, A, B, C0, M, N, K, alpha, beta, rows_d, stream):
    """Compensated (double-double) reference and componentwise denominator of the sampled rows,
    computed on the device by the library (lt_dot2_rows)."""
    Cref = torch.empty(rows_d.numel(), N, dtype=torch.float64, device=A.device)
    den = torch.empty_like(Cref)
    lt.dot2_rows(A, B, C0, M, N, K, alpha, beta, rows_d, Cref, den, stream)
    return Cref, den


def max_error(lt, Crows, Cref, den, stream) -> float:
    """max |C - Cref| / den over the sampled rows (lt_componentwise_error, on the device)."""
    return lt.componentwise_error(Crows.contiguous(), Cref, den, Cref.numel(), 0.0, stream)[0]

def pairs(s: int) -> int:
    return s * (s + 1) // 2


def event_loop(torch, stream, fn, steps: int, warmup: int) -> float:
    """Mean milliseconds per call of fn over `steps` calls after `warmup`, CUDA events on `stream`."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        fn()
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b) / steps


def fill_problem(lt, torch, dev, stream, M, N, K, phi, smax):
    A = torch.empty(M, K, dtype=torch.float64, device=dev)
    B = torch.empty(K, N, dtype=torch.float64, device=dev)
    C0 = torch.empty(M, N, dtype=torch.float64, device=dev)
    lt.fill(A, M * K, SEED, 1, phi, stream)
    lt.fill(B, K * N, SEED, 2, phi, stream)
    lt.fill(C0, M * N, SEED, 3, phi, stream)
    if smax > 0:
        lt.scale_rows(A, M, K, SEED, 4, smax, stream)
        lt.scale_cols(B, K, N, SEED, 5, smax, stream)
    torch.cuda.synchronize()
    return A, B, C0


def matched_moduli(lt, torch, stream, A, B, C0, C, M, N, K, alpha, beta, ws, err_of, target, first=13):
    """Smallest modulus count (first .. 20) whose CRT-form error on the sampled rows is no worse than
    `target`; returns (n, {n: error})."""
    errs = {}
    for n in range(first, lt.LT_OZAKI_CRT_MAX_MODULI + 1):
        C.copy_(C0)
        lt.dgemm_ozaki_crt(A, B, C, M, N, K, alpha, beta, n, stream, workspace=ws)
        torch.cuda.synchronize()
        errs[n] = err_of(C)
        if errs[n] <= target:
            return n, errs
    return max(errs), errs


def config_point(lt, torch, dev, stream, M, N, K, alpha, beta, phi, smax, steps, nrows=8) -> dict:
    """One BASELINE configuration: native FP64, cuBLAS and the accuracy-matched CRT form, each with its
    TFLOP/s and max componentwise error on `nrows` sampled rows against the compensated reference."""
    A, B, C0 = fill_problem(lt, torch, dev, stream, M, N, K, phi, smax)
    C = torch.empty_like(C0)
    rows_d = torch.from_numpy(np.linspace(0, M - 1, nrows).astype(np.int64)).to(dev)
    Cref, den = dot2_reference(lt, torch, A, B, C0, M, N, K, alpha, beta, rows_d, stream)

    def err_of(Cdev):
        return max_error(lt, Cdev[rows_d], Cref, den, stream)

    flop = 2.0 * M * N * K
    out = {"M": M, "N": N, "K": K, "alpha": alpha, "beta": beta, "phi": phi, "scale_s": smax, "rows_checked": nrows}
    C.copy_(C0)
    lt.dgemm_fp64(A, B, C, M, N, K, alpha, beta, stream)
    torch.cuda.synchronize()
    e64 = err_of(C)
    ms = event_loop(torch, stream, lambda: lt.dgemm_fp64(A, B, C, M, N, K, alpha, beta, stream), steps, 2)
    out["native_fp64"] = {"tflops": flop / (ms * 1e-3) / 1e12, "ms": ms, "max_err": e64}
    C.copy_(C0)
    lt.dgemm_cublas(A, B, C, M, N, K, alpha, beta, stream)
    torch.cuda.synchronize()
    ecb = err_of(C)
    ms = event_loop(torch, stream, lambda: lt.dgemm_cublas(A, B, C, M, N, K, alpha, beta, stream), steps, 2)
    out["cublas_fp64"] = {"tflops": flop / (ms * 1e-3) / 1e12, "ms": ms, "max_err": ecb}
    ws = torch.empty(lt.ozaki_crt_workspace_size(M, N, K, lt.LT_OZAKI_CRT_MAX_MODULI), dtype=torch.uint8, device=dev)
    n, errs = matched_moduli(lt, torch, stream, A, B, C0, C, M, N, K, alpha, beta, ws, err_of, e64)
    ms = event_loop(torch, stream, lambda: lt.dgemm_ozaki_crt(A, B, C, M, N, K, alpha, beta, n, stream, workspace=ws),
                    steps, 2)
    out["ozaki_crt"] = {"moduli": n, "tflops": flop / (ms * 1e-3) / 1e12, "ms": ms, "max_err": errs[n],
                        "err_by_moduli": errs, "speedup_vs_native_fp64": out["native_fp64"]["ms"] / ms}
    lt.device_status()
    del A, B, C0, C, ws, Cref, den
    torch.cuda.empty_cache()
    return out


def grouped_point(lt, torch, dev, stream, steps, count=512) -> dict:
    """The batched configuration: `count` problems with M, N, K log-uniform in [32, 1024] (seeded),
    U[-1,1) entries, alpha = 1, beta = 0, as one grouped plan replayed from a CUDA graph (FP64 form and
    the Ozaki slice form s = 7), with aggregate TFLOP/s and the max componentwise error over one
    sampled row of every problem (compensated reference on the device)."""
    import ctypes

    rng = np.random.default_rng(SEED)
    dims = np.rint(np.exp(rng.uniform(np.log(32), np.log(1024), size=(count, 3)))).astype(int)
    bufs, table = [], (lt.GemmProblem * count)()
    flop = 0.0
    for i, (M, N, K) in enumerate(dims):
        M, N, K = int(M), int(N), int(K)
        A = torch.empty(M, K, dtype=torch.float64, device=dev)
        B = torch.empty(K, N, dtype=torch.float64, device=dev)
        C = torch.zeros(M, N, dtype=torch.float64, device=dev)
        lt.fill(A, M * K, SEED + i, 1, 0, stream)
        lt.fill(B, K * N, SEED + i, 2, 0, stream)
        bufs.append((A, B, C))
        table[i] = lt.GemmProblem(M, N, K, A.data_ptr(), B.data_ptr(), C.data_ptr(), 1.0, 0.0)
        flop += 2.0 * M * N * K
    torch.cuda.synchronize()
    refs = []
    for (A, B, C) in bufs:
        M, K, N = A.shape[0], A.shape[1], B.shape[1]
        r = torch.tensor([M // 2], dtype=torch.int64, device=dev)
        refs.append((r,) + dot2_reference(lt, torch, A, B, None, M, N, K, 1.0, 0.0, r, stream))
    L = lt.lib()
    out = {"problems": count, "dims": "M, N, K log-uniform in [32, 1024]", "flop": flop}
    for form, slices, key in ((lt.LT_FORM_FP64, 0, "fp64_plan"), (lt.LT_FORM_OZAKI, 7, "ozaki_slices7_plan")):
        plan = ctypes.c_void_p()
        lt.check(L.lt_grouped_plan_create(table, count, form, slices, ctypes.byref(plan)))
        try:
            lt.check(L.lt_grouped_plan_run_graph(plan, stream.cuda_stream))
            torch.cuda.synchronize()
            err = max(max_error(lt, C[r], Cref, den, stream) for (A, B, C), (r, Cref, den) in zip(bufs, refs))
            ms = event_loop(torch, stream, lambda: lt.check(L.lt_grouped_plan_run_graph(plan, stream.cuda_stream)),
                            steps, 2)
            name = ctypes.create_string_buffer(64)
            L.lt_grouped_plan_config(plan, name, 64)
            out[key] = {"tflops": flop / (ms * 1e-3) / 1e12, "ms": ms, "max_err_per_problem_max": err,
                        "config": name.value.decode()}
        finally:
            L.lt_grouped_plan_destroy(plan)
    lt.device_status()
    del bufs
    torch.cuda.empty_cache()
    return out


def run_ours(args) -> None:
    import torch

    import libthom_b200 as lt

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    M, N, K, alpha, beta, smax, wname = workload(args)
    flop = 2.0 * M * N * K
    A, B, C0 = fill_problem(lt, torch, dev, stream, M, N, K, args.phi, smax)
    C = torch.empty_like(C0)

    # ---- accuracy selection (untimed): the smallest modulus count of the CRT form (and slice count
    # of the slice form) no worse than native FP64, against the library's compensated (Dot2)
    # reference of sampled rows computed on the device ----
    rows = np.linspace(0, M - 1, args.check_rows).astype(np.int64)
    rows_d = torch.from_numpy(rows).to(dev)
    t0 = time.perf_counter()
    Cref, den = dot2_reference(lt, torch, A, B, C0, M, N, K, alpha, beta, rows_d, stream)
    torch.cuda.synchronize()
    ref_s = time.perf_counter() - t0

    def err_of(Cdev):
        return max_error(lt, Cdev[rows_d], Cref, den, stream)

    C.copy_(C0)
    lt.dgemm_fp64(A, B, C, M, N, K, alpha, beta, stream)
    torch.cuda.synchronize()
    err_fp64 = err_of(C)
    C.copy_(C0)
    lt.dgemm_cublas(A, B, C, M, N, K, alpha, beta, stream)
    torch.cuda.synchronize()
    err_cublas = err_of(C)
    ws = torch.empty(lt.ozaki_crt_workspace_size(M, N, K, lt.LT_OZAKI_CRT_MAX_MODULI), dtype=torch.uint8, device=dev)
    if args.moduli:
        n = args.moduli
        C.copy_(C0)
        lt.dgemm_ozaki_crt(A, B, C, M, N, K, alpha, beta, n, stream, workspace=ws)
        torch.cuda.synchronize()
        crt_errs = {n: err_of(C)}
    else:
        n, crt_errs = matched_moduli(lt, torch, stream, A, B, C0, C, M, N, K, alpha, beta, ws, err_of, err_fp64)
    ws_sl = torch.empty(lt.ozaki_workspace_size(M, N, K, lt.LT_OZAKI_MAX_SLICES), dtype=torch.uint8, device=dev)
    sl_errs, s = {}, None
    for cand in (range(args.slices, args.slices + 1) if args.slices else range(6, lt.LT_OZAKI_MAX_SLICES + 1)):
        C.copy_(C0)
        lt.dgemm_ozaki(A, B, C, M, N, K, alpha, beta, cand, stream, workspace=ws_sl)
        torch.cuda.synchronize()
        sl_errs[cand] = err_of(C)
        s = cand
        if sl_errs[cand] <= err_fp64:
            break
    lt.device_status()

    # ---- roofline denominators, measured on this GPU now with the instruction forms the kernels
    # use (lt_measure_peak: operands on chip, every SM); the FP64 probe runs after a warm-up launch
    # so that its burst figure is taken at the ramped clock ----
    int8_kind = lt.LT_PEAK_INT8_MMA_PAIR
    int8_burst = max(lt.measure_peak(int8_kind, stream) for _ in range(2)) / 1e12
    int8_peak = lt.measure_peak(int8_kind | lt.LT_PEAK_SUSTAINED, stream) / 1e12
    lt.measure_peak(lt.LT_PEAK_FP64_MMA, stream)
    fp64_burst = max(lt.measure_peak(lt.LT_PEAK_FP64_MMA, stream) for _ in range(3)) / 1e12
    fp64_peak = lt.measure_peak(lt.LT_PEAK_FP64_MMA | lt.LT_PEAK_SUSTAINED, stream) / 1e12

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        return reduce_max(x, dist, dev)

    def crt_step(ev=None):
        if ev is not None:
            ev[0].record(stream)
        lt.ozaki_crt_split(A, B, M, N, K, n, ws, stream)
        if ev is not None:
            ev[1].record(stream)
        lt.ozaki_crt_multiply(M, N, K, n, ws, stream)
        if ev is not None:
            ev[2].record(stream)
        lt.ozaki_crt_reconstruct(C, M, N, K, alpha, beta, n, ws, stream)
        if ev is not None:
            ev[3].record(stream)

    # ---- headline: the CRT form, inputs resident in HBM (512 MiB each > 126 MB L2); the clocks are
    # sampled from before the warm-up to the end of the timed steps ----
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        for _ in range(args.warmup):
            crt_step()
        barrier()
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for i in range(args.steps):
            crt_step(ev[i])
        stop.record(stream)
        barrier()
    total_ms = max_over_ranks(start.elapsed_time(stop))
    split_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in ev)
    mult_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in ev)
    recon_ms = statistics.mean(e[2].elapsed_time(e[3]) for e in ev)
    lt.device_status()
    ms_step = total_ms / args.steps
    value = world * flop / (ms_step * 1e-3) / 1e12

    # ---- native FP64 tensor-core path, cuBLAS and the slice form, same inputs ----
    def time_loop(fn) -> float:
        for _ in range(args.warmup):
            fn()
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            fn()
        b.record(stream)
        barrier()
        return max_over_ranks(a.elapsed_time(b)) / args.steps

    fp64_ms = time_loop(lambda: lt.dgemm_fp64(A, B, C, M, N, K, alpha, beta, stream))
    cublas_ms = time_loop(lambda: lt.dgemm_cublas(A, B, C, M, N, K, alpha, beta, stream))
    slices_ms = time_loop(lambda: lt.dgemm_ozaki(A, B, C, M, N, K, alpha, beta, s, stream, workspace=ws_sl))
    lt.device_status()
    del ws_sl

    # ---- end to end through the C ABI with host buffers (pinned): lt_dgemm_ozaki_crt_host copies A,
    # B and C0 in and C out inside the call (row panels, copies overlapping the kernels). C is updated
    # in place, so each step reads the previous step's C as its C0: same work every step. ----
    Ah = torch.empty(M, K, dtype=torch.float64, pin_memory=True)
    Bh = torch.empty(K, N, dtype=torch.float64, pin_memory=True)
    Ch = torch.empty(M, N, dtype=torch.float64, pin_memory=True)
    Ah.copy_(A)
    Bh.copy_(B)
    Ch.copy_(C0)
    e2e_steps = max(1, min(args.steps, 5))

    def e2e_step():
        lt.dgemm_ozaki_crt_host(Ah, Bh, Ch, M, N, K, alpha, beta, n, stream)

    e2e_step()
    barrier()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    b.record(stream)
    barrier()
    e2e_ms = max_over_ranks(a.elapsed_time(b)) / e2e_steps
    e2e_value = world * flop / (e2e_ms * 1e-3) / 1e12
    del Ah, Bh, Ch

    extra = {}
    if args.configs and world == 1:
        del A, B, C0, C, ws
        torch.cuda.empty_cache()
        st = max(2, min(args.steps, 3))
        extra["config2_phi8"] = config_point(lt, torch, dev, stream, 8192, 8192, 8192, 1.5, 0.5, 8, 0, st)
        extra["config2_phi32"] = config_point(lt, torch, dev, stream, 8192, 8192, 8192, 1.5, 0.5, 32, 0, st)
        extra["config4a_tall"] = config_point(lt, torch, dev, stream, 65536, 64, 4096, 1.0, 0.0, 0, 64, st)
        extra["config4b_longk"] = config_point(lt, torch, dev, stream, 2048, 2048, 65536, 1.0, 0.0, 0, 64, st)
        extra["config3_grouped"] = grouped_point(lt, torch, dev, stream, st)

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    peaks = measured_peaks()
    bf16 = peaks.get("bf16_tflops")
    hbm = peaks.get("hbm_gbs")
    int8_ops = n * flop
    achieved = int8_ops / (mult_ms * 1e-3) / 1e12
    traffic = profile_traffic(f"crt_pair_{M}x{N}x{K}_n{n}")
    split_bytes = (16 + n) * (M * K + K * N)
    recon_bytes = (n + (16 if beta != 0.0 else 8)) * M * N
    cpu = None
    if world == 1 and not args.no_cpu:
        cpu = cpu_baseline_blocked(M, N, K, args.cpu_rows, args.phi, smax, len(os.sched_getaffinity(0)))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 (int8 residues, int32 accumulate, f64 reconstruction)",
        "data": "synthetic (seeded generator)",
        "config": {"workload": f"{wname}, Ozaki-II CRT form with {n} moduli",
                   "M": M, "N": N, "K": K, "alpha": alpha, "beta": beta, "phi": args.phi, "scale_s": smax,
                   "moduli": n, "int8_products": n,
                   "l2": f"inputs larger than L2 (A {8 * M * K / 2**20:.0f} MiB), no flush",
                   "parallelism": f"replicas x{world}"},
        "accuracy": {"max_componentwise_err": {"ozaki_crt": crt_errs[n], "native_fp64": err_fp64, "cublas": err_cublas,
                                               "ozaki_slices": sl_errs[s]},
                     "ozaki_crt_by_moduli": crt_errs, "ozaki_slices_by_count": sl_errs, "rows_checked": len(rows),
                     "reference": f"compensated Dot2 on {len(rows)} rows, on the device (lt_dot2_rows, "
                                  f"{ref_s:.2f} s)"},
        "native_fp64": {"value": world * flop / (fp64_ms * 1e-3) / 1e12, "ms_per_step": fp64_ms,
                        "frac_of_dmma_peak": flop / (fp64_ms * 1e-3) / 1e12 / fp64_peak},
        "cublas_fp64": {"value": world * flop / (cublas_ms * 1e-3) / 1e12, "ms_per_step": cublas_ms},
        "ozaki_slices": {"slices": s, "pairs": pairs(s), "value": world * flop / (slices_ms * 1e-3) / 1e12,
                         "ms_per_step": slices_ms},
        "speedup_vs_native_fp64": fp64_ms / ms_step,
        "stages_ms": {"split": split_ms, "multiply": mult_ms, "reconstruct": recon_ms},
        "roofline": {"bound": "tensor", "kernel": "crt_pair_kernel",
                     "achieved": achieved, "peak": int8_peak, "unit": "TOP/s (INT8)", "frac": achieved / int8_peak,
                     "peak_source": "measured in this run, sustained: lt_measure_peak(tcgen05.mma.cta_group::2 "
                                    "kind::i8 M256 N128 | LT_PEAK_SUSTAINED), operands on chip, all SMs, after 0.5 s "
                                    "at the power limit",
                     "peak_burst": int8_burst, "frac_of_burst": achieved / int8_burst,
                     "peak_bf16x2": 2.0 * bf16 if bf16 else None,
                     "frac_of_bf16x2": achieved / (2.0 * bf16) if bf16 else None,
                     "traffic": traffic,
                     "algorithmic": f"{n} INT8 residue products x 2MNK = {int8_ops:.4g} ops per launch"},
        "roofline_split": {"bound": "hbm",
                           "kernels": "crt_stats_kernel, crt_shift_kernel, crt_split_rows_kernel, crt_split_cols_kernel",
                           "achieved": split_bytes / (split_ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                           "frac": split_bytes / (split_ms * 1e-3) / 1e9 / hbm if hbm else None,
                           "algorithmic": f"(16 + {n}) (MK + KN) bytes: A, B read twice, {n} residue bytes written"},
        "roofline_reconstruct": {"bound": "hbm", "kernel": "crt_recon_kernel",
                                 "achieved": recon_bytes / (recon_ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                                 "frac": recon_bytes / (recon_ms * 1e-3) / 1e9 / hbm if hbm else None,
                                 "algorithmic": f"({n} residue bytes + C0 read + C written) per element of C"},
        "roofline_fp64": {"bound": "tensor", "kernel": "dgemm_fp64_kernel",
                          "achieved": flop / (fp64_ms * 1e-3) / 1e12, "peak": fp64_peak,
                          "unit": "TFLOP/s (FP64)", "frac": flop / (fp64_ms * 1e-3) / 1e12 / fp64_peak,
                          "peak_source": "measured in this run, sustained: lt_measure_peak(mma.sync m16n8k16 f64 "
                                         "| LT_PEAK_SUSTAINED)", "peak_burst": fp64_burst},
        "e2e": {"value": e2e_value, "unit": UNIT,
                "h2d_bytes_per_step": 8 * (M * K + K * N + (M * N if beta != 0.0 else 0)),
                "d2h_bytes_per_step": 8 * M * N, "ms_per_step": e2e_ms,
                "path": "lt_dgemm_ozaki_crt_host C ABI on pinned host buffers: H2D of A, B, C0 and D2H of C inside "
                        "the call, row panels overlapping the copies with the kernels"},
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        # per timed step: crt_stats_kernel, crt_shift_kernel, crt_split_rows_kernel, crt_split_cols_kernel,
        # crt_pair_kernel, crt_recon_kernel
        "gpu_launches": 6 * args.steps,
    }
    line.update(extra)
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_sweep(args) -> None:
    """The 8192^3 slice-count table: for phi in {0, 8, 32} (entries u 2^e, e ~ U{-phi..phi}), the
    native FP64 kernel, cuBLAS and the Ozaki path at s = 3..8 (and up to 12 when 8 is not enough),
    each with its CUDA-event time and its max componentwise error on sampled rows against the
    compensated Dot2 reference (lt_dot2_rows) and against the native FP64 result C64. One JSON line
    per phi."""
    import numpy as np
    import torch

    import libthom_b200 as lt

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    n = args.size
    flop = 2.0 * n ** 3
    A = torch.empty(n, n, dtype=torch.float64, device=dev)
    B = torch.empty_like(A)
    C0 = torch.empty_like(A)
    C = torch.empty_like(A)
    ws = torch.empty(lt.ozaki_workspace_size(n, n, n, lt.LT_OZAKI_MAX_SLICES), dtype=torch.uint8, device=dev)
    rows = np.linspace(0, n - 1, args.check_rows).astype(np.int64)
    rows_d = torch.from_numpy(rows).to(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for _ in range(args.warmup):
            C.copy_(C0)
            fn()
        ts = []
        for _ in range(args.steps):
            C.copy_(C0)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    for phi in (0, 8, 32):
        lt.fill(A, n * n, SEED, 1, phi, stream)
        lt.fill(B, n * n, SEED, 2, phi, stream)
        lt.fill(C0, n * n, SEED, 3, phi, stream)
        torch.cuda.synchronize()
        Cref, den = dot2_reference(lt, torch, A, B, C0, n, n, n, 1.5, 0.5, rows_d, stream)
        res = {}
        ms = timed(lambda: lt.dgemm_fp64(A, B, C, n, n, n, 1.5, 0.5, stream))
        c64 = C[rows_d]
        res["native_fp64"] = {"tflops": flop / (ms * 1e-3) / 1e12, "ms": ms,
                              "err_vs_dot2": max_error(lt, c64, Cref, den, stream)}
        ms = timed(lambda: lt.dgemm_cublas(A, B, C, n, n, n, 1.5, 0.5, stream))
        res["cublas"] = {"tflops": flop / (ms * 1e-3) / 1e12, "ms": ms,
                         "err_vs_dot2": max_error(lt, C[rows_d], Cref, den, stream)}
        for sl in range(3, lt.LT_OZAKI_MAX_SLICES + 1):
            ms = timed(lambda: lt.dgemm_ozaki(A, B, C, n, n, n, 1.5, 0.5, sl, stream, workspace=ws))
            cs = C[rows_d]
            e = max_error(lt, cs, Cref, den, stream)
            res[f"ozaki{sl}"] = {"tflops": flop / (ms * 1e-3) / 1e12, "ms": ms, "err_vs_dot2": e,
                                 "err_vs_c64": max_error(lt, cs, c64, den, stream)}
            if sl >= 8 and e <= res["native_fp64"]["err_vs_dot2"]:
                break
        lt.device_status()
        print(json.dumps({"sweep": f"{n}^3 alpha=1.5 beta=0.5 phi={phi}", "rows_checked": len(rows),
                          "reference": "compensated Dot2 on the device (lt_dot2_rows)", "results": res}), flush=True)


# ------------------------------------------------------------------------------------------------
# hgemm routine (routines/hgemm/hgemm.cu): FP16 GEMM on the tcgen05 kind::f16 kernel
# ------------------------------------------------------------------------------------------------
HGEMM_METRIC = "HGEMM TFLOP/s (FP16 inputs, FP32 accumulation, FP16 output), 8192^3 on 1 B200"


def _hgemm_inputs_host(n: int, rows: int):
    """Rows 0..rows-1 of A and all of B of the hgemm workload, uniform [0, 1) rounded to FP16 (the
    reference runner's inputs, routines/hgemm/hgemm.cu:107-121), from numpy's seeded generator."""
    import numpy as np

    rng = np.random.default_rng(SEED)
    B = rng.random((n, n), dtype=np.float32).astype(np.float16).view(np.uint16)
    A = rng.random((rows, n), dtype=np.float32).astype(np.float16).view(np.uint16)
    return np.ascontiguousarray(A), np.ascontiguousarray(B)


def _hgemm_ref_rows(args_tuple):
    """One worker's share of the reference's HGEMM host loop (built into oracle/_ref), or of its
    restatement when that build is absent: rows of C = A B for A rows x B."""
    A, B, n = args_tuple
    import numpy as np
    import oracle

    C = np.zeros((A.shape[0], n), dtype=np.uint16)
    R = oracle.ref_hgemm_lib()
    t0 = time.perf_counter()
    if R is not None:
        R.ref_hgemm_host(A.ctypes.data, B.ctypes.data, C.ctypes.data, A.shape[0], n, n, 0x3C00, 0x0000)
        kind = "reference"
    else:
        oracle.lib().oracle_hgemm_ref(A.ctypes.data, B.ctypes.data, C.ctypes.data, C.ctypes.data, A.shape[0], n, n,
                                      1.0, 0.0, None, 0)
        kind = "port"
    return time.perf_counter() - t0, kind


def hgemm_cpu_rows(n: int, rows: int, workers: int) -> dict:
    """Times the reference HGEMM host loop on `rows` rows of the n^3 problem with `workers`
    processes (the loop keeps its operands in process-wide statics, so one process per worker)."""
    import multiprocessing as mp

    A, B = _hgemm_inputs_host(n, rows)
    per = max(1, rows // workers)
    chunks = [(A[i:i + per], B, n) for i in range(0, rows, per)]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(len(chunks)) as pool:
        res = pool.map(_hgemm_ref_rows, chunks)
    wall = time.perf_counter() - t0
    loop = max(r[0] for r in res)
    flop = 2.0 * rows * n * n
    return {"value": flop / loop / 1e12, "unit": UNIT, "cores": len(chunks), "kind": res[0][1],
            "seconds": loop, "wall_seconds": wall, "flop": flop}


def run_hgemm(args) -> None:
    import torch

    import libthom_b200 as lt

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    n = args.size
    M = N = K = n
    flop = 2.0 * M * N * K
    g = torch.Generator(device=dev).manual_seed(SEED + rank)
    A = torch.rand(M, K, device=dev, generator=g).half()
    B = torch.rand(K, N, device=dev, generator=g).half()
    C = torch.zeros(M, N, dtype=torch.float16, device=dev)
    R = torch.zeros_like(C)
    cfg = lt.lib().lt_hgemm_default_config(M, N, K)

    # ---- agreement with cuBLAS (FP32 accumulation) under the reference's acceptance test ----
    lt.hgemm_tc(A, B, C, M, N, K, 1.0, 0.0, stream)
    lt.hgemm_cublas(A, B, R, M, N, K, 1.0, 0.0, compute_f32=True, stream=stream)
    torch.cuda.synchronize()
    c, r = C.float(), R.float()
    diff = (c - r).abs()
    rel = diff / r.abs().clamp_min(1e-3)
    differ = int(((rel > 1e-2) & (diff > 1e-3)).sum().item())
    max_rel = float(rel.max().item())
    bitwise = float((C.view(torch.int16) == R.view(torch.int16)).float().mean().item())
    del c, r, diff, rel
    lt.device_status()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- headline: inputs resident in HBM (A, B, C: 384 MiB in all, above the 126 MB L2) ----
    for _ in range(args.warmup):
        lt.hgemm_tc(A, B, C, M, N, K, 1.0, 0.0, stream)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    with ClockSampler(local) as clk:
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for i in range(args.steps):
            ev[i][0].record(stream)
            lt.hgemm_tc(A, B, C, M, N, K, 1.0, 0.0, stream)
            ev[i][1].record(stream)
        stop.record(stream)
        barrier()
    total_ms = reduce_max(start.elapsed_time(stop), dist, dev)
    kern_ms = statistics.mean(a.elapsed_time(b) for a, b in ev)
    lt.device_status()
    ms_step = total_ms / args.steps
    value = world * flop / (ms_step * 1e-3) / 1e12

    def time_loop(fn) -> float:
        for _ in range(args.warmup):
            fn()
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            fn()
        b.record(stream)
        barrier()
        return reduce_max(a.elapsed_time(b), dist, dev) / args.steps

    cublas32_ms = time_loop(lambda: lt.hgemm_cublas(A, B, R, M, N, K, 1.0, 0.0, True, stream))
    cublas16_ms = time_loop(lambda: lt.hgemm_cublas(A, B, R, M, N, K, 1.0, 0.0, False, stream))

    # ---- end to end: pinned host A and B copied in, the product, C copied out, every step ----
    Ah = torch.empty(M, K, dtype=torch.float16, pin_memory=True)
    Bh = torch.empty(K, N, dtype=torch.float16, pin_memory=True)
    Ch = torch.empty(M, N, dtype=torch.float16, pin_memory=True)
    Ah.copy_(A)
    Bh.copy_(B)
    e2e_steps = max(1, min(args.steps, 5))

    def e2e_step():
        A.copy_(Ah, non_blocking=True)
        B.copy_(Bh, non_blocking=True)
        lt.hgemm_tc(A, B, C, M, N, K, 1.0, 0.0, stream)
        Ch.copy_(C, non_blocking=True)

    e2e_step()
    barrier()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    b.record(stream)
    barrier()
    e2e_ms = reduce_max(a.elapsed_time(b), dist, dev) / e2e_steps
    del Ah, Bh, Ch

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    peaks = measured_peaks()
    burst, sustained = peaks.get("bf16_tflops"), peaks.get("bf16_tflops_sustained")
    achieved = flop / (kern_ms * 1e-3) / 1e12
    peak = burst if burst else 1590.0
    cpu = None
    if world == 1 and not args.no_cpu:
        rows = max(1, args.cpu_rows // 64)
        cb = hgemm_cpu_rows(n, rows, 1)
        cpu = {"value": cb["value"], "unit": UNIT, "cores": cb["cores"], "kind": cb["kind"],
               "sample": f"the reference's HGEMM host loop (routines/hgemm/hgemm.cu:135-149) on {rows} of {M} "
                         f"rows of the {n}^3 problem ({cb['flop']:.3g} flop, {cb['seconds']:.2f} s, 1 thread)"}
    line = {
        "metric": HGEMM_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f16 (f32 accumulate)", "data": "synthetic (uniform [0,1) rounded to FP16)",
        "config": {"workload": f"hgemm {n}^3 alpha=1 beta=0 (the reference runner's setting), config "
                               f"{lt.hgemm_configs()[cfg]}", "M": M, "N": N, "K": K,
                   "l2": "inputs larger than L2 in total (A, B, C 128 MiB each), no flush",
                   "parallelism": f"replicas x{world}"},
        "accuracy": {"vs_cublas_f32": {"entries_failing_reference_test": differ, "max_rel_diff": max_rel,
                                       "bitwise_equal_fraction": bitwise}},
        "cublas_f32_accumulate": {"value": world * flop / (cublas32_ms * 1e-3) / 1e12, "ms_per_step": cublas32_ms},
        "cublas_f16_accumulate": {"value": world * flop / (cublas16_ms * 1e-3) / 1e12, "ms_per_step": cublas16_ms,
                                  "note": "the reference's own baseline call (hgemm_cublas.cu:10-22)"},
        "roofline": {"bound": "tensor", "kernel": "hgemm_pair_kernel", "achieved": achieved, "peak": peak,
                     "unit": "TFLOP/s", "frac": achieved / peak,
                     "peak_source": "MEASURED_PEAKS.json bf16_tflops (cuBLAS bf16 GEMM burst; FP16 runs at "
                                    "the bf16 rate)" if burst else "fallback 1590 TFLOP/s",
                     "peak_sustained": sustained, "frac_of_sustained": achieved / sustained if sustained else None,
                     "traffic": profile_traffic("hgemm_pair_8192") if n == 8192 else None,
                     "algorithmic": f"2MNK = {flop:.4g} flop per launch"},
        "e2e": {"value": world * flop / (e2e_ms * 1e-3) / 1e12, "unit": UNIT,
                "h2d_bytes_per_step": 2 * (M * K + K * N), "d2h_bytes_per_step": 2 * M * N, "ms_per_step": e2e_ms,
                "path": "pinned host A, B copied in, lt_hgemm, C copied out, on one stream"},
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "gpu_launches": args.steps,
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_reference_hgemm(args) -> None:
    """The reference's own CPU implementation of the hgemm check loop (routines/hgemm/hgemm.cu:
    135-149, built from its sources into oracle/_ref; the restatement if absent), one process per
    host core, each on its own rows of the 8192^3 problem."""
    rank, world, _ = env_rank()
    if rank != 0:
        return
    n = args.size
    cores = len(os.sched_getaffinity(0))
    times, kind = [], "reference"
    for step in range(args.warmup + args.steps):
        cb = hgemm_cpu_rows(n, cores, cores)
        kind = cb["kind"]
        if step >= args.warmup:
            times.append(cb["seconds"])
    flop = 2.0 * cores * n * n
    ms = 1e3 * statistics.mean(times)
    value = flop / (ms * 1e-3) / 1e12
    sample = f"{cores} rows of the {n}^3 problem per step ({flop:.3g} flop), one process per core"
    line = {"metric": HGEMM_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f16 (f32 accumulate)", "data": "synthetic (uniform [0,1) rounded to FP16)",
            "config": {"workload": f"hgemm {n}^3 alpha=1 beta=0", "M": n, "N": n, "K": n,
                       "sample_rows_per_step": cores},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_peaks(args) -> None:
    """Prints the measured tensor-pipe rates of the current GPU (lt_measure_peak) as one JSON line:
    FP64 mma.sync and the INT8 tcgen05 shapes (M128 N128, M128 N256, CTA pair M256 N128), each as
    the best of three single launches (burst) and after 0.5 s at the power limit (sustained), with
    the SM clock (NVML, read only) before and after."""
    import libthom_b200 as lt

    def sm_mhz():
        try:
            import pynvml as nv

            nv.nvmlInit()
            return nv.nvmlDeviceGetClockInfo(nv.nvmlDeviceGetHandleByIndex(0), nv.NVML_CLOCK_SM)
        except Exception:
            return None

    kinds = {"fp64_mma_tflops": lt.LT_PEAK_FP64_MMA, "int8_m128n128_tops": lt.LT_PEAK_INT8_MMA_N128,
             "int8_m128n256_tops": lt.LT_PEAK_INT8_MMA_N256, "int8_pair_m256n128_tops": lt.LT_PEAK_INT8_MMA_PAIR}
    res = {"sm_mhz_before": sm_mhz()}
    for name, kind in kinds.items():
        vals = [lt.measure_peak(kind) / 1e12 for _ in range(3)]
        res[name] = max(vals)
        res[name + "_all"] = vals
        res[name + "_sustained"] = lt.measure_peak(kind | lt.LT_PEAK_SUSTAINED) / 1e12
    res["sm_mhz_after"] = sm_mhz()
    print(json.dumps(res), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--size", type=int, default=8192)
    ap.add_argument("--workload", choices=list(WORKLOADS), default="square",
                    help="square: size^3, alpha=1.5, beta=0.5 (the headline); tall: 65536x64x4096 and longk: "
                         "2048x2048x65536, alpha=1, beta=0, rows of A / columns of B scaled by 2^s, s ~ U{-64..64}")
    ap.add_argument("--phi", type=int, default=0)
    ap.add_argument("--slices", type=int, default=0, help="fix the slice form's slice count (0 = accuracy-matched)")
    ap.add_argument("--moduli", type=int, default=0, help="fix the CRT form's modulus count (0 = accuracy-matched)")
    ap.add_argument("--no-configs", dest="configs", action="store_false",
                    help="skip the other BASELINE configurations (phi 8 and 32, 65536x64x4096, 2048x2048x65536, "
                         "the 512-problem grouped set)")
    ap.add_argument("--check-rows", type=int, default=16)
    ap.add_argument("--cpu-rows", type=int, default=1024)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--routine", choices=["dgemm", "hgemm"], default="dgemm",
                    help="dgemm: the headline (default); hgemm: the FP16 routine on its tcgen05 kernel")
    ap.add_argument("--sweep", action="store_true",
                    help="print the phi x slice-count table (error and TFLOP/s of every form) instead")
    ap.add_argument("--peaks", action="store_true",
                    help="print the measured tensor-pipe rates of this GPU (lt_measure_peak) instead")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)  # at least 3 untimed warm-up steps, reported as run
    if args.peaks:
        run_peaks(args)
    elif args.routine == "hgemm":
        run_reference_hgemm(args) if args.impl == "reference" else run_hgemm(args)
    elif args.sweep:
        run_sweep(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
