#!/usr/bin/env python
"""Coded signals/s of LARS-Lasso on B200 (one JSON line on stdout).

Workload (per GPU): D 256 x 512 with unit-norm N(0,1) columns; X 256 x 100000
whose columns are D a + 0.01 N(0,1) with 12 uniformly placed N(0,1)
non-zeros; lasso mode 2 (PENALTY), lambda1 = 0.15, float32.  A step codes
the whole batch: Gram, ||x||^2, D^T X, the LARS homotopy of every signal and
the CSC assembly.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision bf16x3|fp32] [--workload lasso|uneven_omp|serve]

`value` is measured through the device entry point with inputs resident in
HBM (CUDA events on the call's stream, an L2-flushing write between steps);
`e2e` through the host entry point with pinned host buffers, copies inside
the timed region.  The correlations D^T X run as BF16 hi/lo tensor-core
products (FP32-grade, see the parity tests) unless --precision fp32; the
plain FP32 path is timed beside it (`fp32_value`).  With N > 1 (torchrun)
every rank codes its own batch with the same dictionary (weak scaling, no
collective on the data path); rank 0 prints the aggregate.  `--impl
reference` times the SPAMS reference's own CPU code (oracle/_ref) on the host
cores instead.

On one GPU the default line also carries the other benchmarked
configurations as sub-objects, each with its own value, e2e, roofline and CPU
baseline, at bounded sizes (the whole run takes a few minutes):
  "uneven_omp" (2e5 signals, --uneven-n), "dictlearn" (2000 minibatches),
  "serve" (2000 req/s for 5 s, then 1000 and 500 req/s); --no-sub-workloads
  leaves them out.

The same workloads at full size, each printing its own JSON line (one GPU):
  --workload uneven_omp  batched uneven OMP: D 512 x 2048, X 512 x 1e6,
                         s_i ~ U{1..64}, L_i = s_i + 4, eps_i = 0.5 ||noise_i||^2
  --workload serve       serving stream: Poisson arrivals at --rate req/s over
                         eight resident dictionaries, p50 / p99 latency
  --workload dictlearn   online dictionary-learning minibatch step (12x12 patches,
                         D 144 x 1024, batch 1024), one CUDA graph replay per
                         minibatch, minibatches/s (--n minibatches, default 2000)
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "spams-devel_b200"))

import numpy as np  # noqa: E402

M, K, S, NOISE, LAMBDA = 256, 512, 12, 0.01, 0.15
# The coding-kernel family on this shape: the autotuner's choice in plain runs
# (warp per signal), pinned so that a run under a profiler, whose serialised
# launches distort the tuner's timings, codes with the same kernel.
KERNEL = "warp"
METRIC = "coded signals/s (LARS-Lasso mode 2, lambda1=0.15, D 256x512, 12-sparse + 0.01 noise)"
UNIT = "signals/s"


def workload(n: int, rank: int):
    from spams_b200 import workloads as W
    if rank == 0:
        return W.config_lasso(n=n, seed=0, m=M, K=K, s=S, noise=NOISE)
    D = W.gaussian_dictionary(M, K, np.random.Generator(np.random.PCG64(0)))
    X, _, _ = W.sparse_signals(D, n, S, NOISE, np.random.Generator(np.random.PCG64(1000 + rank)))
    return X, D


def config_dict(n: int, ngpu: int, precision: str) -> dict:
    return {"workload": f"lasso_mode2_D{M}x{K}_n{n}_s{S}_noise{NOISE}_lambda{LAMBDA}",
            "m": M, "K": K, "n_per_gpu": n, "lambda1": LAMBDA, "mode": 2,
            "precision": precision, "kernel": KERNEL, "between_steps": "L2 flush (256 MiB write)",
            "parallelism": f"column shards x{ngpu}, no data-path collective"}


def measured_peaks() -> dict:
    """HBM GB/s and dense bf16 TFLOP/s (burst) measured on this pool's B200s,
    else the profiling recipe's fallback figures."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        out = {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
        try:
            out["bf16_tflops"] = float(d["bf16_tflops"])
            out["tensor_source"] = "measured"
        except Exception:
            out["bf16_tflops"], out["tensor_source"] = 1590.0, "fallback"
        return out
    except Exception:
        return {"hbm_gbs": 6650.0, "source": "fallback", "bf16_tflops": 1590.0,
                "tensor_source": "fallback"}


def corr_roofline(m: int, K: int, Kp: int, n: int, ms: float, peaks: dict, terms: int = 3) -> dict:
    """The correlation stage D^T X on the tensor cores: algorithmic FLOPs 2 m K n
    (the BF16 split executes `terms` times as many: 3 for the hi / lo form of
    the Lasso, 6 for the three-piece form of OMP), and its bytes (X in, the
    Kp x n correlations out) against HBM."""
    if not ms or ms <= 0:
        return None
    alg = 2.0 * m * K * n
    exe = float(terms) * alg
    byt = 4.0 * m * n + 4.0 * Kp * n
    return {"kernel": "tc_corr_xs_kernel", "bound": "tensor", "ms": ms, "terms": terms,
            "achieved_tflops": exe / (ms / 1e3) / 1e12,
            "achieved_tflops_algorithmic": alg / (ms / 1e3) / 1e12,
            "peak": peaks["bf16_tflops"], "unit": "TFLOP/s",
            "frac": exe / (ms / 1e3) / 1e12 / peaks["bf16_tflops"],
            "frac_algorithmic": alg / (ms / 1e3) / 1e12 / peaks["bf16_tflops"],
            "peak_source": peaks["tensor_source"],
            "hbm_gbs": byt / (ms / 1e3) / 1e9, "hbm_frac": byt / (ms / 1e3) / 1e9 / peaks["hbm_gbs"],
            "flops_executed": exe, "flops_algorithmic": alg, "bytes": byt}


def profiled_traffic() -> float | None:
    """DRAM bytes per launch of the LARS kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "lars_kernel_lasso256x512.md")
    try:
        with open(p) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) > 8:
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_reference_rate(X, D, target_s: float, threads: int):
    """The reference's lasso (oracle/_ref, OpenMP) on a bounded sample of the
    workload: returns (signals/s, sample size, threads used)."""
    from oracle import oracle as O
    O.build_ref()
    n = X.shape[1]
    cal = min(n, 2000)
    t = time.perf_counter()
    O.ref_lasso(X[:, :cal], D, lambda1=LAMBDA, numThreads=threads)
    dt = max(time.perf_counter() - t, 1e-6)
    sample = int(min(n, max(cal, cal * target_s / dt)))
    t = time.perf_counter()
    O.ref_lasso(X[:, :sample], D, lambda1=LAMBDA, numThreads=threads)
    dt = time.perf_counter() - t
    return sample / dt, sample


def omp_threads(requested: int) -> int:
    # init_omp (linalg/misc.h:288-300): -1 -> min(64, number of processors)
    return min(64, os.cpu_count() or 1) if requested == -1 else requested


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    if O.build_ref() is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built"}))
        return
    X, D = workload(args.n, 0)
    X, D = X.astype(np.float32), D.astype(np.float32)
    threads = omp_threads(-1)
    # size the per-step sample to ~`args.ref_step_s` seconds of CPU work
    _, sample = cpu_reference_rate(X, D, args.ref_step_s, -1)
    Xs = np.asfortranarray(X[:, :sample])
    for _ in range(args.warmup):
        O.ref_lasso(Xs[:, : min(sample, 2000)], D, lambda1=LAMBDA, numThreads=-1)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        O.ref_lasso(Xs, D, lambda1=LAMBDA, numThreads=-1)
        times.append(time.perf_counter() - t)
    value = sample * len(times) / sum(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": dict(config_dict(args.n, args.gpus, args.precision),
                       precision="reference float build on the host cores"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{sample} of the {args.n} signals per step, "
                                   f"reference lasso2 float build, OpenMP {threads} threads, "
                                   "OPENBLAS_NUM_THREADS=1"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args) -> None:
    import torch
    import spams_b200

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    prec = spams_b200.SC_PREC_BF16X3 if args.precision == "bf16x3" else spams_b200.SC_PREC_FP32

    X, D = workload(args.n, rank)
    Xf = X.astype(np.float32)
    Df = D.astype(np.float32)
    n = Xf.shape[1]
    Xt = torch.from_numpy(np.ascontiguousarray(Xf.T)).to(dev).t()
    Dt = torch.from_numpy(np.ascontiguousarray(Df.T)).to(dev).t()
    cap = n * min(M, K)
    outs = (torch.empty(n + 1, dtype=torch.int64, device=dev),
            torch.empty(cap, dtype=torch.int32, device=dev),
            torch.empty(cap, dtype=torch.float32, device=dev))
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > L2
    stream = torch.cuda.current_stream(dev)

    def step(profile=False):
        return spams_b200.lasso_device(Xt, Dt, LAMBDA, stream=stream, precision=prec, kernel=KERNEL,
                                       out=outs, sync=False, profile=profile)

    def barrier():
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(args.warmup):
        step()
    barrier()

    # ---- timed region A: throughput with inputs resident in HBM
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    launches = 0
    with Clocks(torch.cuda.current_device()) as clk:
        barrier()
        for i in range(args.steps):
            flush.fill_(float(i))
            evs[i][0].record(stream)
            step()
            evs[i][1].record(stream)
            launches += spams_b200.last_profile()["launches"]
        barrier()
    total_ms = sum(a.elapsed_time(b) for a, b in evs)
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    nnz = int(outs[0][n].item())

    # ---- the plain FP32 path on the same inputs, same timing rules
    fp32_ms = None
    if prec != spams_b200.SC_PREC_FP32:
        def step32():
            return spams_b200.lasso_device(Xt, Dt, LAMBDA, stream=stream, kernel=KERNEL,
                                           precision=spams_b200.SC_PREC_FP32, out=outs,
                                           sync=False)
        for _ in range(2):
            step32()
        barrier()
        evs32 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                 for _ in range(args.steps)]
        for i in range(args.steps):
            flush.fill_(float(i))
            evs32[i][0].record(stream)
            step32()
            evs32[i][1].record(stream)
        barrier()
        t = torch.tensor([sum(a.elapsed_time(b) for a, b in evs32)], dtype=torch.float64,
                         device=dev)
        if dist is not None:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        fp32_ms = float(t.item())

    # ---- timed region B: per-stage device times of the same call
    stage = {"ms_gram": 0.0, "ms_norms": 0.0, "ms_corr": 0.0, "ms_code": 0.0, "ms_refine": 0.0,
             "ms_csc": 0.0, "steps": 0, "overflowed": 0}
    for i in range(args.steps):
        flush.fill_(float(i))
        step(profile=True)
        p = spams_b200.last_profile()
        for k in stage:
            stage[k] += p[k]
    for k in stage:
        stage[k] /= args.steps

    # ---- end to end through the host entry point (pinned host buffers)
    Xh = torch.empty((n, M), dtype=torch.float32, pin_memory=True)
    Xh.numpy()[:] = Xf.T
    Xnp = Xh.numpy().T  # Fortran-ordered view, pinned
    # warm-up in the steady state of a caller that keeps each result until the
    # next one arrives (two results alive: the result pool holds two sets of
    # page-locked blocks from then on)
    a = None
    for _ in range(max(2, args.warmup // 2)):
        a = spams_b200.lasso(Xnp, Df, lambda1=LAMBDA, precision=prec, kernel=KERNEL)
    barrier()
    e2e_t = []
    e2e_steps = max(1, min(args.steps, 10))
    for _ in range(e2e_steps):
        t0 = time.perf_counter()
        a = spams_b200.lasso(Xnp, Df, lambda1=LAMBDA, precision=prec, kernel=KERNEL)
        e2e_t.append(time.perf_counter() - t0)
    e2e_s = torch.tensor([sum(e2e_t) / len(e2e_t)], dtype=torch.float64, device=dev)
    if dist is not None:
        dist.all_reduce(e2e_s, op=dist.ReduceOp.MAX)
    e2e_s = float(e2e_s.item())
    h2d = Xf.nbytes + Df.nbytes
    d2h = (n + 1) * 8 + a.nnz * 8

    # ---- CPU baseline (rank 0, one GPU only): all host threads, and one
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            rate, sample = cpu_reference_rate(Xf, Df, args.cpu_seconds, -1)
            rate1, sample1 = cpu_reference_rate(Xf, Df, max(1.0, args.cpu_seconds / 3), 1)
            thr = omp_threads(-1)
            cpu = {"value": rate, "unit": UNIT, "cores": thr, "kind": "reference",
                   "sample": f"first {sample} signals of the workload, reference lasso2 "
                             f"(T=float), OpenMP {thr} threads, OPENBLAS_NUM_THREADS=1",
                   "single_thread_value": rate1,
                   "single_thread_sample": f"first {sample1} signals, numThreads=1"}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {e}"}

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    peaks = measured_peaks()
    value = world * n * args.steps / (total_ms / 1e3)
    code_ms = stage["ms_code"]
    # algorithmic bytes of the LARS kernel per launch: per signal the K-float
    # correlation column, one K-float Gram column per homotopy step, and the
    # (index, value) pair of every output coefficient
    alg_bytes = 4 * K * n + 4 * K * stage["steps"] + 8 * nnz
    achieved = alg_bytes / (code_ms / 1e3) / 1e9 if code_ms > 0 else None
    traffic = profiled_traffic()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": config_dict(n, world, args.precision),
        "e2e": {"value": world * n / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "roofline": {"kernel": "lars_kernel", "bound": "hbm", "achieved": achieved,
                     "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": (achieved / peaks["hbm_gbs"]) if achieved else None,
                     "traffic": traffic, "peak_source": peaks["source"],
                     "algorithmic_bytes_per_launch": alg_bytes, "kernel_ms": code_ms},
        "stages_ms": {k: stage[k] for k in ("ms_gram", "ms_norms", "ms_corr", "ms_code",
                                            "ms_refine", "ms_csc")},
        "corr_roofline": (corr_roofline(M, K, K, n, stage["ms_corr"], peaks)
                          if args.precision == "bf16x3" else None),
        "fp32_value": (world * n * args.steps / (fp32_ms / 1e3)) if fp32_ms else value,
        "homotopy_steps_per_signal": stage["steps"] / n,
        "nnz_per_signal": nnz / n,
        "overflowed_signals": stage["overflowed"],
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
    }
    if world == 1 and not args.no_sub_workloads:
        # the other benchmarked configurations, bounded to a few minutes in all
        sub_cpu = min(args.cpu_seconds, 5.0)
        line["uneven_omp"] = uneven_omp_result(args.uneven_n, 5, 3, args.precision, sub_cpu,
                                               args.no_cpu_baseline)
        line["dictlearn"] = dictlearn_result(2000, 3, args.precision, sub_cpu,
                                             args.no_cpu_baseline)
        line["serve"] = serve_result(2000.0, 5.0, args.slots, args.precision, (500.0, 1000.0))
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# batched uneven OMP (D 512 x 2048, X 512 x 1e6)

UO_M, UO_K = 512, 2048
UO_METRIC = ("coded signals/s (batched uneven OMP, D 512x2048, s~U{1..64}, L=s+4, "
             "eps=0.5||noise||^2)")


def uneven_omp_result(n: int, steps: int, warmup: int, precision: str, cpu_seconds: float,
                      no_cpu: bool = False) -> dict:
    """The batched uneven OMP workload on n device-drawn signals."""
    import torch
    import spams_b200
    from spams_b200 import workloads as W
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    prec = spams_b200.SC_PREC_BF16X3 if precision == "bf16x3" else spams_b200.SC_PREC_FP32
    X, D, Lv, eps = W.config_uneven_omp_device(n=n, seed=0, m=UO_M, K=UO_K, device=dev)
    Lmax = int(Lv.max().item())
    cap = n * Lmax
    outs = (torch.empty(n + 1, dtype=torch.int64, device=dev),
            torch.empty(cap, dtype=torch.int32, device=dev),
            torch.empty(cap, dtype=torch.float32, device=dev))
    stream = torch.cuda.current_stream(dev)

    def step(profile=False, p=prec, s=None):
        return spams_b200.omp_device(X, D, L=Lmax, L_vec=Lv, eps_vec=eps,
                                     stream=s if s is not None else stream, precision=p,
                                     out=outs, sync=False, profile=profile)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    # the whole call (correlations, longest-first order, coding, overflow
    # pass, CSC) captured once as a CUDA graph and replayed per batch
    side = torch.cuda.Stream(dev)
    side.wait_stream(stream)
    with torch.cuda.stream(side):
        step(s=side)
    stream.wait_stream(side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        step(s=torch.cuda.current_stream(dev))
    torch.cuda.synchronize()
    step()
    launches_per_call = spams_b200.last_profile()["launches"]
    # inputs (X and the correlations of a pass) exceed L2
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(steps)]
    with Clocks(0) as clk:
        torch.cuda.synchronize()
        for i in range(steps):
            evs[i][0].record(stream)
            graph.replay()
            evs[i][1].record(stream)
        torch.cuda.synchronize()
    launches = launches_per_call * steps
    total_ms = sum(a.elapsed_time(b) for a, b in evs)
    nnz = int(outs[0][n].item())
    fp32_ms = None
    if prec != spams_b200.SC_PREC_FP32:
        step(p=spams_b200.SC_PREC_FP32)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step(p=spams_b200.SC_PREC_FP32)
        e1.record(stream)
        torch.cuda.synchronize()
        fp32_ms = e0.elapsed_time(e1)
    step(profile=True)
    prof = spams_b200.last_profile()
    # end to end: host arrays (pinned) in, CSC on the host out
    Xh = torch.empty((n, UO_M), dtype=torch.float32, pin_memory=True)
    Xh.copy_(X.t())
    Xnp = Xh.numpy().T
    Dnp = np.asfortranarray(D.cpu().numpy())
    Lnp, Enp = Lv.cpu().numpy(), eps.cpu().numpy()
    a = None
    for _ in range(2):  # two results alive, as in the timed loop
        a = spams_b200.omp(Xnp, Dnp, L=Lnp, eps=Enp, precision=prec)
    e2e_t = []
    for _ in range(max(1, min(steps, 3))):
        t0 = time.perf_counter()
        a = spams_b200.omp(Xnp, Dnp, L=Lnp, eps=Enp, precision=prec)
        e2e_t.append(time.perf_counter() - t0)
    e2e_s = sum(e2e_t) / len(e2e_t)
    cpu = None
    if not no_cpu:
        try:
            from oracle import oracle as O
            O.build_ref()
            cal = 500
            t0 = time.perf_counter()
            O.ref_omp(Xnp[:, :cal], Dnp, L=Lnp[:cal], eps=Enp[:cal], numThreads=-1)
            dt = max(time.perf_counter() - t0, 1e-6)
            sample = int(min(n, max(cal, cal * cpu_seconds / dt)))
            t0 = time.perf_counter()
            O.ref_omp(np.asfortranarray(Xnp[:, :sample]), Dnp, L=Lnp[:sample], eps=Enp[:sample],
                      numThreads=-1)
            rate = sample / (time.perf_counter() - t0)
            thr = omp_threads(-1)
            cpu = {"value": rate, "unit": UNIT, "cores": thr, "kind": "reference",
                   "sample": f"first {sample} signals, reference omp (T=float), OpenMP {thr} "
                             "threads, OPENBLAS_NUM_THREADS=1"}
        except Exception as e:
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {e}"}
    peaks = measured_peaks()
    code_ms = prof["ms_code"]
    # per signal: the K-float correlation column, one K-float Gram column per
    # selected atom, the (index, value) pair of each coefficient
    alg_bytes = 4 * UO_K * n + 4 * UO_K * prof["steps"] + 8 * nnz
    achieved = alg_bytes / (code_ms / 1e3) / 1e9 if code_ms > 0 else None
    kname = "omp_cta_kernel" if prof["kernel"] == spams_b200.SC_KERNEL_CTA else "omp_kernel"
    value = n * steps / (total_ms / 1e3)
    return {
        "metric": UO_METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": steps,
        "warmup": warmup, "ms_per_step": total_ms / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded, drawn on the device)",
        "config": {"workload": f"uneven_omp_D{UO_M}x{UO_K}_n{n}_s1-64_noise0.02",
                   "m": UO_M, "K": UO_K, "n": n, "precision": precision,
                   "between_steps": "inputs larger than L2 (X and the correlations of a pass)",
                   "launch": "one CUDA graph replay per batch (the whole call captured)",
                   "parallelism": "one GPU"},
        "e2e": {"value": n / e2e_s, "unit": UNIT, "h2d_bytes_per_step": Xnp.nbytes + Dnp.nbytes
                + Lnp.nbytes + Enp.nbytes, "d2h_bytes_per_step": (n + 1) * 8 + a.nnz * 8},
        "gpu_launches": launches,
        "roofline": {"kernel": kname, "bound": "hbm", "achieved": achieved,
                     "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": (achieved / peaks["hbm_gbs"]) if achieved else None,
                     "traffic": None, "peak_source": peaks["source"],
                     "algorithmic_bytes_per_launch": alg_bytes, "kernel_ms": code_ms,
                     "active_set_capacity": prof["lcap"]},
        "stages_ms": {k: prof[k] for k in ("ms_gram", "ms_norms", "ms_corr", "ms_code",
                                           "ms_refine", "ms_csc")},
        "corr_roofline": (corr_roofline(UO_M, UO_K, UO_K, n, prof["ms_corr"], peaks, terms=6)
                          if precision == "bf16x3" else None),
        "fp32_value": (n * steps / (fp32_ms / 1e3)) if fp32_ms else value,
        "omp_steps_per_signal": prof["steps"] / n, "nnz_per_signal": nnz / n,
        "overflowed_signals": prof["overflowed"],
        "clocks": clk.summary(), "cpu_baseline": cpu,
    }


def run_uneven_omp(args) -> None:
    print(json.dumps(uneven_omp_result(args.n or 1000000, args.steps, args.warmup, args.precision,
                                       args.cpu_seconds, args.no_cpu_baseline)), flush=True)


# ---------------------------------------------------------------------------
# serving stream

SERVE_METRIC = ("p99 request latency (serving stream: Poisson arrivals over 8 resident "
                "dictionaries, n log-uniform 1..5e4, OMP L~U{4..32} or Lasso lambda1~U[0.05,0.3])")


def _serve_requests(pools, rate, duration, seed, prec):
    import spams_b200
    rng = np.random.Generator(np.random.PCG64(seed))
    count = max(1, int(rng.poisson(rate * duration)))
    arrival = np.sort(rng.random(count) * duration)
    dsel = rng.integers(0, len(pools), size=count)
    pool = pools[0].shape[1]
    n = np.maximum(1, np.minimum(pool, np.floor(np.exp(rng.random(count) * np.log(50001)))
                                 .astype(np.int64)))
    off = (rng.random(count) * (pool - n + 1)).astype(np.int64)
    algo = rng.integers(0, 2, size=count)
    L = rng.integers(4, 33, size=count)
    lam = 0.05 + 0.25 * rng.random(count)
    recs = []
    for k in range(count):
        Xk = pools[dsel[k]][:, off[k]:off[k] + n[k]]
        if algo[k] == 0:
            recs.append(spams_b200.request(int(dsel[k]), Xk, "omp", L=int(L[k]), precision=prec,
                                           discard=True))
        else:
            recs.append(spams_b200.request(int(dsel[k]), Xk, "lasso", lambda1=float(lam[k]),
                                           precision=prec, discard=True))
    return recs, arrival, int(n.sum())


def serve_result(rate: float, duration: float, slots: int, precision: str,
                 sweep_rates=(250.0, 500.0, 1000.0)) -> dict:
    """The serving stream at `rate` requests/s (then each lower rate of
    sweep_rates), p50 / p99 latency from arrival to the result on the host."""
    import torch
    import spams_b200
    from spams_b200 import workloads as W
    torch.cuda.set_device(0)
    prec = spams_b200.SC_PREC_BF16X3 if precision == "bf16x3" else spams_b200.SC_PREC_FP32
    dicts, pools, _ = W.config_serving(rate=1.0, duration_s=1.0, seed=0)
    pinned = []
    for P in pools:  # request signals live in pinned host memory
        h = torch.empty((P.shape[1], P.shape[0]), dtype=torch.float32, pin_memory=True)
        h.numpy()[:] = P.T
        pinned.append(h.numpy().T)
    with spams_b200.Server(hbm_budget=150e9, slots=slots) as srv:
        for i, D in enumerate(dicts):
            srv.add_dictionary(i, D)
        # warm-up: one second of the stream (kernels loaded, shapes tuned), then
        # a burst at four times the rate, whose queue merges batches up to the
        # server's largest, so that every slot's workspaces reach the sizes a
        # backlog in the measured stream would need (growing a multi-GB
        # workspace mid-stream stalls every slot for up to a second)
        recs, arr, _ = _serve_requests(pinned, rate, 1.0, 99, prec)
        srv.replay(recs, arr)
        recs, arr, _ = _serve_requests(pinned, 4 * rate, 1.0, 98, prec)
        srv.replay(recs, arr)
        sweep = []
        rates = [rate] + [r for r in sweep_rates if r < rate]
        clk_summary = None
        for r in rates:
            recs, arr, offered = _serve_requests(pinned, r, duration, int(r), prec)
            srv.stats(reset=True)
            with Clocks(0) as clk:
                t0 = time.perf_counter()
                srv.replay(recs, arr)
                wall = time.perf_counter() - t0
            st = srv.stats(reset=True)
            if clk_summary is None:
                clk_summary = clk.summary()
            sweep.append({"rate_req_s": r, "requests": len(recs),
                          "offered_signals_s": offered / duration,
                          "served_signals_s": st["signals"] / wall, "wall_s": wall,
                          "p50_ms": st["lat_p50_ms"], "p99_ms": st["lat_p99_ms"],
                          "mean_ms": st["lat_mean_ms"], "max_ms": st["lat_max_ms"],
                          "requests_per_launch": st["mean_batch_requests"],
                          "rejected": st["rejected"], "gpu_busy_s": st["busy_s"],
                          "peak_device_bytes": st["peak_device_bytes"]})
    out = sweep[0]
    return {
        "metric": SERVE_METRIC, "value": out["p99_ms"], "unit": "ms", "n_gpus": 1,
        "steps": 1, "warmup": 2, "ms_per_step": out["wall_s"] * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded; signals drawn once into per-dictionary pools)",
        "config": {"workload": f"serving_poisson{rate:g}rps_{duration:g}s",
                   "dictionaries": [list(t) for t in W.SERVING_DICTS], "slots": slots,
                   "hbm_budget_bytes": 150e9, "precision": precision,
                   "between_steps": "inputs larger than L2 (pools of 0.39 GB)",
                   "parallelism": "one GPU"},
        "rate_req_s": rate, "p50_ms": out["p50_ms"], "p99_ms": out["p99_ms"],
        "served_signals_s": out["served_signals_s"],
        "offered_signals_s": out["offered_signals_s"],
        "e2e": {"value": out["p99_ms"], "unit": "ms", "h2d_bytes_per_step": None,
                "d2h_bytes_per_step": None},
        "sweep": sweep, "clocks": clk_summary,
    }


def run_serve(args) -> None:
    print(json.dumps(serve_result(args.rate, args.duration, args.slots, args.precision,
                                  () if args.no_sweep else (250.0, 500.0, 1000.0))), flush=True)


# ---------------------------------------------------------------------------
# online dictionary-learning inner loop

DL_M, DL_K, DL_BATCH, DL_LAMBDA = 144, 1024, 1024, 0.1
DL_METRIC = ("minibatches/s (online dictionary-learning step: 1024 signals of 12x12 smooth "
             "patches, D 144x1024 perturbed and renormalised per minibatch, Gram recomputed, "
             "Lasso lambda1=0.1, A/B accumulations)")


def dictlearn_result(nb: int, warmup: int, precision: str, cpu_seconds: float,
                     no_cpu: bool = False) -> dict:
    """nb minibatches of the online dictionary-learning step, one CUDA-graph
    replay each; e2e runs the same nb minibatches through the eager API with
    each minibatch copied in from pinned host memory."""
    import torch
    import spams_b200
    from spams_b200 import workloads as W
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    prec = spams_b200.SC_PREC_BF16X3 if precision == "bf16x3" else spams_b200.SC_PREC_FP32
    rng = np.random.Generator(np.random.PCG64(0))
    nwin = 195
    pool = nwin * DL_BATCH  # 199680 signals: minibatch i is window i mod 195 of the permutation
    Xnp = W.smooth_patches(pool, rng, side=12).astype(np.float32)
    D0 = Xnp[:, rng.choice(pool, DL_K, replace=False)]  # random signals, as train() starts
    D0 = np.asfortranarray(D0 / np.linalg.norm(D0, axis=0, keepdims=True))
    perm_np = rng.permutation(pool).astype(np.int32)
    perm = torch.from_numpy(perm_np).to(dev)
    Xd = torch.from_numpy(np.ascontiguousarray(Xnp.T)).to(dev).t()
    U = torch.from_numpy(rng.standard_normal((DL_M, nb + 1)).astype(np.float32)).to(dev)
    V = torch.from_numpy(rng.standard_normal((DL_K, nb + 1)).astype(np.float32)).to(dev)

    def fresh():
        Dd = torch.from_numpy(np.ascontiguousarray(D0.T)).to(dev).t()
        A = torch.zeros((DL_K, DL_K), device=dev).t()
        B = torch.zeros((DL_K, DL_M), device=dev).t()
        it = torch.zeros(1, dtype=torch.int64, device=dev)
        return Dd, A, B, it

    step = spams_b200.MinibatchStep(DL_M, DL_K, DL_BATCH, lambda1=DL_LAMBDA, precision=prec)
    Dd, A, B, it = fresh()

    def perturb(ui, vi):
        # the dictionary changes every minibatch: rank-1 perturbation, then
        # unit columns again
        Dd.add_(0.01 * torch.outer(ui, vi))
        Dd.div_(Dd.norm(dim=0, keepdim=True))

    def body():
        # the minibatch's column of U and V is picked by the device counter
        perturb(U.index_select(1, it).squeeze(1), V.index_select(1, it).squeeze(1))
        step(Dd, Xd, it, perm=perm, A=A, B=B, beta=1.0, gamma=1.0 / DL_BATCH)

    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(warmup):
            body()
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        body()
    # ---- timed: nb minibatches, one graph replay each
    Dd.copy_(torch.from_numpy(np.ascontiguousarray(D0.T)).to(dev).t())
    A.zero_()
    B.zero_()
    it.zero_()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(0) as clk:
        e0.record()
        for _ in range(nb):
            graph.replay()
        e1.record()
        torch.cuda.synchronize()
    graph_ms = e0.elapsed_time(e1)
    done = int(it.item())
    # ---- the same loop without the graph (launch-bound comparison)
    ne = min(nb, 200)
    Dd, A, B, it = fresh()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(ne):
        body()
    e1.record()
    torch.cuda.synchronize()
    eager_ms = e0.elapsed_time(e1)
    # ---- stage times and launches of one eager step
    step.profile(True)
    body()
    torch.cuda.synchronize()
    prof = spams_b200.last_profile()
    step.profile(False)
    cp, rows, vals = step.codes()
    nnz = int(cp[-1].item())
    # ---- end to end: the same nb minibatches, each copied in from pinned
    # host memory (minibatch i = window i mod 195 of the permuted pool, the
    # columns the graph loop reads), D perturbed and renormalised, coded and
    # accumulated, its code count read back
    Xh = torch.empty((pool, DL_M), dtype=torch.float32, pin_memory=True)
    Xh.numpy()[:] = Xnp[:, perm_np].T
    Xbuf = torch.empty((DL_BATCH, DL_M), device=dev).t()
    it1 = torch.zeros(1, dtype=torch.int64, device=dev)
    Dd, A, B, it = fresh()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(nb):
        w = i % nwin
        Xbuf.copy_(Xh[w * DL_BATCH:(w + 1) * DL_BATCH].t(), non_blocking=True)
        perturb(U[:, i], V[:, i])
        step(Dd, Xbuf, it1, A=A, B=B, beta=1.0, gamma=1.0 / DL_BATCH)
        int(step.codes()[0][-1].item())
    e2e_s = (time.perf_counter() - t0) / nb
    cpu = None
    if not no_cpu:
        try:
            from oracle import oracle as O
            O.build_ref()
            Ah = np.zeros((DL_K, DL_K), np.float32, order="F")
            Bh = np.zeros((DL_M, DL_K), np.float32, order="F")
            reps, t0 = 0, time.perf_counter()
            while time.perf_counter() - t0 < cpu_seconds and reps < 200:
                O.ref_dl_minibatch(D0, Xnp, perm_np, reps, DL_BATCH, DL_LAMBDA, Ah, Bh,
                                   1.0, 1.0 / DL_BATCH)
                reps += 1
            rate = reps / (time.perf_counter() - t0)
            thr = omp_threads(-1)
            cpu = {"value": rate, "unit": "minibatches/s", "cores": thr, "kind": "reference",
                   "sample": f"{reps} minibatches of {DL_BATCH} signals: the reference's own "
                             "Gram (XtX + ridge), multTrans, coreLARS2, sort and rank-1 A/B "
                             f"accumulations (dictLearn/dicts.h:526-603, T=float), OpenMP "
                             f"{thr} threads; D held fixed"}
        except Exception as e:
            cpu = {"value": None, "unit": "minibatches/s", "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {e}"}
    peaks = measured_peaks()
    code_ms = prof["ms_code"]
    alg_bytes = 4 * DL_K * DL_BATCH + 4 * DL_K * prof["steps"] + 8 * nnz
    achieved = alg_bytes / (code_ms / 1e3) / 1e9 if code_ms > 0 else None
    kname = "lars_cta_kernel" if prof["kernel"] == spams_b200.SC_KERNEL_CTA else "lars_kernel"
    value = done / (graph_ms / 1e3)
    return {
        "metric": DL_METRIC, "value": value, "unit": "minibatches/s", "n_gpus": 1,
        "steps": done, "warmup": warmup, "ms_per_step": graph_ms / done,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": f"synthetic (seeded smooth 12x12 patches, pool of {pool})",
        "config": {"workload": f"dictlearn_m{DL_M}_K{DL_K}_batch{DL_BATCH}_lambda{DL_LAMBDA}",
                   "minibatches": done, "precision": precision,
                   "between_steps": "none (a minibatch's inputs are 0.6 MB; the loop is the unit)",
                   "launch": "one CUDA graph replay per minibatch", "parallelism": "one GPU"},
        "eager_value": ne / (eager_ms / 1e3),
        "e2e": {"value": 1.0 / e2e_s, "unit": "minibatches/s",
                "h2d_bytes_per_step": DL_BATCH * DL_M * 4, "d2h_bytes_per_step": 8},
        "gpu_launches": prof["launches"] * done,
        "roofline": {"kernel": kname, "bound": "hbm", "achieved": achieved,
                     "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": (achieved / peaks["hbm_gbs"]) if achieved else None,
                     "traffic": None, "peak_source": peaks["source"],
                     "algorithmic_bytes_per_launch": alg_bytes, "kernel_ms": code_ms,
                     "active_set_capacity": prof["lcap"]},
        "stages_ms": {k: prof[k] for k in ("ms_norms", "ms_corr", "ms_code", "ms_csc")},
        "homotopy_steps_per_signal": prof["steps"] / DL_BATCH, "nnz_per_signal": nnz / DL_BATCH,
        "clocks": clk.summary(), "cpu_baseline": cpu,
    }


def run_dictlearn(args) -> None:
    print(json.dumps(dictlearn_result(args.n or 2000, args.warmup, args.precision,
                                      args.cpu_seconds, args.no_cpu_baseline)), flush=True)


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["lasso", "uneven_omp", "serve", "dictlearn"],
                    default="lasso")
    ap.add_argument("--n", type=int, default=None, help="signals per GPU")
    ap.add_argument("--precision", choices=["fp32", "bf16x3"], default="bf16x3")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--ref-step-s", type=float, default=5.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--rate", type=float, default=2000.0, help="serve: requests/s")
    ap.add_argument("--duration", type=float, default=5.0, help="serve: seconds of arrivals")
    ap.add_argument("--slots", type=int, default=3, help="serve: concurrent launches")
    ap.add_argument("--no-sweep", action="store_true", help="serve: skip the lower rates")
    ap.add_argument("--no-sub-workloads", action="store_true",
                    help="lasso: leave the uneven-OMP, dictionary-learning and serving "
                         "sub-objects out of the line")
    ap.add_argument("--uneven-n", type=int, default=200000,
                    help="signals of the uneven-OMP sub-workload of the default line")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)  # at least three untimed steps
    if args.workload == "uneven_omp":
        if args.impl == "ours":
            run_uneven_omp(args)
        else:
            print(json.dumps({"impl": "reference", "metric": UO_METRIC,
                              "unavailable": "reference arm is timed on the lasso workload"}))
        return 0
    if args.workload == "serve":
        if args.impl == "ours":
            run_serve(args)
        else:
            print(json.dumps({"impl": "reference", "metric": SERVE_METRIC,
                              "unavailable": "the reference has no serving loop"}))
        return 0
    if args.workload == "dictlearn":
        if args.impl == "ours":
            run_dictlearn(args)
        else:
            print(json.dumps({"impl": "reference", "metric": DL_METRIC,
                              "unavailable": "reference arm is timed on the lasso workload"}))
        return 0
    args.n = args.n or 100000
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)
    return 0


if __name__ == "__main__":
    sys.exit(main())
