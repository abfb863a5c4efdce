#!/usr/bin/env python
"""Coded signals/s of LARS-Lasso on B200 (one JSON line on stdout).

Workload (per GPU): D 256 x 512 with unit-norm N(0,1) columns; X 256 x 100000
whose columns are D a + 0.01 N(0,1) with 12 uniformly placed N(0,1)
non-zeros; lasso mode 2 (PENALTY), lambda1 = 0.15, float32.  A step codes
the whole batch: Gram, ||x||^2, D^T X, the LARS homotopy of every signal and
the CSC assembly.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is measured through the device entry point with inputs resident in
HBM (CUDA events on the call's stream, an L2-flushing write between steps);
`e2e` through the host entry point with pinned host buffers, copies inside
the timed region.  With N > 1 (torchrun) every rank codes its own batch with
the same dictionary (weak scaling, no collective on the data path); rank 0
prints the aggregate.  `--impl reference` times the SPAMS reference's own CPU
code (oracle/_ref) on the host cores instead.
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
            "precision": precision, "between_steps": "L2 flush (256 MiB write)",
            "parallelism": f"column shards x{ngpu}, no data-path collective"}


def measured_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    except Exception:
        return {"hbm_gbs": 6650.0, "source": "fallback"}


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
                 "--format=csv,noheader,nounits", "-lms", "100"],
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
        "config": config_dict(args.n, args.gpus, "fp32"),
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
        return spams_b200.lasso_device(Xt, Dt, LAMBDA, stream=stream, precision=prec,
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
    for _ in range(max(1, args.warmup // 2)):
        spams_b200.lasso(Xnp, Df, lambda1=LAMBDA, precision=prec)
    barrier()
    e2e_t = []
    e2e_steps = max(1, min(args.steps, 10))
    for _ in range(e2e_steps):
        t0 = time.perf_counter()
        a = spams_b200.lasso(Xnp, Df, lambda1=LAMBDA, precision=prec)
        e2e_t.append(time.perf_counter() - t0)
    e2e_s = torch.tensor([sum(e2e_t) / len(e2e_t)], dtype=torch.float64, device=dev)
    if dist is not None:
        dist.all_reduce(e2e_s, op=dist.ReduceOp.MAX)
    e2e_s = float(e2e_s.item())
    h2d = Xf.nbytes + Df.nbytes
    d2h = (n + 1) * 8 + a.nnz * 8

    # ---- CPU baseline (rank 0, one GPU only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            rate, sample = cpu_reference_rate(Xf, Df, args.cpu_seconds, -1)
            thr = omp_threads(-1)
            cpu = {"value": rate, "unit": UNIT, "cores": thr, "kind": "reference",
                   "sample": f"first {sample} signals of the workload, reference lasso2 "
                             f"(T=float), OpenMP {thr} threads, OPENBLAS_NUM_THREADS=1"}
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
        "homotopy_steps_per_signal": stage["steps"] / n,
        "nnz_per_signal": nnz / n,
        "overflowed_signals": stage["overflowed"],
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=100000, help="signals per GPU")
    ap.add_argument("--precision", choices=["fp32", "bf16x3"], default="fp32")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--ref-step-s", type=float, default=5.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)  # at least three untimed steps
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)
    return 0


if __name__ == "__main__":
    sys.exit(main())
