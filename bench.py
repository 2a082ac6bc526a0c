#!/usr/bin/env python
"""Throughput benchmark of the periodic DMK evaluate path on B200.

Workload (one step = one evaluate of one charge vector on a resident tree):
  uniform cube, L = 1, N = 10^6 positions uniform in [0,1)^3 (seed 1), charges
  uniform in [-1,1] minus their mean, n_digits = 6, n_per_leaf = 300, nz = 4,
  plain FP64 path, 1 RHS.  Synthetic data; the tree is built once (untimed),
  as in the reference's build-once / evaluate-many contract.

Metric: Mpts*RHS/s = N * RHS / t_evaluate / 1e6 (whole job: summed over ranks).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

For --gpus N > 1 launch one process per GPU with torch.distributed.run; the
path does not shard (one system per evaluate), so every rank runs an
independent replica and value is the sum over ranks ("replicas only").
--impl reference times the CPU restatement of the reference evaluate (the
oracle) on the host cores on a bounded sample of the same workload, rank 0 only.
"""
import argparse
import csv
import io
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mpts*RHS/s per B200 at 1e-6 rel L2: mixed-prec batched vs plain FP64 GPU"


def make_system(n, seed=1, scale=1.0):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.0, 1.0, (n, 3)) * scale
    q = rng.uniform(-1.0, 1.0, n)
    q -= q.mean()
    return np.eye(3) * scale, pos, q


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc is not None:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                self.out = ""

    def summary(self):
        rows = [r for r in csv.reader(io.StringIO(getattr(self, "out", ""))) if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_baseline(n_target, steps, threads):
    """Oracle (CPU restatement of the reference evaluate) on a bounded sample:
    a cell scaled so the sample keeps the workload's point density (10^6 per
    unit volume), hence the same leaves, expansion orders and far-field modes
    per point.  Returns (Mpts/s, sample description, seconds per step)."""
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    import oracle
    n = 100000
    scale = (n / float(n_target)) ** (1.0 / 3.0)
    cell, pos, q = make_system(n, seed=2, scale=scale)
    oracle.evaluate(cell, pos, q, 6, 300, 4, with_far=True, fast_far=True)  # warm-up
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        oracle.evaluate(cell, pos, q, 6, 300, 4, with_far=True, fast_far=True)
        ts.append(time.perf_counter() - t0)
    t = statistics.median(ts)
    desc = ("CPU oracle (FP64 restatement of the reference evaluate: upward/plane-wave/near/self stages + "
            "CPU NUFFT far field), N=%d uniform in a cube of side %.4f (same density as the N=%d workload), "
            "6 digits, npl 300, nz 4, %d OpenMP threads, median of %d" % (n, scale, n_target, threads, steps))
    return n / t / 1e6, desc, t


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    for _ in range(max(0, args.warmup - 1)):
        pass
    v, desc, t = cpu_baseline(args.n, max(1, args.steps), threads)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mpts*RHS/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "uniform cube N=1e6, 6 digits, n_per_leaf 300, nz 4, 1 RHS (bounded sample)"},
            "cpu_baseline": {"value": v, "unit": "Mpts*RHS/s", "cores": threads, "kind": "port", "sample": desc},
            "e2e": {"value": v, "unit": "Mpts*RHS/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import periodicdmk_b200 as pd

    n = args.n
    cell, pos, q = make_system(n, seed=1)
    t_build = time.perf_counter()
    tree = pd.PeriodicDMKTree(cell, pos, n_digits=6, n_per_leaf=300, nz=4, precision="double")
    t_build = time.perf_counter() - t_build
    info = tree.info()
    dev = torch.device("cuda", local)
    q_d = torch.from_numpy(q).to(dev)
    pot_d = torch.empty(n, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2
    for _ in range(args.warmup):
        tree.evaluate_device(q_d.data_ptr(), pot_d.data_ptr())
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- device-resident throughput: per-step device time from the events the
    # library records on its launching stream; L2 flushed between steps.
    step_ms = []
    stages = []
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            tree.evaluate_device(q_d.data_ptr(), pot_d.data_ptr())
            st = tree.stage_times()
            stages.append(st)
            step_ms.append(st["total_ms"])
    torch.cuda.synchronize()
    barrier()
    t_dev = sum(step_ms) / 1e3
    if dist is not None:
        tt = torch.tensor([t_dev], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_dev = float(tt.item())
    ms_per_step = t_dev / args.steps * 1e3
    value = world * n / (t_dev / args.steps) / 1e6

    # ---- end to end through the public C ABI with host (pinned) buffers
    q_h = torch.from_numpy(q).pin_memory()
    pot_h = torch.empty(n, dtype=torch.float64).pin_memory()
    import ctypes
    D = ctypes.POINTER(ctypes.c_double)
    qp = ctypes.cast(q_h.data_ptr(), D)
    pp = ctypes.cast(pot_h.data_ptr(), D)
    lib = pd.library()
    e2e = []
    barrier()
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc = lib.pdmk_evaluate_double(tree._h, n, None, qp, pp)
        e2e.append(time.perf_counter() - t0)
        if rc != 0:
            raise RuntimeError("pdmk_evaluate_double failed: " + pd._last_error())
    barrier()
    t_e2e = sum(e2e)
    if dist is not None:
        tt = torch.tensor([t_e2e], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_e2e = float(tt.item())
    e2e_value = world * n / (t_e2e / args.steps) / 1e6
    assert np.allclose(pot_h.numpy(), pot_d.cpu().numpy(), rtol=1e-12, atol=1e-12)

    # ---- roofline of the dominant kernel (residual near field, FP64 CUDA cores)
    near_ms = statistics.median(s["near_ms"] for s in stages)
    flop_per_pair = 2 * int(stages[0]["near_ncoef"]) + 14
    near_flop = stages[0]["near_pairs_culled"] * flop_per_pair
    achieved = near_flop / (near_ms * 1e-3) / 1e12
    peak = pd.fma_peak_tflops(fp64=True)
    roofline = {"bound": "fp64", "kernel": "k_near (residual near field)", "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
                "peak_source": "measured FP64 FMA probe on this GPU (pdmk_fma_peak)",
                "algorithmic_flop_per_launch": near_flop,
                "stage_ms_median": {k: statistics.median(s[k] for s in stages)
                                    for k in ("dmk_ms", "near_ms", "nufft_ms", "finalize_ms", "total_ms")}}

    line = {"metric": METRIC, "value": value, "unit": "Mpts*RHS/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "uniform cube N=1e6 (seed 1), charges U[-1,1] minus mean, 6 digits, "
                                   "n_per_leaf 300, nz 4, 1 RHS, plain FP64 path",
                       "n_points": n, "rhs": 1, "n_digits": 6, "n_per_leaf": 300, "nz": 4,
                       "parallelism": "replicas x%d" % world, "l2": "flushed between steps (256 MB write)",
                       "tree": {k: info[k] for k in ("n_all", "n_boxes", "n_levels", "n_target_leaves", "p",
                                                     "n_pw", "device_bytes")},
                       "tree_build_s": t_build},
            "e2e": {"value": e2e_value, "unit": "Mpts*RHS/s", "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
                    "ms_per_step": t_e2e / args.steps * 1e3},
            "gpu_launches": info["launches_per_evaluate"] * args.steps,
            "roofline": roofline, "clocks": clk.summary()}
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, desc, _ = cpu_baseline(n, 3, threads)
        line["cpu_baseline"] = {"value": v, "unit": "Mpts*RHS/s", "cores": threads, "kind": "port", "sample": desc}
    if rank == 0:
        print(json.dumps(line), flush=True)
    tree.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=1000000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
