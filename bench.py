#!/usr/bin/env python
"""Throughput benchmark of the periodic DMK evaluate path on B200.

Workload (one step = one batched evaluate of 64 charge vectors on a resident tree):
  uniform cube, L = 1, N = 10^6 positions uniform in [0,1)^3 (seed 1), 64
  charge vectors uniform in [-1,1] minus their mean, n_digits = 6,
  n_per_leaf = 300, nz = 4, mixed-precision path.  The plain FP64 evaluate of
  one charge vector on the same tree is measured beside it.  Synthetic data;
  the trees are built once (untimed), as in the reference's build-once /
  evaluate-many contract.  Extra fragments of the same JSON line: the
  many-systems batch (--batch-systems) and the plain FP64 evaluate of a
  clustered triclinic system of 2e6 points at 9 and 12 digits
  (--clustered-digits, --clustered-n).

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


def batch_systems(nsys, seed):
    """Many-systems workload: triclinic cells (lengths U[0.8, 1.2], angles
    U[75, 105] degrees, a1 along x, a2 in the xy plane), N log-uniform in
    [1e3, 1e5], fractional-uniform points, +-1 neutral charges."""
    rng = np.random.default_rng(seed)
    cells, pos, qs = [], [], []
    for _ in range(nsys):
        n = int(round(np.exp(rng.uniform(np.log(1e3), np.log(1e5)))))
        n += n % 2
        L = rng.uniform(0.8, 1.2, 3)
        al, be, ga = np.radians(rng.uniform(75.0, 105.0, 3))
        cx = np.cos(be)
        cy = (np.cos(al) - np.cos(be) * np.cos(ga)) / np.sin(ga)
        cell = np.column_stack([[L[0], 0.0, 0.0], L[1] * np.array([np.cos(ga), np.sin(ga), 0.0]),
                                L[2] * np.array([cx, cy, np.sqrt(max(1.0 - cx * cx - cy * cy, 1e-12))])])
        q = np.ones(n)
        q[: n // 2] = -1.0
        rng.shuffle(q)
        cells.append(cell)
        pos.append(rng.uniform(0.0, 1.0, (n, 3)) @ cell.T)
        qs.append(q)
    return cells, pos, qs


def clustered_system(n, seed=3):
    """High-accuracy workload: triclinic cell with columns (1,0,0), (0.3,0.9,0),
    (0.2,0.25,0.85); half the points uniform in fractional coordinates, half
    from 64 isotropic Gaussian clusters (sigma 0.01 Cartesian, centres uniform
    in the cell, wrapped back into the cell); +-1 neutral charges."""
    rng = np.random.default_rng(seed)
    cell = np.array([[1.0, 0.3, 0.2], [0.0, 0.9, 0.25], [0.0, 0.0, 0.85]])  # columns = lattice vectors
    inv = np.linalg.inv(cell)
    nu = n // 2
    frac_u = rng.uniform(0.0, 1.0, (nu, 3))
    centres = rng.uniform(0.0, 1.0, (64, 3)) @ cell.T
    which = rng.integers(0, 64, n - nu)
    pts = centres[which] + rng.normal(0.0, 0.01, (n - nu, 3))
    frac_c = (pts @ inv.T) % 1.0
    pos = np.vstack([frac_u, frac_c]) @ cell.T
    q = np.ones(n)
    q[: n // 2] = -1.0
    rng.shuffle(q)
    return cell, pos, q


def run_clustered(pd, args, world, dev, flush, barrier, max_over_ranks):
    """Plain FP64 evaluate of the clustered triclinic workload at each digit
    count of --clustered-digits (device-resident charges, L2 flushed, CUDA-event
    stage times); the highest digit count is the accuracy reference."""
    import torch
    digits = [int(x) for x in args.clustered_digits.split(",") if x.strip()]
    n = args.clustered_n
    cell, pos, q = clustered_system(n)
    q_d = torch.from_numpy(q).to(dev)
    pot_d = torch.empty(n, dtype=torch.float64, device=dev)
    out = {"workload": "triclinic cell (1,0,0),(0.3,0.9,0),(0.2,0.25,0.85); N=%d, 50%% fractional-uniform, "
                       "50%% in 64 Gaussian clusters (sigma 0.01), +-1 charges; npl 300, nz 4; plain FP64 "
                       "evaluate, one charge vector" % n,
           "n_points": n, "digits": {}}
    pots = {}
    for nd in digits:
        t0 = time.perf_counter()
        tree = pd.PeriodicDMKTree(cell, pos, n_digits=nd, n_per_leaf=300, nz=4, precision="double")
        tb = time.perf_counter() - t0
        for _ in range(args.warmup):
            tree.evaluate_device(q_d.data_ptr(), pot_d.data_ptr())
        torch.cuda.synchronize()
        st = []
        barrier()
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            tree.evaluate_device(q_d.data_ptr(), pot_d.data_ptr())
            st.append(tree.stage_times())
        torch.cuda.synchronize()
        barrier()
        t = max_over_ranks(sum(x["total_ms"] for x in st) / 1e3) / args.steps
        info = tree.info()
        out["digits"][str(nd)] = {
            "ms_per_evaluate": t * 1e3, "value": world * n / t / 1e6, "unit": "Mpts/s",
            "stage_ms_median": {kk: statistics.median(x[kk] for x in st)
                                for kk in ("dmk_ms", "near_ms", "nufft_ms", "total_ms")},
            "device_bytes": info["device_bytes"], "tree_build_s": tb, "p": info["p"], "n_pw": info["n_pw"]}
        pots[nd] = pot_d.cpu().numpy()
        tree.close()
    if len(pots) > 1:
        ref = pots[max(pots)]
        out["rel_l2_vs_highest_digits"] = {str(nd): float(np.linalg.norm(v - ref) / np.linalg.norm(ref))
                                           for nd, v in pots.items() if nd != max(pots)}
    return out


def lpt_partition(costs, parts):
    """Greedy longest-processing-time assignment of items to parts."""
    loads = [0.0] * parts
    owner = [0] * len(costs)
    for i in sorted(range(len(costs)), key=lambda j: -costs[j]):
        r = min(range(parts), key=lambda p: loads[p])
        owner[i] = r
        loads[r] += costs[i]
    return owner


def run_batch(pd, args, world, rank, barrier, max_over_ranks):
    """512 independent triclinic systems (N log-uniform in [1e3, 1e5]) through pdmk_batch_evaluate, host
    buffers in and out; systems split across ranks by LPT on their point
    counts.  Returns the JSON fragment for the bench line."""
    cells, pos, qs = batch_systems(args.batch_systems, seed=11)
    owner = lpt_partition([len(q) for q in qs], world)
    mine = [i for i in range(len(qs)) if owner[i] == rank]
    t0 = time.perf_counter()
    b = pd.PeriodicDMKBatch([cells[i] for i in mine], [pos[i] for i in mine], n_digits=6, n_per_leaf=300, nz=4)
    t_build = time.perf_counter() - t0
    q_mine = [qs[i] for i in mine]
    # the systems' charges held concatenated and a reused output array, as a
    # caller evaluating the same batch repeatedly keeps them
    q_flat = np.concatenate(q_mine) if q_mine else np.zeros(0)
    out = np.empty(q_flat.shape[0], dtype=np.float64)
    for _ in range(max(3, args.warmup)):   # 1st creates the device state, 2nd records the graphs
        b.evaluate(q_flat, out=out)
    barrier()
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        b.evaluate(q_flat, out=out)
        ts.append(time.perf_counter() - t0)
    barrier()
    t = max_over_ranks(statistics.median(ts))
    total = sum(len(q) for q in qs)
    info = b.info()
    b.close()
    # the same systems as a loop of plain per-system calls (one float tree per
    # system, pdmk_evaluate_float with host buffers, one after another); trees
    # built on host threads (the ctypes calls release the GIL)
    import concurrent.futures as cf
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        singles = list(ex.map(lambda i: pd.PeriodicDMKTree(cells[i], pos[i], n_digits=6, n_per_leaf=300, nz=4,
                                                           precision="float"), mine))
    for tr, q in zip(singles, q_mine):
        tr.evaluate(q)
        tr.evaluate(q)
    barrier()
    tl = []
    for _ in range(max(1, min(args.steps, 3))):
        t0 = time.perf_counter()
        for tr, q in zip(singles, q_mine):
            tr.evaluate(q)
        tl.append(time.perf_counter() - t0)
    barrier()
    t_loop = max_over_ranks(statistics.median(tl))
    for tr in singles:
        tr.close()
    return {"workload": "%d independent periodic systems: triclinic cells (lengths U[0.8,1.2], angles "
                        "U[75,105] deg), N log-uniform in [1e3,1e5] (total %d points), +-1 charges, 6 digits, "
                        "npl 300, nz 4, float trees (mixed precision), one RHS" % (len(qs), total),
            "value": total / t / 1e6, "unit": "Mpts/s", "ms_per_step": t * 1e3,
            "timing": "host wall clock of the synchronous pdmk_batch_evaluate call (charges H2D and potentials "
                      "D2H included; pageable numpy buffers: concatenated charges, a reused float64 output), "
                      "median of steps, max over ranks",
            "partition": "LPT on point counts over %d rank(s)" % world,
            "loop_of_plain_calls": {"value": total / t_loop / 1e6, "unit": "Mpts/s", "ms_per_step": t_loop * 1e3,
                                    "api": "pdmk_evaluate_float per system, one after another (host buffers)"},
            "batch_vs_loop": t_loop / t,
            "host_build_s": t_build, "device_bytes_rank0": info["device_bytes"]}


def smi_id(local):
    """nvidia-smi / NVML identifier of CUDA device `local` (its UUID: nvidia-smi
    indexes ignore CUDA_VISIBLE_DEVICES); the index if the UUID is unknown."""
    try:
        import torch
        return "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        return str(local)


def bind_host_to_gpu(local):
    """Restrict this process to the CPUs NVML reports as local to the GPU (the
    pinned host buffers are then first touched on the GPU's NUMA node).
    Returns the previous affinity, or None if nothing changed."""
    try:
        import pynvml
        pynvml.nvmlInit()
        h = pynvml.nvmlDeviceGetHandleByUUID(smi_id(local))
        old = os.sched_getaffinity(0)
        words = (max(max(old), os.cpu_count() or 1) + 64) // 64
        masks = pynvml.nvmlDeviceGetCpuAffinity(h, words)
        cpus = {64 * w + b for w, m in enumerate(masks) for b in range(64) if (int(m) >> b) & 1} & old
        if not cpus or cpus == old:
            return None
        os.sched_setaffinity(0, cpus)
        return old
    except Exception:
        return None


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
                ["nvidia-smi", "-i", smi_id(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
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
    pl = oracle.Plan(cell, pos, 6, 300, 4)  # build once (not timed), as the reference's tree
    pl.evaluate(q, fast_far=True)  # warm-up
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        pl.evaluate(q, fast_far=True)
        ts.append(time.perf_counter() - t0)
    pl.close()
    t = statistics.median(ts)
    desc = ("CPU oracle (FP64 restatement of the reference evaluate: upward/plane-wave/near/self stages + "
            "CPU NUFFT far field; plan built once, not timed), N=%d uniform in a cube of side %.4f (same density "
            "as the N=%d workload), 6 digits, npl 300, nz 4, %d OpenMP threads, median of %d"
            % (n, scale, n_target, threads, steps))
    return n / t / 1e6, desc, t


def near_traffic_per_launch(pairs_full):
    """DRAM bytes per k_near_tc launch at the bench workload, from the committed
    ncu summary of a smaller case of the same workload (its dram__bytes read +
    write per launch, scaled by the culled pair count: the kernel streams its
    sources once per target tile and kept chunk, which grows with the pairs)."""
    import re
    path = os.path.join(ROOT, "profiles", "k_near_tc_cube2e5_6digits_64rhs.md")
    try:
        text = open(path).read()
    except OSError:
        return None
    b = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", text)
    pr = re.search(r"culled_pairs:\s*([0-9.eE+]+)", text)
    if not b or not pr:
        return None
    v = float(b.group(1)) * pairs_full / float(pr.group(1))
    return {"bytes": v, "source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_near_tc launch at "
                                  "N=2e5 (profiles/k_near_tc_cube2e5_6digits_64rhs.md), scaled by culled pairs"}


def parity_vs_oracle(cell, pos, Q, P_mixed, pot_plain, cols):
    """Accuracy of the timed results against the CPU oracle at the full
    workload size (part of the CPU-baseline leg: the oracle is the checker
    here, nothing timed runs through it).  Q: (N, k) charges; P_mixed: (k, N)
    mixed-precision potentials; pot_plain: FP64 potentials of column 0.
    Relative L2 and max error, max|u - u_ref| / max|u_ref|."""
    import oracle
    t0 = time.perf_counter()
    ref = oracle.evaluate_multi(cell, pos, Q[:, list(cols)], 6, 300, 4)

    def rl2(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    def mx(a, b):
        return float(np.abs(a - b).max() / np.abs(b).max())
    out = {"columns": list(cols),
           "mixed_rel_l2": [rl2(P_mixed[c], ref[:, j]) for j, c in enumerate(cols)],
           "mixed_max_err": [mx(P_mixed[c], ref[:, j]) for j, c in enumerate(cols)],
           "plain_fp64_rel_l2": rl2(pot_plain, ref[:, 0]), "plain_fp64_max_err": mx(pot_plain, ref[:, 0]),
           "oracle": "CPU DMK restatement (FP64, exact reciprocal-lattice far field) at N=%d" % len(pos),
           "oracle_s": time.perf_counter() - t0}
    return out


def run_cpu_configs(args):
    """CPU baseline per workload: the oracle (FP64 restatement of the reference
    evaluate with its CPU NUFFT far field) timed on all host cores on a bounded
    sample of each configuration (same density, digits, n_per_leaf and nz;
    tree build excluded).  Prints one JSON line."""
    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    import oracle

    def timed(cell, pos, q, nd, reps=2):
        pl = oracle.Plan(cell, pos, nd, 300, 4)
        pl.evaluate(q, fast_far=True)
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            pl.evaluate(q, fast_far=True)
            ts.append(time.perf_counter() - t0)
        pl.close()
        return statistics.median(ts)

    out = {"cpu_configs": {}, "cores": threads, "omp_num_threads": threads,
           "kind": "port (FP64 oracle restatement, CPU NUFFT far field; plan build not timed)"}
    rows = out["cpu_configs"]
    # cube workloads at their full size are timed on N = 1e5 samples at the same density
    n = 100000
    for nd in (6, 3):
        scale = (n / 1e6) ** (1.0 / 3.0)
        cell, pos, q = make_system(n, seed=1, scale=scale)
        t = timed(cell, pos, q, nd)
        rows["cube_1e6_%d_digits" % nd] = {"sample_n": n, "s_per_evaluate": t, "mpts_per_s": n / t / 1e6,
                                           "note": "N=1e5 in a cube of the 1e6 workload's density"}
    rows["cube_1e6_64rhs_6_digits"] = dict(rows["cube_1e6_6_digits"],
                                           note="per charge vector: the CPU path evaluates the 64 vectors one "
                                                "after another, so its Mpts*RHS/s equals the 1-RHS rate")
    cell, pos, q = make_system(20000, seed=1)
    t = timed(cell, pos, q, 6)
    rows["cube_2e4_6_digits"] = {"sample_n": 20000, "s_per_evaluate": t, "mpts_per_s": 20000 / t / 1e6,
                                 "note": "the full workload"}
    # clustered triclinic: N = 2e5 sample with the same cell and cluster shape
    cl_cell, cl_pos, cl_q = clustered_system(200000)
    for nd in (9, 12):
        t = timed(cl_cell, cl_pos, cl_q, nd, reps=1)
        rows["clustered_triclinic_2e6_%d_digits" % nd] = {
            "sample_n": 200000, "s_per_evaluate": t, "mpts_per_s": 200000 / t / 1e6,
            "note": "N=2e5 with the workload's cell, 64 clusters of sigma 0.01 and half uniform"}
    # many systems: a loop of per-system evaluates over the first 64 of the 512
    cells, bpos, qs = batch_systems(64, seed=11)
    plans = [oracle.Plan(c, p, 6, 300, 4) for c, p in zip(cells, bpos)]
    t0 = time.perf_counter()
    for pl, qq in zip(plans, qs):
        pl.evaluate(qq, fast_far=True)
    t = time.perf_counter() - t0
    for pl in plans:
        pl.close()
    npts = sum(len(qq) for qq in qs)
    rows["batch_512_systems_6_digits"] = {"sample_n": npts, "s_per_evaluate": t, "mpts_per_s": npts / t / 1e6,
                                          "note": "loop of per-system evaluates over 64 of the 512 systems "
                                                  "(plans built beforehand, not timed)"}
    print(json.dumps(out), flush=True)
    return 0


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    # cpu_baseline runs one untimed evaluate first (the CPU oracle keeps no
    # state between evaluates beyond its thread pool and touched pages)
    v, desc, t = cpu_baseline(args.n, max(1, args.steps), threads)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mpts*RHS/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "uniform cube N=1e6, 6 digits, n_per_leaf 300, nz 4, 1 RHS (bounded sample)"},
            "cpu_baseline": {"value": v, "unit": "Mpts*RHS/s", "cores": threads, "kind": "port", "sample": desc},
            "e2e": {"value": v, "unit": "Mpts*RHS/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_digits3(pd, cell, pos, q, Q, args, world, dev, flush, barrier, max_over_ranks):
    """The same cube at 3 digits: plain FP64 evaluate of one RHS and the
    mixed-precision batched evaluate of the k RHS (device buffers, L2 flushed
    between steps), with the mixed result's rel L2 against the plain one on
    RHS 0.  Returns the JSON fragment."""
    import torch

    n, k = len(q), Q.shape[1]
    td = pd.PeriodicDMKTree(cell, pos, n_digits=3, n_per_leaf=300, nz=4, precision="double")
    tf = pd.PeriodicDMKTree(cell, pos, n_digits=3, n_per_leaf=300, nz=4, precision="float")
    q_d = torch.from_numpy(q).to(dev)
    p_d = torch.empty(n, dtype=torch.float64, device=dev)
    Qc = torch.from_numpy(np.ascontiguousarray(Q.T)).to(dev)
    Pc = torch.empty_like(Qc)
    out = {}
    for name, run, rhs in (("plain_fp64_single_rhs", lambda: td.evaluate_device(q_d.data_ptr(), p_d.data_ptr()), 1),
                           ("mixed_batched", lambda: tf.evaluate_multi_device(k, Qc.data_ptr(), Pc.data_ptr()), k)):
        tree = td if rhs == 1 else tf
        for _ in range(args.warmup):
            run()
        torch.cuda.synchronize()
        sts = []
        barrier()
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            run()
            sts.append(tree.stage_times())
        torch.cuda.synchronize()
        barrier()
        t = max_over_ranks(sum(s["total_ms"] for s in sts) / 1e3) / args.steps
        out[name] = {"value": world * n * rhs / t / 1e6, "unit": "Mpts*RHS/s", "ms_per_step": t * 1e3,
                     "stage_ms_median": {kk: statistics.median(s[kk] for s in sts)
                                         for kk in ("dmk_ms", "near_ms", "nufft_ms", "total_ms")}}
    ref = p_d.cpu().numpy()
    mixed0 = Pc.cpu().numpy()[0]
    td.close()
    tf.close()
    out["mixed_vs_plain_fp64"] = out["mixed_batched"]["value"] / out["plain_fp64_single_rhs"]["value"]
    out["rel_l2_mixed_vs_plain_rhs0"] = float(np.linalg.norm(mixed0 - ref) / np.linalg.norm(ref))
    out["workload"] = "the headline cube (N=%d) at 3 digits, npl 300, nz 4; %d RHS for the batched form" % (n, k)
    return out


def run_ours(args):
    import ctypes

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    host_affinity = bind_host_to_gpu(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import periodicdmk_b200 as pd

    if args.clustered_only:
        dev = torch.device("cuda", local)
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

        def max_over(x):
            if dist is None:
                return x
            tt = torch.tensor([x], device=dev, dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            return float(tt.item())

        out = run_clustered(pd, args, world, dev, flush, (dist.barrier if dist is not None else (lambda: None)),
                            max_over)
        if rank == 0:
            print(json.dumps({"clustered_triclinic": out, "n_gpus": world, "steps": args.steps,
                              "warmup": args.warmup}), flush=True)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    if args.batch_only:
        dev = torch.device("cuda", local)

        def max_over_b(x):
            if dist is None:
                return x
            tt = torch.tensor([x], device=dev, dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            return float(tt.item())

        out = run_batch(pd, args, world, rank, (dist.barrier if dist is not None else (lambda: None)), max_over_b)
        if rank == 0:
            print(json.dumps({"batch": out, "n_gpus": world, "steps": args.steps, "warmup": args.warmup}), flush=True)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    n, k = args.n, args.rhs
    cell, pos, q = make_system(n, seed=1)
    rng = np.random.default_rng(7)
    Q = rng.uniform(-1.0, 1.0, (n, k))
    Q -= Q.mean(axis=0)
    Q[:, 0] = q
    t_build = time.perf_counter()
    tree_d = pd.PeriodicDMKTree(cell, pos, n_digits=6, n_per_leaf=300, nz=4, precision="double")
    t_build = time.perf_counter() - t_build
    tree_f = pd.PeriodicDMKTree(cell, pos, n_digits=6, n_per_leaf=300, nz=4, precision="float")
    info = tree_d.info()
    dev = torch.device("cuda", local)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        tt = torch.tensor([x], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return float(tt.item())

    # ---------------- plain FP64, one RHS (the reference's double evaluate)
    q_d = torch.from_numpy(q).to(dev)
    pot_d = torch.empty(n, dtype=torch.float64, device=dev)
    for _ in range(args.warmup):
        tree_d.evaluate_device(q_d.data_ptr(), pot_d.data_ptr())
    torch.cuda.synchronize()
    plain_st = []
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk1:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            tree_d.evaluate_device(q_d.data_ptr(), pot_d.data_ptr())
            plain_st.append(tree_d.stage_times())
    torch.cuda.synchronize()
    barrier()
    t_plain = max_over_ranks(sum(s["total_ms"] for s in plain_st) / 1e3)
    plain_value = world * n / (t_plain / args.steps) / 1e6
    pot_plain = pot_d.cpu().numpy()

    # ---------------- mixed precision, k RHS in one batched call (headline)
    Qc_d = torch.from_numpy(np.ascontiguousarray(Q.T)).to(dev)       # column-major N x k
    P_d = torch.empty_like(Qc_d)
    for _ in range(args.warmup):
        tree_f.evaluate_multi_device(k, Qc_d.data_ptr(), P_d.data_ptr())
    torch.cuda.synchronize()
    mixed_st = []
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk2:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            tree_f.evaluate_multi_device(k, Qc_d.data_ptr(), P_d.data_ptr())
            mixed_st.append(tree_f.stage_times())
    torch.cuda.synchronize()
    barrier()
    t_mixed = max_over_ranks(sum(s["total_ms"] for s in mixed_st) / 1e3)
    value = world * n * k / (t_mixed / args.steps) / 1e6
    finfo = tree_f.info()
    P_mixed = P_d.cpu().numpy()  # (k, N): row c = RHS c

    # accuracy of the mixed batched result vs the plain FP64 evaluate
    errs = [float(np.linalg.norm(P_mixed[0] - pot_plain) / np.linalg.norm(pot_plain))]
    for c in (1, k // 2, k - 1):
        if c <= 0 or c >= k:
            continue
        qc = torch.from_numpy(np.ascontiguousarray(Q[:, c])).to(dev)
        tree_d.evaluate_device(qc.data_ptr(), pot_d.data_ptr())
        ref = pot_d.cpu().numpy()
        errs.append(float(np.linalg.norm(P_mixed[c] - ref) / np.linalg.norm(ref)))

    # ---------------- end to end through the public C ABI, pinned host buffers:
    # pdmk_evaluate_multi_float (float tree = mixed path), charges N x k doubles in,
    # potentials N x k floats out
    Qh = torch.from_numpy(np.ascontiguousarray(Q.T)).pin_memory()
    Ph = torch.empty((k, n), dtype=torch.float32).pin_memory()
    lib = pd.library()
    D = ctypes.POINTER(ctypes.c_double)
    F = ctypes.POINTER(ctypes.c_float)
    qp = ctypes.cast(Qh.data_ptr(), D)
    pp = ctypes.cast(Ph.data_ptr(), F)
    # warm-up: the first host-buffer call creates the staging buffers, the
    # far-field stream and its chunk FFT plans
    for _ in range(args.warmup):
        if lib.pdmk_evaluate_multi_float(tree_f._h, n, k, qp, pp) != 0:
            raise RuntimeError("pdmk_evaluate_multi_float failed: " + pd._last_error())
    torch.cuda.synchronize()
    e2e = []
    barrier()
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc = lib.pdmk_evaluate_multi_float(tree_f._h, n, k, qp, pp)
        e2e.append(time.perf_counter() - t0)
        if rc != 0:
            raise RuntimeError("pdmk_evaluate_multi_float failed: " + pd._last_error())
    barrier()
    t_e2e = max_over_ranks(sum(e2e))
    e2e_value = world * n * k / (t_e2e / args.steps) / 1e6
    assert np.allclose(Ph.numpy()[0], P_mixed[0], rtol=1e-5, atol=1e-5)

    # the same, with the charges stored in float32 (pdmk_evaluate_multi_float_qf32:
    # half the bytes in, widened to double on the device)
    Qh32 = torch.from_numpy(np.ascontiguousarray(Q.T).astype(np.float32)).pin_memory()
    qp32 = ctypes.cast(Qh32.data_ptr(), F)
    for _ in range(args.warmup):
        if lib.pdmk_evaluate_multi_float_qf32(tree_f._h, n, k, qp32, pp) != 0:
            raise RuntimeError("pdmk_evaluate_multi_float_qf32 failed: " + pd._last_error())
    torch.cuda.synchronize()
    e2e32 = []
    barrier()
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc = lib.pdmk_evaluate_multi_float_qf32(tree_f._h, n, k, qp32, pp)
        e2e32.append(time.perf_counter() - t0)
        if rc != 0:
            raise RuntimeError("pdmk_evaluate_multi_float_qf32 failed: " + pd._last_error())
    barrier()
    t_e2e32 = max_over_ranks(sum(e2e32))
    e2e32_value = world * n * k / (t_e2e32 / args.steps) / 1e6

    # ---------------- rooflines: dominant kernel of each path
    # k_near_tc (mixed): the kernel values run on the CUDA cores (FP32 FMA pipe),
    # the products with the k charge vectors on the tensor cores (tcgen05 TF32),
    # so the ideal time is split by pipe: t_ideal = F_cuda / P_fma32 + F_tc / P_tf32,
    # F_cuda = culled pairs x (2*NC + 14), F_tc = culled pairs x 2k (each product
    # counted once, though a 3xTF32 split issues three MMAs for it);
    # frac = t_ideal / t_measured; achieved / peak are the same ratio expressed
    # as rates over F_cuda + F_tc.
    pk64 = pd.fma_peak_tflops(fp64=True)
    pk32 = pd.fma_peak_tflops(fp64=False)
    pk_tf32 = pd.tc_peak_tflops("tf32")
    pk_dmma = pd.tc_peak_tflops("fp64")

    def med(sts, key):
        return statistics.median(s[key] for s in sts)

    ncoef = int(plain_st[0]["near_ncoef"])
    pairs = plain_st[0]["near_pairs_culled"]
    near_flop_plain = pairs * (2 * ncoef + 14)
    f_cuda = pairs * (2 * ncoef + 14)
    f_tc = pairs * 2 * k
    t_near_mixed = med(mixed_st, "near_ms") * 1e-3
    t_ideal = f_cuda / (pk32 * 1e12) + f_tc / (pk_tf32 * 1e12)
    ach_plain = near_flop_plain / (med(plain_st, "near_ms") * 1e-3) / 1e12
    ach_mixed = (f_cuda + f_tc) / t_near_mixed / 1e12
    peak_mixed = (f_cuda + f_tc) / t_ideal / 1e12
    traffic = near_traffic_per_launch(pairs)
    stage_keys = ("dmk_ms", "near_ms", "nufft_ms", "finalize_ms", "total_ms")
    roofline = {"bound": "tensor", "kernel": "k_near_tc (residual near field, %d RHS per call: FP32 kernel values on "
                                             "the CUDA cores, TF32 hi/lo products on the tensor cores)" % k,
                "achieved": ach_mixed, "peak": peak_mixed, "unit": "TFLOP/s", "frac": t_ideal / t_near_mixed,
                "traffic": traffic["bytes"] if traffic else None,
                "traffic_source": traffic["source"] if traffic else "no ncu summary found",
                "split": {"f_cuda_flop": f_cuda, "f_tc_flop": f_tc, "p_fma32_tflops": pk32,
                          "p_tf32_tflops": pk_tf32, "t_ideal_ms": t_ideal * 1e3, "t_measured_ms": t_near_mixed * 1e3,
                          "frac_counting_three_tf32_products": (f_cuda / (pk32 * 1e12) + 3 * f_tc / (pk_tf32 * 1e12))
                          / t_near_mixed},
                "peak_source": "of measured: FP32 FMA probe (pdmk_fma_peak) and tcgen05 TF32 MMA probe "
                               "(pdmk_tc_peak) on this GPU, combined by pipe",
                "flop_convention": "culled pairs x (2*NC + 14) on the CUDA cores + culled pairs x 2k on the tensor "
                                   "cores",
                "stage_ms_median": {kk: med(mixed_st, kk) for kk in stage_keys}}
    measured_peaks = {"fma_fp32_tflops": pk32, "fma_fp64_tflops": pk64, "tcgen05_tf32_tflops": pk_tf32,
                      "dmma_fp64_tflops": pk_dmma}
    plain = {"value": plain_value, "unit": "Mpts*RHS/s", "ms_per_step": t_plain / args.steps * 1e3,
             "gpu_launches": info["launches_per_evaluate"] * args.steps,
             "roofline": {"bound": "fp64", "kernel": "k_near (residual near field)", "achieved": ach_plain,
                          "peak": pk64, "unit": "TFLOP/s", "frac": ach_plain / pk64,
                          "peak_source": "measured FP64 FMA probe on this GPU (pdmk_fma_peak)",
                          "algorithmic_flop_per_launch": near_flop_plain,
                          "stage_ms_median": {kk: med(plain_st, kk) for kk in stage_keys}},
             "clocks": clk1.summary()}
    line = {"metric": METRIC, "value": value, "unit": "Mpts*RHS/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_mixed / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "uniform cube N=1e6 (seed 1), %d charge vectors U[-1,1] minus mean, "
                                   "6 digits, n_per_leaf 300, nz 4, mixed-precision batched evaluate" % k,
                       "n_points": n, "rhs": k, "n_digits": 6, "n_per_leaf": 300, "nz": 4,
                       "parallelism": "replicas x%d" % world, "l2": "flushed between steps (256 MB write)",
                       "tree": {kk: info[kk] for kk in ("n_all", "n_boxes", "n_levels", "n_target_leaves",
                                                         "p", "n_pw", "device_bytes")},
                       "tree_build_s": t_build,
                       "precision": "FP32 near field (double-float coordinate differences, FP64 merge), FP32 "
                                    "moments / transforms / leaf evaluation (tensor-core products on TF32 hi/lo "
                                    "splits, short accumulation segments), FP64 far field and accumulation"},
            "rel_l2_vs_fp64": max(errs),
            "mixed_vs_plain_fp64": value / plain_value,
            "plain_fp64_single_rhs": plain,
            "e2e": {"value": e2e_value, "unit": "Mpts*RHS/s", "h2d_bytes_per_step": 8 * n * k,
                    "d2h_bytes_per_step": 4 * n * k, "ms_per_step": t_e2e / args.steps * 1e3,
                    "api": "pdmk_evaluate_multi_float (pinned host buffers)"},
            "e2e_float32_charges": {"value": e2e32_value, "unit": "Mpts*RHS/s", "h2d_bytes_per_step": 4 * n * k,
                                    "d2h_bytes_per_step": 4 * n * k, "ms_per_step": t_e2e32 / args.steps * 1e3,
                                    "api": "pdmk_evaluate_multi_float_qf32 (charges stored in float32, pinned "
                                           "host buffers)"},
            "gpu_launches": finfo["launches_last_multi"] * args.steps,
            "roofline": roofline, "measured_peaks": measured_peaks, "clocks": clk2.summary()}
    tree_d.close()
    tree_f.close()
    if not args.no_digits3:
        line["digits_3"] = run_digits3(pd, cell, pos, q, Q, args, world, dev, flush, barrier, max_over_ranks)
    if args.batch_systems > 0:
        line["batch"] = run_batch(pd, args, world, rank, barrier, max_over_ranks)
    if args.clustered_digits.strip():
        line["clustered_triclinic"] = run_clustered(pd, args, world, dev, flush, barrier, max_over_ranks)
    if host_affinity is not None:
        os.sched_setaffinity(0, host_affinity)  # the CPU baseline gets every host core
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, desc, _ = cpu_baseline(n, 3, threads)
        line["cpu_baseline"] = {"value": v, "unit": "Mpts*RHS/s", "cores": threads, "kind": "port", "sample": desc}
        par = parity_vs_oracle(cell, pos, Q, P_mixed, pot_plain, (0, k - 1))
        line["parity_vs_oracle"] = par
        line["rel_l2_vs_oracle"] = max(par["mixed_rel_l2"])
        line["max_err_vs_oracle"] = max(par["mixed_max_err"])
    if rank == 0:
        print(json.dumps(line), flush=True)
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
    ap.add_argument("--rhs", type=int, default=64)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-systems", type=int, default=512,
                    help="systems of the many-systems measurement (0 skips it)")
    ap.add_argument("--clustered-digits", default="9,12",
                    help="digit counts of the clustered triclinic FP64 measurement ('' skips it)")
    ap.add_argument("--clustered-n", type=int, default=2000000)
    ap.add_argument("--cpu-configs", action="store_true",
                    help="time only the CPU oracle on bounded samples of every workload (JSON line)")
    ap.add_argument("--clustered-only", action="store_true",
                    help="run only the clustered triclinic FP64 measurement (its JSON fragment alone)")
    ap.add_argument("--no-digits3", action="store_true",
                    help="skip the 3-digit measurement of the headline cube")
    ap.add_argument("--batch-only", action="store_true",
                    help="run only the many-systems measurement of --batch-systems systems (its JSON fragment alone)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.cpu_configs:
        return run_cpu_configs(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
