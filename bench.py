"""Benchmark of the Kino-PAX tree-expansion iteration on one B200 (or N independent replicas).

Metric: valid expansions/s (children that passed every RK4-step validity and collision check),
the reference's own counter (sum of d_validCounterArray_, src/planners/KPAX.cu:393).

  value  one planner iteration per step (frontier scan, fused expansion, region scores) on the
         12D-quadrotor configuration (building scene, 1000 AABBs, 2^16 expansions/iteration,
         25 RK4 steps of 0.02 s), inputs resident on the device, L2 flushed before every timed
         iteration, kernels timed with CUDA events on the planner stream;
  e2e    whole plans through the C ABI (kpax_plan_host) from host buffers: obstacles, start and
         goal copied in and the path read back inside the timed region (host wall clock);
  roofline  the expansion kernel: executed RK4 steps x FP32 FLOP per step / kernel time;
  cpu_baseline  the reference's own propagation + collision + region routines compiled for the
         host (oracle/_ref, OpenMP over all cores) on a bounded sample of the same children.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload quad|dubins|di|segments|collide|learned|batch|quad-ref|expansion-scan]

Other workloads: dubins / di (the same iteration on the other models), segments (2^22 independent
Dubins segments through kpax_propagate_batch), collide (2^22 swept-box queries through
kpax_collide_batch), learned (learned-vs-plain A/B on 256 held-out scenes, tensor-core pass and
training rates), batch (1024 mixed queries in one batched plan), quad-ref (the reference's own
quadrotor block on its quadTrees scene, beside the reference's CUDA build), expansion-scan (the
fused iteration's phase times against the children per iteration, building and empty scenes).
The reference arm has no counterpart for learned and batch and says so.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path[:0] = [str(ROOT / "kino-pax-fork_b200")]

import kpax  # noqa: E402
import kpax_envs as E  # noqa: E402

METRIC = "valid expansions/s"
UNIT = "expansions/s"
# Algorithmic FP32 work per RK4 step (FMA = 2), counted from a CSE'd restatement of the models.
FLOP_PER_STEP = {kpax.MODEL_DOUBLE_INTEGRATOR: 18, kpax.MODEL_DUBINS_AIRPLANE: 51, kpax.MODEL_QUADROTOR: 498}
# dram__bytes_read.sum + dram__bytes_write.sum of one steady-state k_iterate launch (the fused
# iteration, 2^16 children, L2 flushed before it) in an ncu capture of the default workload; none
# for the others
ITERATE_DRAM_BYTES = {kpax.MODEL_QUADROTOR: 2093824 + 0}
# the same sum for the one-pass kernel (kpax_propagate_batch_noalloc) on 2^20 Dubins segments, L2
# flushed before the step, per segment
ONE_PASS_DRAM_BYTES_PER_SEGMENT = (25186304 + 48397824) / (1 << 20)
# the same sum over the three phase kernels of one 2^20-segment Dubins batch (L2 flushed before the
# step, no cache flush between the kernels), per segment: scaled by the segment count, as the
# traffic grows with it
PHASED_DRAM_BYTES_PER_SEGMENT = (30508800 + 103499264) / (1 << 20)
WORKLOADS = {
    "quad": (kpax.PRESET_QUAD, E.quad_scene, "12D quadrotor, building scene (1000 AABBs incl. windowed wall), "
             "2^16 expansions/iteration, 25 RK4 steps of 0.02 s"),
    "dubins": (kpax.PRESET_DUBINS, E.dubins_scene, "Dubins airplane, forest of 200 columns, 2^16 expansions/iteration, "
               "20 RK4 steps of 0.05 s"),
    "di": (kpax.PRESET_DI, E.di_scene, "6D double integrator, 20 AABBs, 2^14 expansions/iteration, U{1..10} steps of 0.1 s"),
}
FLUSH_BYTES = 256 << 20  # > 126 MB L2
COLLIDE_DESC = ("swept-box queries against the spatial hash (isMotionValidSpatialHash): 2^22 boxes, corners uniform in "
                "[0,100]^3, extents U[0,0.2] m per axis (one integration step), building scene of 1000 AABBs")
COLLIDE_BYTES_PER_BOX = 25  # algorithmic: two corners in (6 floats), one verdict byte out
# DRAM bytes (read + write) per box of one k_collide_batch launch on 2^20 boxes, L2 flushed before it,
# in an ncu capture (dram__bytes.sum.per_second x gpu__time_duration.sum / boxes)
COLLIDE_DRAM_BYTES_PER_BOX = 937.433526e9 * 27.68e-6 / (1 << 20)
SEGMENTS_DESC = ("Dubins airplane propagation/collision microbench: 2^22 independent segments, parents uniform within "
                 "the bounds, forest of 200 columns, 20 RK4 steps of 0.05 s")


def load_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0, "fallback": True}


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(tempfile.mkstemp(prefix="kpax_clocks_", suffix=".csv")[1])

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader",
                                          "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self) -> dict | None:
        if not self.proc:
            return None
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1].split()[0]))
                mx.append(float(f[2].split()[0]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        self.path.unlink(missing_ok=True)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def frontier_parents(cfg, obs, start, goal, n_parents: int = 2048, iters: int = 12):
    """Parents for the CPU baseline: the nodes a short CPU plan (the oracle, same configuration)
    appended in its last iterations, i.e. a steady-state frontier like the GPU's timed iterations."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    small = cfg.copy()
    small.expansions_per_iter = min(cfg.expansions_per_iter, 1 << 15)
    r = O.plan(small, start, goal, obs, plan_idx=7, max_iters=iters, stop_at_goal=False)
    new = int(r["iter_appended"][-3:].sum())
    rows = r["rows"][-max(min(new, n_parents), 1):, : cfg.state_dim]
    return np.ascontiguousarray(rows, np.float32)


def cpu_reference_rate(cfg, obs, parents, budget_s: float, per_parent: int = 32, max_children: int = 1 << 16):
    """The reference's own per-child expansion body (oracle/_ref, OpenMP, all host threads)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    ref = O.RefLib(cfg.model)
    ref.set_obstacles(obs)
    threads = ref.L.kref_max_threads()
    n1, P = ref.num_r1, ref.r2_per_r1
    n = min(max_children, parents.shape[0] * per_parent)
    draws = E.uniform_draws(n, 99)
    if cfg.fixed_steps:
        N = cfg.max_propagation_duration
        draws[:, 4] = np.float32((N - 0.5) / N)
    scores = np.zeros(n1, np.float32)
    valid_total, t_total, batches = 0, 0.0, 0
    # size the sample to the budget: shrink the batch if one batch takes too long
    while t_total < budget_s:
        flags = np.zeros(n1 * P, np.int32)
        counter = np.zeros(n1, np.int32)
        vc = np.zeros(n1, np.int32)
        t0 = time.perf_counter()
        nv, _, _ = ref.expand(parents, per_parent, draws[:n], scores, flags, counter, vc, threads)
        dt = time.perf_counter() - t0
        valid_total += nv
        t_total += dt
        batches += 1
        if batches == 1 and dt > budget_s / 3 and n > 4096:
            n //= 4
    return valid_total / t_total, threads, (f"{batches} batches of {n} children (32 per parent) of {parents.shape[0]} "
                                            f"steady-state frontier parents, {valid_total / (batches * n):.2f} valid, "
                                            f"{t_total:.1f} s")


def combine_over_ranks(dist, device, t_s: float, valid: float) -> tuple[float, float]:
    """Replicas: the job time is the slowest rank's device time, the work is the sum over ranks."""
    if dist is None:
        return t_s, float(valid)
    import torch

    tt = torch.tensor([t_s], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    vv = torch.tensor([float(valid)], dtype=torch.float64, device=device)
    dist.all_reduce(vv, op=dist.ReduceOp.SUM)
    return float(tt.item()), float(vv.item())


def dist_setup(n_gpus: int):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def segment_inputs(n: int, seed: int):
    """The microbench's parents (uniform within the Dubins bounds) and its forest scene."""
    cfg = kpax.preset(kpax.PRESET_DUBINS)
    obs, _, _ = E.dubins_scene()
    parents = E.sample_states(kpax.MODEL_DUBINS_AIRPLANE, n, seed, vmin=cfg.v_min, vmax=cfg.v_max)
    return cfg, obs, parents


def cpu_segments_rate(budget_s: float, n: int = 1 << 16, steps: int = 3):
    """The reference's own propagate + collide routine (oracle/_ref, OpenMP, all host threads) on
    microbench segments: valid segments per second, threads, sample description."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    cfg, obs, parents = segment_inputs(n, 3)
    ref = O.RefLib(cfg.model)
    ref.set_obstacles(obs)
    threads = ref.L.kref_max_threads()
    draws = E.uniform_draws(n, 97)
    draws[:, 4] = np.float32((cfg.max_propagation_duration - 0.5) / cfg.max_propagation_duration)  # 20 steps
    tot_v, tot_t, runs = 0, 0.0, 0
    while runs < steps or tot_t < budget_s:
        t0 = time.perf_counter()
        _, valid = ref.propagate(parents, draws, use_hash=True, nthreads=threads)
        tot_t += time.perf_counter() - t0
        tot_v += int(valid.sum())
        runs += 1
        if tot_t > 4 * budget_s:
            break
    return (tot_v / tot_t, threads,
            f"{runs} runs of {n} segments (20 steps each), {tot_v / (runs * n):.2f} valid, {tot_t:.1f} s", 1000 * tot_t / runs)


def collide_inputs(n: int, seed: int):
    """Boxes of the collision microbench and the scene, with the quadrotor preset's hash cell."""
    cfg = kpax.preset(kpax.PRESET_QUAD)
    obs, _, _ = E.quad_scene()
    rng = np.random.default_rng(seed)
    lo = rng.uniform(0.0, 100.0, (n, 3)).astype(np.float32)
    hi = (lo + rng.uniform(0.0, 0.2, (n, 3))).astype(np.float32)
    return cfg, obs, lo, hi


def cpu_collide_rate(budget_s: float, n: int = 1 << 18):
    """The reference's own isMotionValidSpatialHash (oracle/_ref, OpenMP, all host threads) on the
    microbench's boxes: queries per second, threads, sample description, ms per run."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    cfg, obs, lo, hi = collide_inputs(n, 11)
    ref = O.RefLib(cfg.model)
    ref.set_obstacles(obs)
    threads = ref.L.kref_max_threads()
    tot_t, runs = 0.0, 0
    while runs < 3 or tot_t < budget_s:
        t0 = time.perf_counter()
        ref.collide_batch(lo, hi, use_hash=True, nthreads=threads)
        tot_t += time.perf_counter() - t0
        runs += 1
        if tot_t > 4 * budget_s:
            break
    return n * runs / tot_t, threads, f"{runs} runs of {n} boxes (reference 5 m / 16-slot grid), {tot_t:.1f} s", 1000 * tot_t / runs


def run_collide(args) -> None:
    """2^22 swept-box queries per step through kpax_collide_batch (the expansion's per-step query)."""
    import torch

    ws, rank, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    n = 1 << args.boxes_log2
    cfg, obs, lo, hi = collide_inputs(n, 13 + rank)
    if not args.no_tune:
        import kpax_autotune

        cfg, _ = kpax_autotune.tuned(cfg, obs.shape[0])
    d_obs = torch.from_numpy(obs).cuda()
    env = kpax.Env(cfg, d_obs.data_ptr(), obs.shape[0])
    d_lo, d_hi = torch.from_numpy(lo).cuda(), torch.from_numpy(hi).cuda()
    free = torch.empty(n, dtype=torch.uint8, device="cuda")
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    def launch():
        kpax.collide_batch(env, d_lo.data_ptr(), d_hi.data_ptr(), n, free.data_ptr(), stream=stream.cuda_stream)

    for _ in range(max(args.warmup, 3)):
        launch()
    launches0 = kpax.kernel_launches()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with Clocks(local) as clk:
        for i in range(args.steps):
            flush.fill_(i & 0xFF)  # evict the 126 MB L2 between steps, outside the events
            ev[i][0].record(stream)
            launch()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = kpax.kernel_launches() - launches0
    t_s = sum(a.elapsed_time(b) for a, b in ev) / 1000.0
    t_job, boxes_all = combine_over_ranks(dist, "cuda", t_s, n * args.steps)
    value = boxes_all / t_job
    free_fraction = float(free.float().mean().item())
    peaks = load_peaks()
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    achieved = COLLIDE_BYTES_PER_BOX * n * args.steps / t_s / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": int(COLLIDE_DRAM_BYTES_PER_BOX * n),
                "traffic_note": "DRAM bytes per launch from an ncu capture of 2^20 boxes (summary under profiles/), scaled "
                                "to the box count: 24.7 B per box against 25 algorithmic, no re-reads",
                "kernel": "k_collide_batch", "work": f"{COLLIDE_BYTES_PER_BOX} algorithmic bytes per box (corners in, "
                "verdict out); the grid's offsets, entries and boxes are read from L2",
                "peak_source": "measured copy" if "fallback" not in peaks else "fallback",
                "ms_per_launch": 1000 * t_s / args.steps}
    # end to end through the C ABI from pinned host buffers: corners in, verdicts out
    h_lo, h_hi = torch.from_numpy(lo).pin_memory(), torch.from_numpy(hi).pin_memory()
    h_free = torch.empty(n, dtype=torch.uint8).pin_memory()
    e_steps = max(2, min(args.steps, 5))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(e_steps):
        d_lo.copy_(h_lo, non_blocking=True)
        d_hi.copy_(h_hi, non_blocking=True)
        launch()
        h_free.copy_(free, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e = {"value": n * e_steps / (e0.elapsed_time(e1) / 1000.0), "unit": "queries/s",
           "h2d_bytes_per_step": int(2 * lo.nbytes), "d2h_bytes_per_step": int(h_free.numel())}
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        try:
            rate, cores, sample, _ = cpu_collide_rate(args.cpu_seconds)
            cpu = {"value": rate, "unit": "queries/s", "cores": cores, "kind": "reference", "sample": sample}
        except (FileNotFoundError, OSError) as exc:
            cpu = {"value": None, "unit": "queries/s", "cores": 0, "kind": "reference", "sample": f"unavailable: {exc}"}
    if rank == 0:
        line = {
            "metric": "swept-box queries/s", "value": value, "unit": "queries/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * t_job / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
            "config": {"workload": COLLIDE_DESC if n == 1 << 22 else COLLIDE_DESC.replace("2^22", f"2^{args.boxes_log2}"),
                       "boxes_per_step": n, "hash_cell_size": cfg.hash_cell_size, "free_fraction": free_fraction,
                       "l2": "flushed before each timed step (256 MiB write, outside the events)",
                       "parallelism": f"replicas x{ws}"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def run_reference(args) -> None:
    ws, rank, _ = dist_setup(args.gpus)
    if rank != 0:
        return
    if args.workload in ("learned", "batch"):
        why = ("the reference has no learned proposal" if args.workload == "learned" else
               "the reference plans one query per plan() call with a compile-time model; its per-child routines are "
               "timed by the single-query workloads")
        print(json.dumps({"impl": "reference", "unavailable": why}), flush=True)
        return
    if args.workload == "collide":
        rate, threads, sample, ms = cpu_collide_rate(min(20.0, 2.0 * max(args.steps, 1)))
        line = {
            "impl": "reference", "metric": "swept-box queries/s", "value": rate, "unit": "queries/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
            "config": {"workload": COLLIDE_DESC, "boxes_per_step": 1 << 18, "parallelism": "host OpenMP"},
            "cpu_baseline": {"value": rate, "unit": "queries/s", "cores": threads, "kind": "reference", "sample": sample},
            "e2e": {"value": rate, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return
    if args.workload == "segments":
        rate, threads, sample, ms = cpu_segments_rate(min(20.0, 2.0 * max(args.steps, 1)), steps=max(args.steps, 1))
        line = {
            "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32", "data": "synthetic",
            "config": {"workload": SEGMENTS_DESC, "segments_per_step": 1 << 16, "parallelism": "host OpenMP"},
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return
    if args.workload == "quad-ref":
        pre, scene, desc = kpax.PRESET_QUAD_REF, quad_trees_scene, QUAD_REF_DESC
    else:
        pre, scene, desc = WORKLOADS[args.workload]
    cfg = kpax.preset(pre)
    obs, start, goal = scene()
    parents = frontier_parents(cfg, obs, start, goal)
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    ref = O.RefLib(cfg.model, "quad_ref" if args.workload == "quad-ref" else None)
    ref.set_obstacles(obs)
    threads = ref.L.kref_max_threads()
    n1, P = ref.num_r1, ref.r2_per_r1
    n = min(cfg.expansions_per_iter, parents.shape[0] * 32)
    draws = E.uniform_draws(n, 98)
    if cfg.fixed_steps:
        draws[:, 4] = np.float32((cfg.max_propagation_duration - 0.5) / cfg.max_propagation_duration)
    scores = np.zeros(n1, np.float32)

    def step(m):
        flags = np.zeros(n1 * P, np.int32)
        c = np.zeros(n1, np.int32)
        v = np.zeros(n1, np.int32)
        t0 = time.perf_counter()
        nv, _, _ = ref.expand(parents, 32, draws[:m], scores, flags, c, v, threads)
        return nv, time.perf_counter() - t0

    m = n
    for i in range(max(args.warmup, 1)):
        _, dt = step(m)
        if i == 0 and dt * args.steps > 120 and m > 4096:  # keep the whole run within a few minutes
            m = max(4096, int(m * 120 / (dt * args.steps)))
    tot_v, tot_t = 0, 0.0
    for _ in range(args.steps):
        nv, dt = step(m)
        tot_v += nv
        tot_t += dt
    value = tot_v / tot_t
    sample = f"{m} children of frontier parents per step (reference per-child body, KPAX.cu:381-396)"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * tot_t / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": {"workload": desc, "expansions_per_iter": m, "parallelism": "host OpenMP"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def pct_all(ms, q: float):
    """Nearest-rank percentile of plan times with unsolved plans as +inf (None when it is one)."""
    if not len(ms):
        return None
    v = float(np.quantile(np.asarray(ms, np.float64), q / 100.0, method="inverted_cdf"))
    return v if np.isfinite(v) else None


def query_outcomes(pl, queries: np.ndarray, obs: np.ndarray) -> dict:
    """Whole plans of a query set (rows: start xyz, goal xyz) through kpax_plan_host from host
    buffers: success (goal reached), time to solution (host clock of the call), path costs."""
    S = pl.sample_dim
    tts, all_ms, costs, found = [], [], [], 0
    valid, secs = 0, 0.0
    for q in queries:
        st, gl = np.zeros(S, np.float32), np.zeros(S, np.float32)
        st[:3], gl[:3] = q[:3], q[3:6]
        t0 = time.perf_counter()
        r = pl.plan_host(st, gl, obs)
        dt = 1000.0 * (time.perf_counter() - t0)
        all_ms.append(dt if r.found else float("inf"))
        valid += r.valid_expansions
        secs += dt / 1000.0
        if r.found:
            found += 1
            tts.append(dt)
            costs.append(float(r.path_cost))
    n = len(queries)
    return {"queries": n, "success_rate": found / max(n, 1),
            "tts_ms_p50": float(np.percentile(tts, 50)) if tts else None,
            "tts_ms_p95": float(np.percentile(tts, 95)) if tts else None,
            "tts_ms_p50_all": pct_all(all_ms, 50), "tts_ms_p95_all": pct_all(all_ms, 95),
            "path_cost_median": float(np.median(costs)) if costs else None,
            "valid_expansions_per_s": valid / secs if secs > 0 else None}


def reference_cuda_leg(cfg, obs, start, goal, queries, args) -> dict:
    """The reference's own CUDA planner (KPAX::plan compiled unmodified for sm_100a, run as a
    subprocess by oracle/refcuda) on this workload at the reference's duration draw (steps
    1 + (int)(u * 25)), beside this library at the same configuration: whole plans of the fixed pair
    (valid expansions per second of plan time), the rate of its large iterations, and the outcomes
    of the query set."""
    sys.path.insert(0, str(ROOT / "oracle" / "refcuda"))
    import refcuda

    pair = [[*start[:3], *goal[:3]]]
    res = refcuda.run("quad_c2", obs, pair, iteration_cap=cfg.max_iter, repeats=args.ref_cuda_plans, timeout_s=300)
    summ = refcuda.summarise(res)
    if "unavailable" in summ:
        return summ
    out = {"value": summ["value"], "unit": UNIT, "kind": "reference CUDA build: KPAX::plan from its own sources, sm_100a",
           "config": "12D quadrotor, building scene, h 0.02 s, steps 1 + (int)(u * 25) (the reference's draw), "
                     "Zc in [0, 2g], torques in [-0.1, 0.1], tree capacity 2^20, 300 iterations",
           "plans": summ["plans"], "iterations": summ["iterations"], "capacity_stops": summ["capacity_stops"],
           "children": summ["children"], "valid": summ["valid"], "seconds": summ["seconds"], "steady": summ["steady"],
           "timing": "host clock around KPAX::plan, less the harness's own check before each iteration"}
    # this library at the same configuration (drawn steps), the same plans through kpax_plan
    c = cfg.copy()
    c.fixed_steps = 0
    import torch

    d_obs = torch.from_numpy(obs).cuda()
    pl = kpax.KPAX(c)
    pl.plan(start, goal, d_obs.data_ptr(), obs.shape[0])  # warm-up (graph capture)
    v, t = 0, 0.0
    for _ in range(args.ref_cuda_plans):
        t0 = time.perf_counter()
        r = pl.plan(start, goal, d_obs.data_ptr(), obs.shape[0])
        t += time.perf_counter() - t0
        v += r.valid_expansions
    out["ours_same_config"] = {"value": v / t if t > 0 else None, "unit": UNIT, "plans": args.ref_cuda_plans,
                               "note": "kpax_plan with the reference's duration draw, 2^16 children per iteration, "
                                       "host clock around the call"}
    # plan outcomes on the query set, both sides at that configuration
    if len(queries):
        rq = refcuda.summarise(refcuda.run("quad_c2", obs, queries, iteration_cap=cfg.max_iter, repeats=1, timeout_s=300))
        if "unavailable" not in rq:
            tts = rq["tts_ms"]
            out["query_set"] = {"queries": rq["plans"], "success_rate": rq["success_rate"],
                                "tts_ms_p50": float(np.percentile(tts, 50)) if tts else None,
                                "tts_ms_p95": float(np.percentile(tts, 95)) if tts else None,
                                "path_cost_median": float(np.median(rq["path_costs"])) if rq["path_costs"] else None,
                                "capacity_stops": rq["capacity_stops"]}
        out["ours_same_config"]["query_set"] = query_outcomes(pl, queries, obs)
    pl.close()
    return out


QUAD_REF_DESC = ("12D quadrotor with the reference's own configuration block (h 0.1 s, steps 1 + (int)(u * 10), Zc in "
                 "[0, 30], torques in [-pi, pi], tree capacity 400000, 300 iterations) on its quadTrees scene (158 boxes) "
                 "with its drivers' pair (10, 8, 5) -> (80, 95, 90)")


def quad_trees_scene():
    """The reference's quadTrees obstacle file (include/config/obstacles/quadTrees), committed as a
    fixture, with its drivers' start and goal (comprehensive_benchmark.cu:251-252)."""
    obs = np.ascontiguousarray(np.load(ROOT / "tests" / "golden" / "quad_quadTrees.npz")["obstacles"], np.float32)
    start, goal = np.zeros(12, np.float32), np.zeros(12, np.float32)
    start[:3], goal[:3] = (10.0, 8.0, 5.0), (80.0, 95.0, 90.0)
    return obs, start, goal


def ks_distance(a, b) -> float | None:
    a, b = np.sort(np.asarray(a, np.float64)), np.sort(np.asarray(b, np.float64))
    if not a.size or not b.size:
        return None
    x = np.union1d(a, b)
    return float(np.max(np.abs(np.searchsorted(a, x, "right") / a.size - np.searchsorted(b, x, "right") / b.size)))


def ours_plans(cfg, obs, start, goal, n: int, warmup: int) -> dict:
    """n plans of this library through kpax_plan_host (host buffers), host clock per call."""
    pl = kpax.KPAX(cfg)
    for _ in range(max(warmup, 1)):
        pl.plan_host(start, goal, obs)
    found, tts, costs, valid, secs, iters = 0, [], [], 0, 0.0, []
    for _ in range(n):
        t0 = time.perf_counter()
        r = pl.plan_host(start, goal, obs)
        dt = time.perf_counter() - t0
        secs += dt
        valid += r.valid_expansions
        iters.append(r.iters)
        if r.found:
            found += 1
            tts.append(1000 * dt)
            costs.append(float(r.path_cost))
    pl.close()
    return {"plans": n, "success_rate": found / n, "tts_ms_p50": float(np.percentile(tts, 50)) if tts else None,
            "tts_ms_p95": float(np.percentile(tts, 95)) if tts else None,
            "path_cost_median": float(np.median(costs)) if costs else None, "iterations_median": float(np.median(iters)),
            "valid_expansions_per_s": valid / secs, "seconds": secs, "path_costs": costs}


def reference_plans(ref_cfg: str, obs, start, goal, n: int, iteration_cap: int) -> dict:
    """n plans of the reference's CUDA build (KPAX::plan) through oracle/refcuda."""
    sys.path.insert(0, str(ROOT / "oracle" / "refcuda"))
    import refcuda

    rs = refcuda.summarise(refcuda.run(ref_cfg, obs, [[*start[:3], *goal[:3]]], iteration_cap=iteration_cap, repeats=n,
                                       timeout_s=300))
    if "unavailable" in rs:
        return rs
    t = rs["tts_ms"]
    return {"plans": rs["plans"], "success_rate": rs["success_rate"],
            "tts_ms_p50": float(np.percentile(t, 50)) if t else None,
            "tts_ms_p95": float(np.percentile(t, 95)) if t else None,
            "path_cost_median": float(np.median(rs["path_costs"])) if rs["path_costs"] else None,
            "capacity_stops": rs["capacity_stops"], "valid_expansions_per_s": rs["value"], "path_costs": rs["path_costs"],
            "kind": "reference CUDA build: KPAX::plan from its own sources, sm_100a; seeds from the wall clock as in the "
                    "reference (KPAX.cu:90-91); a plan is ended (unsolved) before an iteration whose frontier has more "
                    "entries than the tree has free slots, where the reference appends past its buffers (KPAX.cu:325-333)"}


def run_quad_ref(args) -> None:
    """Whole plans at the reference's own quadrotor configuration: this library through
    kpax_plan_host (host buffers) beside the reference's CUDA build through KPAX::plan, the same
    number of plans each, at the configured tree capacity (400000) and at 2^22: success (goal
    reached), time to solution, path-cost distributions."""
    import torch

    ws, rank, local = dist_setup(args.gpus)
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device (no CPU fallback)")
    torch.cuda.set_device(local)
    obs, start, goal = quad_trees_scene()
    n = args.plans_ref
    sides = []
    launches0 = kpax.kernel_launches()
    with Clocks(local) as clk:
        # the 2^22 capacity costs the reference a curand_init of 4M generator states per plan (and larger
        # iterations): fewer plans there
        for cap, ref_cfg, n_cap in ((400000, "quad_ref", n), (1 << 22, "quad_ref_4m", min(n, args.plans_ref_big))):
            cfg = kpax.preset(kpax.PRESET_QUAD_REF)
            cfg.seed = cfg.seed + 1000003 * rank
            cfg.max_tree_size = cap
            cfg.expansions_per_iter = cap
            sides.append({"tree_capacity": cap, "ours": ours_plans(cfg, obs, start, goal, n_cap, args.warmup), "cfg": cfg,
                          "ref_cfg": ref_cfg, "n": n_cap})
    launches = kpax.kernel_launches() - launches0
    for sd in sides:
        ref = None
        if rank == 0 and not args.no_ref_cuda:
            ref = reference_plans(sd["ref_cfg"], obs, start, goal, sd["n"], sd["cfg"].max_iter)
            if "path_costs" in ref:
                ref["path_cost_ks_vs_ours"] = ks_distance(sd["ours"]["path_costs"], ref.pop("path_costs"))
        sd["reference_cuda"] = ref
        sd["ours"].pop("path_costs")
        del sd["cfg"], sd["ref_cfg"], sd["n"]
    if rank == 0:
        head = sides[0]["ours"]
        value = head["valid_expansions_per_s"]
        cfg = kpax.preset(kpax.PRESET_QUAD_REF)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": n, "warmup": args.warmup,
                "ms_per_step": 1000 * head["seconds"] / n, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "fp32", "data": "the reference's quadTrees obstacle file",
                "config": {"workload": QUAD_REF_DESC, "expansions_per_iter": cfg.expansions_per_iter,
                           "l2": "whole plans back to back (each plan's data is larger than L2 only late in a plan)",
                           "parallelism": f"replicas x{ws}"},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": obs.nbytes + 2 * 4 * cfg.sample_dim,
                        "d2h_bytes_per_step": 128, "plans": n, "success_rate": head["success_rate"],
                        "tts_ms_p50": head["tts_ms_p50"], "tts_ms_p95": head["tts_ms_p95"]},
                "plan_outcomes": sides, "gpu_launches": launches, "clocks": clk.summary()}
        print(json.dumps(line), flush=True)


def run_ours(args) -> None:
    import torch

    ws, rank, local = dist_setup(args.gpus)
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device (no CPU fallback)")
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    pre, scene, desc = WORKLOADS[args.workload]
    cfg = kpax.preset(pre)
    cfg.seed = cfg.seed + 1000003 * rank
    obs, start, goal = scene()
    tuning = None
    if not args.no_tune:  # launch parameters from the autotuner's cache (plans are unchanged)
        import kpax_autotune

        cfg, tuning = kpax_autotune.tuned(cfg, obs.shape[0])
    d_obs = torch.from_numpy(obs).cuda()
    pl = kpax.KPAX(cfg)
    stream = torch.cuda.ExternalStream(pl.stream)
    pl.begin(start, goal, d_obs.data_ptr(), obs.shape[0])
    _, grow0 = pl.iterate_timed(8, 0)  # grow the frontier until every iteration uses the full budget
    _, grow1 = pl.iterate_timed(max(args.warmup, 3), FLUSH_BYTES)
    tree0 = 1 + grow0["appended"] + grow1["appended"]  # nodes when the timed iterations start
    launches0 = kpax.kernel_launches()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        # whole iterations, events only between them: the kernels overlap their launches as in a plan
        times, tot = pl.iterate_timed(args.steps, FLUSH_BYTES, split=False)
        torch.cuda.synchronize()
        # the FP32 roofline's denominator: an FMA-chain kernel on the same GPU and clocks
        fp32_peak = max(kpax.fp32_peak(1 << 16)[0] for _ in range(3))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = kpax.kernel_launches() - launches0
    t_s = float(times[:, 0].sum()) / 1000.0
    t_s, valid_all = combine_over_ranks(dist, "cuda", t_s, tot["valid"])
    value = valid_all / t_s
    # single-launch floor on the planner stream: a one-element fill between two events, queued
    # behind a sleep so that the host's launch time does not show
    one = torch.zeros(1, device="cuda")
    fl = []
    with torch.cuda.stream(stream):
        for _ in range(20):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda._sleep(200000)
            a.record(stream)
            one.fill_(1.0)
            b.record(stream)
            torch.cuda.synchronize()
            fl.append(a.elapsed_time(b))
    launch_floor_ms = float(np.median(fl[5:]))
    # latency floor of the expansion: the propagation kernel on 4096 independent segments (one warp
    # per SM), whose time is the dependency chain of its longest full-length segment
    seg_n = 4096
    seg_par = torch.from_numpy(E.sample_states(cfg.model, seg_n, 17)).cuda()
    seg_rows = torch.empty((seg_n, cfg.sample_dim), device="cuda")
    seg_valid = torch.empty(seg_n, dtype=torch.uint8, device="cuda")
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    def segment_floor(env) -> float:
        ts = []
        with torch.cuda.stream(stream):
            for i in range(8):
                flush.fill_(i & 0xFF)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                kpax.propagate_batch(cfg, env, seg_par.data_ptr(), None, 900 + i, seg_n, seg_rows.data_ptr(),
                                     seg_valid.data_ptr(), stream=stream.cuda_stream)
                b.record(stream)
                torch.cuda.synchronize()
                ts.append(a.elapsed_time(b))
        return float(np.median(ts[3:]))

    seg_env = kpax.Env(cfg, d_obs.data_ptr(), obs.shape[0])
    chain_floor_ms = segment_floor(seg_env)
    seg_env.close()
    # the same chain with no obstacles (every segment runs its steps; the grid queries find empty
    # cells): the share of the floor the obstacle tests take
    seg_env = kpax.Env(cfg, d_obs.data_ptr(), 0)
    chain_floor_empty_ms = segment_floor(seg_env)
    seg_env.close()
    del flush
    # the per-kernel breakdown from as many iterations with events between the kernels, on a new
    # plan grown the same way (the tree stays below its capacity)
    pl.begin(start, goal, d_obs.data_ptr(), obs.shape[0])
    pl.iterate_timed(8, 0)
    pl.iterate_timed(max(args.warmup, 3), FLUSH_BYTES)
    times_split, tot_split = pl.iterate_timed(args.steps, FLUSH_BYTES, split=True)
    t_exp = float(times_split[:, 2].sum()) / 1000.0

    # roofline of the expansion kernel: FP32 issue bound
    peaks = load_peaks()
    flops = tot_split["steps"] * FLOP_PER_STEP[cfg.model]
    achieved = flops / t_exp / 1e12
    sm_mhz = peaks.get("sm_max_mhz", 1965.0)
    nominal = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    roofline = {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                "traffic": ITERATE_DRAM_BYTES.get(cfg.model), "kernel": "k_iterate (its expansion phase)",
                "traffic_note": "DRAM bytes read + written by one steady-state k_iterate launch of this workload (the "
                                "whole fused iteration) in an ncu capture (summary under profiles/); after the L2 flush "
                                "only the first touches of the tree's repeat bytes and region ids, the regions and the "
                                "grid reach DRAM, the rest of what the kernel touches is L2-resident",
                "peak_note": "measured: kpax_fp32_peak (8 independent FMA chains per thread, 2048 threads per SM, "
                             "CUDA events) on this GPU inside the clock-sampling window; MEASURED_PEAKS.json has no "
                             "FP32 figure",
                "nominal_peak": nominal,
                "work": f"{tot_split['steps']} RK4 steps x {FLOP_PER_STEP[cfg.model]} FLOP over {args.steps} launches",
                "expand_ms_per_launch": 1000 * t_exp / args.steps,
                "latency_floor_ms": chain_floor_ms,
                "floor_note": "the propagation kernel on 4096 independent segments of the same model and scene (one warp "
                              "per SM): the dependency chain of one full-length segment, which bounds the expansion "
                              "kernel from below whatever its FP32 rate",
                "floor_frac": chain_floor_ms / (1000 * t_exp / args.steps),
                "latency_floor_no_obstacles_ms": chain_floor_empty_ms}

    # end to end: whole plans from host buffers through the C ABI
    e2e_v, e2e_t, tts, found = 0, 0.0, [], 0
    plans = args.plans
    h2d = obs.nbytes + 2 * 4 * cfg.sample_dim
    d2h = 0
    for i in range(plans):
        t0 = time.perf_counter()
        r = pl.plan_host(start, goal, obs)
        dt = time.perf_counter() - t0
        e2e_v += r.valid_expansions
        e2e_t += dt
        d2h += 4 * cfg.sample_dim * r.path_len + 128
        if r.found:
            found += 1
            tts.append(1000 * dt)
    e2e = {"value": e2e_v / e2e_t if e2e_t > 0 else None, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h // max(plans, 1),
           "plans": plans, "success_rate": found / max(plans, 1),
           "tts_ms_p50": float(np.percentile(tts, 50)) if tts else None,
           "tts_ms_p95": float(np.percentile(tts, 95)) if tts else None,
           "plan": f"the fixed start/goal pair of the workload, {cfg.max_iter} iterations or {cfg.max_tree_size} nodes "
                   "per plan; plan-level success and time to solution over seeded query sets are the learned and "
                   "batch workloads' figures"}

    if args.query_set > 0 and args.workload == "quad":
        qs = E.free_queries(obs, args.query_set, seed=5, min_sep=6.0, max_sep=15.0)
        e2e["query_set"] = query_outcomes(pl, qs, obs)
        e2e["query_set"]["queries_desc"] = (f"{args.query_set} seeded start/goal pairs in the free space of the same scene "
                                            "(>= 1 m from every box), 6-15 m apart; success = goal ball reached; "
                                            "time to solution = host clock of kpax_plan_host from host buffers")
    else:
        qs = np.zeros((0, 6), np.float32)

    clocks = clk.summary()
    ref_cuda = None
    if rank == 0 and ws == 1 and args.workload == "quad" and not args.no_ref_cuda:
        ref_cuda = reference_cuda_leg(cfg, obs, start, goal, qs, args)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        try:
            parents = frontier_parents(cfg, obs, start, goal)
            rate, cores, sample = cpu_reference_rate(cfg, obs, parents, args.cpu_seconds)
            cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample}
        except (FileNotFoundError, OSError) as exc:
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"unavailable: {exc}"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * t_s / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32", "data": "synthetic",
            "config": {"workload": desc, "expansions_per_iter": cfg.expansions_per_iter,
                       "launch": {"block_size": cfg.block_size or 448, "samples_per_thread": cfg.samples_per_thread or 1,
                                  "hash_cell_size": cfg.hash_cell_size,
                                  "source": "autotuner cache" if tuning else "defaults"},
                       "children_per_step": tot["children"] // args.steps,
                       "tree_nodes": [tree0, tree0 + tot["appended"]],  # at the first and after the last timed iteration
                       "l2": "flushed before each timed iteration "
                       "(256 MiB write, outside the events)", "parallelism": f"replicas x{ws}"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
            "reference_cuda": ref_cuda,
            "breakdown_ms_per_step": {"frontier": float(times_split[:, 1].mean()), "expand": float(times_split[:, 2].mean()),
                                      "scores": float(times_split[:, 3].mean()),
                                      "total_with_split_events": float(times_split[:, 0].mean()),
                                      "single_launch_floor": launch_floor_ms},
        }
        print(json.dumps(line), flush=True)
    pl.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def batch_configs(queries):
    """One configuration per batched query: its model's preset with the query's tree budget."""
    pre = {kpax.MODEL_DOUBLE_INTEGRATOR: kpax.PRESET_DI, kpax.MODEL_DUBINS_AIRPLANE: kpax.PRESET_DUBINS,
           kpax.MODEL_QUADROTOR: kpax.PRESET_QUAD}
    cfgs = []
    for q, d in enumerate(queries):
        c = kpax.preset(pre[d["model"]])
        c.max_tree_size = d["tree"]
        c.expansions_per_iter = min(c.expansions_per_iter, c.max_tree_size)
        c.seed = c.seed + 7919 * q
        cfgs.append(c)
    return cfgs


def run_segments(args) -> None:
    """2^22 independent Dubins segments per step through kpax_propagate_batch (device Philox draws)."""
    import torch

    ws, rank, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    n = 1 << args.segments_log2
    cfg, obs, parents = segment_inputs(n, 5 + rank)
    S = cfg.sample_dim
    d_obs = torch.from_numpy(obs).cuda()
    env = kpax.Env(cfg, d_obs.data_ptr(), obs.shape[0])
    d_par = torch.from_numpy(parents).cuda()
    rows = torch.empty((n, S), dtype=torch.float32, device="cuda")
    valid = torch.empty(n, dtype=torch.uint8, device="cuda")
    steps = torch.empty(n, dtype=torch.int32, device="cuda")
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    def launch(i):
        if args.one_pass:  # the allocation-free entry: one pass over every segment at any batch size
            kpax.propagate_batch_noalloc(cfg, d_obs.data_ptr(), obs.shape[0], d_par.data_ptr(), None, i, n, rows.data_ptr(),
                                         valid.data_ptr(), steps.data_ptr(), stream=stream.cuda_stream)
        else:
            kpax.propagate_batch(cfg, env, d_par.data_ptr(), None, i, n, rows.data_ptr(), valid.data_ptr(), steps.data_ptr(),
                                 stream=stream.cuda_stream)

    for i in range(max(args.warmup, 3)):
        launch(1000 + i)
    launches0 = kpax.kernel_launches()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    n_valid, n_steps = 0, 0
    with Clocks(local) as clk:
        for i in range(args.steps):
            flush.fill_(i & 0xFF)  # evict the 126 MB L2 between steps, outside the events
            ev[i][0].record(stream)
            launch(i)
            ev[i][1].record(stream)
            n_valid += valid.sum(dtype=torch.int64)  # device-side tallies, outside the events
            n_steps += steps.sum(dtype=torch.int64)
        torch.cuda.synchronize()
        fp32_peak = max(kpax.fp32_peak(1 << 16)[0] for _ in range(3))  # the same GPU and clocks
    if dist:
        dist.barrier()
    launches = kpax.kernel_launches() - launches0
    t_s = sum(a.elapsed_time(b) for a, b in ev) / 1000.0
    n_valid, n_steps = int(n_valid.item()), int(n_steps.item())
    t_job, valid_all = combine_over_ranks(dist, "cuda", t_s, n_valid)
    value = valid_all / t_job

    peaks = load_peaks()
    sm_mhz = peaks.get("sm_max_mhz", 1965.0)
    phased = n >= 1 << 18 and not args.one_pass
    achieved = n_steps * FLOP_PER_STEP[cfg.model] / t_s / 1e12
    roofline = {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                "traffic": int(PHASED_DRAM_BYTES_PER_SEGMENT * n) if phased
                           else int(ONE_PASS_DRAM_BYTES_PER_SEGMENT * n) if args.one_pass else None,
                "traffic_note": ("DRAM bytes read + written per step by the three phase kernels, from an ncu capture of "
                                 "2^20 segments scaled to the segment count (summary under profiles/); "
                                 "the algorithmic bytes are 69 per segment (parent 24, row 40, verdict 1, steps 4), the "
                                 "rest is the survivors' round trips and partial-sector fills of rows written out of order")
                                if phased else
                                ("DRAM bytes read + written per step by the one-pass kernel, from an ncu capture of 2^20 "
                                 "segments scaled to the segment count (summary under profiles/): 70.2 B per segment "
                                 "against 69 algorithmic"),
                "kernel": "k_propagate_head + 2 x k_propagate_tail<Dubins> (phased batch)" if phased
                          else "k_propagate_batch<Dubins>",
                "peak_note": "measured: kpax_fp32_peak (FMA chains, CUDA events) on this GPU inside the clock-sampling "
                             "window; MEASURED_PEAKS.json has no FP32 figure; plus 12 transcendental per step on the MUFU "
                             "pipe",
                "nominal_peak": 148 * 128 * 2 * sm_mhz * 1e6 / 1e12,
                "work": f"{n_steps} RK4 steps x {FLOP_PER_STEP[cfg.model]} FLOP over {args.steps} launches",
                "ms_per_launch": 1000 * t_s / args.steps, "rk4_steps_per_s": n_steps / t_s}

    # end to end through the C ABI from pinned host buffers: parents in, rows and verdicts out
    h_par = torch.from_numpy(parents).pin_memory()
    h_rows = torch.empty((n, S), dtype=torch.float32).pin_memory()
    h_valid = torch.empty(n, dtype=torch.uint8).pin_memory()
    e2e_steps = max(2, min(args.steps, 5))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_valid = torch.zeros((), dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    e0.record(stream)
    for i in range(e2e_steps):
        d_par.copy_(h_par, non_blocking=True)
        launch(500 + i)
        h_rows.copy_(rows, non_blocking=True)
        h_valid.copy_(valid, non_blocking=True)
        e2e_valid += valid.sum(dtype=torch.int64)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_t = e0.elapsed_time(e1) / 1000.0
    e2e_valid = int(e2e_valid.item())
    e2e = {"value": e2e_valid / e2e_t, "unit": UNIT, "h2d_bytes_per_step": int(h_par.numel() * 4),
           "d2h_bytes_per_step": int(h_rows.numel() * 4 + h_valid.numel())}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        try:
            rate, cores, sample, _ = cpu_segments_rate(args.cpu_seconds)
            cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample}
        except (FileNotFoundError, OSError) as exc:
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"unavailable: {exc}"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * t_job / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32", "data": "synthetic",
            "config": {"workload": SEGMENTS_DESC if n == 1 << 22 else SEGMENTS_DESC.replace("2^22", f"2^{args.segments_log2}"),
                       "segments_per_step": n, "valid_fraction": n_valid / (n * args.steps),
                       "entry": "kpax_propagate_batch_noalloc (one pass)" if args.one_pass else "kpax_propagate_batch",
                       "l2": "flushed before each timed step (256 MiB write, outside the events)",
                       "parallelism": f"replicas x{ws}"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_batch(args) -> None:
    """Many independent queries per launch: each step plans the whole batch once."""
    import torch

    ws, rank, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    queries = E.batch_queries(args.queries, seed=4 + 1000 * rank)
    cfgs = batch_configs(queries)
    if args.batch_iters:  # solvability study: more iterations per query than the presets' 300
        for c in cfgs:
            c.max_iter = args.batch_iters
    tuned_models = {}
    if not args.no_tune:  # per model: the cached parameters of its single-query workload
        import kpax_autotune

        for name, m in (("quad", kpax.MODEL_QUADROTOR), ("dubins", kpax.MODEL_DUBINS_AIRPLANE),
                        ("di", kpax.MODEL_DOUBLE_INTEGRATOR)):
            pre, scene, _ = WORKLOADS[name]
            _, best = kpax_autotune.tuned(kpax.preset(pre), scene()[0].shape[0])
            if best:
                tuned_models[m] = best
        cfgs = [kpax_autotune.apply(c, tuned_models[c.model]) if c.model in tuned_models else c for c in cfgs]
    # children per expansion tile of every query: a batch expands millions of children per
    # iteration, where the batch expansion's 256-child tiles at four or five CTAs per SM hide more
    # latency than the single 14-warp CTA the single-query tuning picks
    if args.batch_block:
        for c in cfgs:
            c.block_size = args.batch_block
    sizes = [d["obstacles"].shape[0] for d in queries]
    offs = np.concatenate([[0], np.cumsum(sizes)])
    h_obs = torch.from_numpy(np.concatenate([d["obstacles"] for d in queries])).pin_memory()
    d_obs = torch.empty_like(h_obs, device="cuda")
    ptrs = [d_obs.data_ptr() + 24 * int(o) for o in offs[:-1]]
    starts, goals = [d["start"] for d in queries], [d["goal"] for d in queries]
    batch = kpax.Batch(cfgs)
    net = None
    if args.proposal == "on":
        import kpax_learn as L

        net = L.load_network(L.DEFAULT_WEIGHTS)
        batch.set_proposal(net, args.eps)
    d_obs.copy_(h_obs)
    for _ in range(args.warmup):
        batch.plan(starts, goals, ptrs, sizes)
    launches0 = kpax.kernel_launches()
    tot_ms, tot_valid, wall, tts, found, n_plans = 0.0, 0, 0.0, [], 0, 0
    per_model = {m: [0, 0, 0] for m in (1, 2, 3)}  # plans, solved, trees filled before the goal
    with Clocks(local) as clk:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            d_obs.copy_(h_obs, non_blocking=True)  # host -> device inside the timed region
            res, st = batch.plan(starts, goals, ptrs, sizes)
            wall += time.perf_counter() - t0
            tot_ms += st["ms"]
            tot_valid += st["valid_expansions"]
            n_plans += len(res)
            for d, r in zip(queries, res):
                per_model[d["model"]][0] += 1
                per_model[d["model"]][2] += int(bool(r["tree_full"]) and not r["found"])
                if r["found"]:
                    found += 1
                    per_model[d["model"]][1] += 1
                    tts.append(r["ms"])
    launches = kpax.kernel_launches() - launches0
    batch.close()
    value = tot_valid / (tot_ms / 1000.0)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tot_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32", "data": "synthetic",
        "config": {"workload": f"batched: {args.queries} queries, 40/30/30 % double integrator / Dubins / quadrotor, "
                               "obstacles log-U[10,5000], trees log-U[2^14,2^20], start/goal >= 50 apart, one launch per "
                               "stage for all queries", "l2": "each step is a whole batch plan (~GB working set)",
                   "learned_proposal": f"quadrotor queries, epsilon {args.eps}" if net is not None else "off",
                   "launch": {str(m): v for m, v in tuned_models.items()} or "defaults",
                   "expansion_block": args.batch_block or "as launch",  # overrides launch's block_size
                   "parallelism": f"replicas x{ws}"},
        "plans_per_s": n_plans / (tot_ms / 1000.0),
        "success_rate": found / max(n_plans, 1),
        "success_by_model": {{1: "double_integrator", 2: "dubins", 3: "quadrotor"}[m]: v[1] / max(v[0], 1)
                             for m, v in per_model.items()},
        "tree_filled_unsolved_by_model": {{1: "double_integrator", 2: "dubins", 3: "quadrotor"}[m]: v[2] / max(v[0], 1)
                                          for m, v in per_model.items()},
        "iterations_per_query": args.batch_iters or "presets' 300",
        "tts_ms_p50": float(np.percentile(tts, 50)) if tts else None,
        "tts_ms_p95": float(np.percentile(tts, 95)) if tts else None,
        "e2e": {"value": tot_valid / wall, "unit": UNIT, "h2d_bytes_per_step": int(h_obs.numel() * 4),
                "d2h_bytes_per_step": 128 * args.queries},
        "gpu_launches": launches, "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_learned(args) -> None:
    """Learned proposal on the 12D quadrotor: the shipped network (trained on the GPU by the
    library's kernels) against the plain uniform sampler on held-out scenes of the learned
    family, with the same random streams; plus the tensor-core proposal pass and the training
    step measured on their own."""
    import torch

    import kpax_learn as L

    ws, rank, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    cfg = L.quad_config()
    w, meta = L.load_params(L.DEFAULT_WEIGHTS)
    net = kpax.MLP(max_batch=4096)
    net.set_params(w)
    seeds = [L.EVAL_SEED0 + 1_000_000 * rank + i for i in range(args.seeds)]
    L.evaluate(seeds[:2], cfg), L.evaluate(seeds[:2], cfg, net, args.eps)  # warm-up
    launches0 = kpax.kernel_launches()
    with Clocks(local) as clk:
        t0 = time.perf_counter()
        plain = L.evaluate(seeds, cfg, progress=True)
        t1 = time.perf_counter()
        learned = L.evaluate(seeds, cfg, net, args.eps, progress=True)
        t2 = time.perf_counter()
    launches = kpax.kernel_launches() - launches0
    sp, sl = L.summarize(plain), L.summarize(learned)
    # the metric at >= 95 % success: the same seeds on a family whose goals lie within the trees'
    # reach (start and goal 6-12 m apart, 100-300 boxes)
    near = {"obs_range": (100, 300), "min_sep": 6.0, "max_sep": 12.0}
    np_ = L.summarize(L.evaluate(seeds, cfg, family=near))
    nl_ = L.summarize(L.evaluate(seeds, cfg, net, args.eps, family=near))
    at95 = {"family": "building scenes of 100-300 AABBs, start/goal 6-12 m apart", "plain": np_, "learned": nl_,
            "both_at_95": bool(np_["success"] >= 0.95 and nl_["success"] >= 0.95),
            "p50_ratio_learned_to_plain": nl_["p50_ms"] / np_["p50_ms"] if np_["p50_ms"] > 0 else None,
            "mean_ratio_learned_to_plain": nl_["mean_ms"] / np_["mean_ms"] if np_["mean_ms"] > 0 else None}
    # tensor-core proposal pass: 2^16 frontier entries (the quadrotor budget), device-timed
    obs, start, goal = E.learned_family(seeds[0])
    d_obs = torch.from_numpy(obs).cuda()
    env = kpax.Env(cfg, d_obs.data_ptr(), obs.shape[0])
    n = 1 << 16
    g = torch.Generator(device="cuda").manual_seed(0)
    st = (torch.rand((n, 12), device="cuda", generator=g) * 100).contiguous()
    go = (torch.rand((n, 3), device="cuda", generator=g) * 100).contiguous()
    mix = torch.zeros((n, kpax.MLP_MIX), device="cuda")
    for _ in range(3):
        net.propose(env, st.data_ptr(), 12, go.data_ptr(), n, mix.data_ptr())
    ms = []
    for _ in range(max(args.steps, 5)):
        net.propose(env, st.data_ptr(), 12, go.data_ptr(), n, mix.data_ptr())
        ms.append(net.last_propose_ms())
    prop_ms = statistics.mean(ms)
    flop = n * 202240
    peaks = load_peaks()
    peak_tf = float(peaks.get("bf16_tflops", 1590.0))
    # training step: batch 4096, FP32 kernels (forward + backward ~ 3x the forward's FLOP)
    X = torch.randn((1 << 16, kpax.MLP_FEATURES), device="cuda", generator=g)
    Y = torch.randn((1 << 16, 5), device="cuda", generator=g)
    idx = torch.randint(0, 1 << 16, (4096,), device="cuda", dtype=torch.int32, generator=g)
    tnet = kpax.MLP(max_batch=4096)
    tnet.set_params(L.init_params(1))
    for _ in range(5):
        tnet.train_step(X.data_ptr(), Y.data_ptr(), idx.data_ptr(), 4096, 1e-4)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(50):
        tnet.train_step(X.data_ptr(), Y.data_ptr(), idx.data_ptr(), 4096, 1e-4)
    e1.record()
    torch.cuda.synchronize()
    train_ms = e0.elapsed_time(e1) / 50
    line = {
        "metric": "p50 time-to-solution of solved plans, learned proposal (quadrotor)", "value": sl["p50_ms_solved"],
        "unit": "ms", "n_gpus": ws, "steps": len(seeds), "warmup": 2, "ms_per_step": (t2 - t1) * 1e3 / len(seeds),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "bf16 inference / fp32 training",
        "data": "synthetic",
        "config": {"workload": f"learned proposal: {len(seeds)} held-out building scenes (200-2000 AABBs incl. windowed "
                               "wall), start/goal 25-45 m apart, 12D quadrotor preset (2^16 expansions/iteration, 2^20 "
                               f"nodes, 300 iterations), epsilon {args.eps}", "parallelism": f"replicas x{ws}",
                   "network": "51-256-256-88 SiLU, 8-component mixture", "training": meta},
        "plain": sp, "learned": sl,
        "success_gain": sl["success"] - sp["success"],
        "at_95_success": at95,
        "proposal_pass": {"rows": n, "ms": prop_ms, "tflops": flop / (prop_ms * 1e-3) / 1e12},
        "roofline": {"bound": "tensor", "achieved": flop / (prop_ms * 1e-3) / 1e12, "peak": peak_tf, "unit": "TFLOP/s",
                     "frac": flop / (prop_ms * 1e-3) / 1e12 / peak_tf, "traffic": None,
                     "kernel": "k_forward_tc (tensor-core proposal pass, 202240 FLOP per row)",
                     "peak_source": "measured bf16 burst" if "fallback" not in peaks else "fallback"},
        "training_step": {"batch": 4096, "ms": train_ms, "samples_per_s": 4096 / (train_ms * 1e-3),
                          "tflops": 3 * 202240 * 4096 / (train_ms * 1e-3) / 1e12},
        "e2e": {"value": len(seeds) / (t2 - t1), "unit": "plans/s (learned arm, wall clock, obstacles copied per plan)",
                "h2d_bytes_per_step": int(np.mean([E.learned_family(s)[0].nbytes for s in seeds[:8]])),
                "d2h_bytes_per_step": 0},
        "plain_plans_per_s_wall": len(seeds) / (t1 - t0),
        "gpu_launches": launches, "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_expansion_scan(args) -> None:
    """Phase times of the fused quadrotor iteration against the children per iteration, in the building
    scene and with no obstacles, at the default expansion block (the pair layout: two warps per 32
    children) and at 128-child blocks (one thread per child).  With 448 children per block the
    expansion's CTAs each hold the same load whatever the budget (only their number changes), so a
    flat expansion time says that the per-SM chain, not anything shared between SMs, sets it; the
    empty scene bounds what any staging of the obstacle lists could save."""
    import torch

    torch.cuda.set_device(0)
    obs, start, goal = E.quad_scene()
    scan = []
    for scene, o in (("building", obs), ("empty", np.zeros((0, 6), np.float32))):
        d_obs = torch.from_numpy(o).cuda() if o.size else torch.zeros(6, device="cuda")
        for bs in (448, 128):
            for budget in (148 * 32, 148 * 32 * 4, 1 << 15, 1 << 16):
                cfg = kpax.preset(kpax.PRESET_QUAD)
                cfg.hash_cell_size, cfg.block_size, cfg.expansions_per_iter = 2.5, bs, budget
                pl = kpax.KPAX(cfg)
                pl.begin(start, goal, d_obs.data_ptr(), o.shape[0])
                pl.iterate_timed(8, 0)
                pl.iterate_timed(max(args.warmup, 3), FLUSH_BYTES)
                times, tot = pl.iterate_timed(args.steps, FLUSH_BYTES, split=True)
                scan.append({"scene": scene, "block_children": bs, "budget": budget,
                             "iteration_ms": float(times[:, 0].mean()), "frontier_ms": float(times[:, 1].mean()),
                             "expansion_ms": float(times[:, 2].mean()), "scores_ms": float(times[:, 3].mean()),
                             "children_per_iter": tot["children"] / args.steps,
                             "steps_per_child": tot["steps"] / max(tot["children"], 1)})
                pl.close()
    print(json.dumps({"metric": "expansion phase time", "unit": "ms", "higher_is_better": False, "n_gpus": 1,
                      "steps": args.steps, "warmup": args.warmup, "data": "synthetic",
                      "config": {"workload": "fused quadrotor iteration, budget scan: " + WORKLOADS["quad"][2],
                                 "l2": "flushed before each timed iteration"},
                      "scan": scan}), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["batch", "learned", "segments", "collide", "quad-ref",
                                                               "expansion-scan"],
                    default="quad")
    ap.add_argument("--plans-ref", type=int, default=256, help="plans per side of the quad-ref workload")
    ap.add_argument("--plans-ref-big", type=int, default=32, help="plans per side at the 2^22 tree capacity (quad-ref)")
    ap.add_argument("--batch-iters", type=int, default=0, help="iteration cap of every batched query (0 = presets)")
    ap.add_argument("--batch-block", type=int, default=256, choices=[0, 128, 256, 448, 512],
                    help="children per expansion tile of every batched query (0 = the single-query tuning / "
                         "presets; 256 measured fastest for batches: four or five CTAs per SM)")
    ap.add_argument("--seeds", type=int, default=256, help="held-out scenes of the learned workload")
    ap.add_argument("--eps", type=float, default=0.2, help="uniform fraction of the learned proposal")
    ap.add_argument("--proposal", choices=["on", "off"], default="on", help="learned proposal for batched quadrotor queries")
    ap.add_argument("--queries", type=int, default=1024)
    ap.add_argument("--plans", type=int, default=8)
    ap.add_argument("--query-set", type=int, default=32, help="seeded start/goal pairs of the e2e query set (quad)")
    ap.add_argument("--ref-cuda-plans", type=int, default=3, help="plans of the reference CUDA leg (quad)")
    ap.add_argument("--no-ref-cuda", action="store_true", help="skip the reference CUDA build's leg")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="ignore the autotuner's cached launch parameters")
    ap.add_argument("--segments-log2", type=int, default=22, help="segments per step of the segments workload (log2)")
    ap.add_argument("--one-pass", action="store_true",
                    help="segments workload through the allocation-free entry (one pass at any size, no phases)")
    ap.add_argument("--boxes-log2", type=int, default=22, help="box queries per step of the collide workload (log2)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "learned":
        run_learned(args)
    elif args.workload == "segments":
        run_segments(args)
    elif args.workload == "collide":
        run_collide(args)
    elif args.workload == "quad-ref":
        run_quad_ref(args)
    elif args.workload == "expansion-scan":
        run_expansion_scan(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
