#!/usr/bin/env python3
"""Benchmark: batched uneven pRRTC planning on B200.

Workload (one "step"): 512 planning problems for the synthetic 7-DOF arm, each
with its own world (4-128 spheres, 0-32 boxes) and 1-8 goals, tree capacity
4096 / 16384 / 65536 nodes by world size; every problem is solved once per
step by the persistent batched planner, all problems in one launch with
per-problem capacities (one captured CUDA graph; --launch buckets: one graph
per capacity on concurrent streams), settings chosen by the autotuner
(--tuning fixes them).  Problems are seeded synthetic stand-ins for the
reference's MBM sets.

  value  plans/s with inputs resident in HBM (graph replays, CUDA events,
         L2 flushed between steps)
  e2e    plans/s through the public API prrtc_plan_batch_async + results()
         with host inputs: host->device copies and the device->host read of
         results and paths inside the timed region, up to three calls in
         flight; at N GPUs every rank runs it and the slowest rank's time counts

Also reported (rank 0): the plain per-problem-launch form on the same GPU
(the reference's batch structure) with its p50 device solve ms, collision
checks/s of the planner and of the standalone FK+collision kernel,
nearest-neighbour GB/s, the smoothing adjoint's waypoint gradients/s, each
kernel's roofline fraction, and the CPU baseline (the reference's
host-driven RRT-Connect loop restated in C, timed on this host).

Multi-GPU (torchrun): weak scaling -- every rank solves its own 512 problems
(seeds offset by rank); no data-path collective; value = all ranks' solved
plans / max over ranks of the timed seconds.

--impl reference: the reference's CPU path (its host-driven RRT-Connect loop,
restated in C by the oracle since JAX and PyRoFFI are absent), on all host
cores, over a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import gc
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
sys.path.insert(0, str(ROOT))

N_PROBLEMS = 512
WORKLOAD = ("uneven512: 512 problems, synthetic 7-DOF arm (56 spheres, 960 self pairs), per-problem world "
            "4-128 spheres + 0-32 boxes, 1-8 goals, max_nodes buckets 4096/16384/65536")
METRIC = "plans/s (batched uneven 512-problem workload)"


def workload_config(problems) -> dict:
    """The workload both arms run (their `config`); each arm's own settings go
    under `arm`."""
    buckets: dict = {}
    for p in problems:
        buckets[str(int(p.max_nodes))] = buckets.get(str(int(p.max_nodes)), 0) + 1
    return {"workload": WORKLOAD, "problems_per_gpu": len(problems),
            "buckets": dict(sorted(buckets.items(), key=lambda kv: -int(kv[0])))}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--problems", type=int, default=N_PROBLEMS)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="budget of the CPU-baseline sample")
    ap.add_argument("--no-extras", action="store_true", help="skip the plain-launch / CC / NN side measurements")
    ap.add_argument("--eager", action="store_true", help="launch every step eagerly instead of replaying graphs")
    ap.add_argument("--launch", choices=["merged", "buckets"], default="merged",
                    help="one launch for every problem with per-problem tree capacities (merged), or one "
                         "launch per capacity bucket on concurrent streams (buckets)")
    ap.add_argument("--tune", choices=["joint", "bucket"], default="bucket",
                    help="with --launch buckets: explorer counts tuned per bucket alone (default; measured 144 K "
                         "vs 139-143 K plans/s) or with the buckets running together (joint)")
    ap.add_argument("--tuning", default=None, metavar="E,T,CW[,R]",
                    help="skip the autotuner: explorers per problem, threads per explorer, waypoints per chunk, "
                         "CTAs per SM (0: as many as fit)")
    ap.add_argument("--kernel", choices=["cc", "checkers", "nn", "smooth"], default=None,
                    help="run only the standalone FK+collision (cc), per-checker (checkers), nearest-neighbour (nn) or "
                         "smoothing adjoint (smooth) measurement")
    ap.add_argument("--configs", default="1,2,4,5,dense",
                    help="comma list of the extra workloads to measure on rank 0 after the headline: 1 (single plan, "
                         "GPU and CPU path), 2 (1000 tabletop plans), 4 (smoothing of the tabletop paths), 5 (1024 "
                         "dual-arm plans + smoothing), dense (the 512-problem batch at the 16-sphere scene's "
                         "density); 'none' skips them")
    ap.add_argument("--split", choices=["weak", "strong"], default="weak",
                    help="multi-GPU: every rank solves its own batch (weak) or one batch is split across ranks by "
                         "longest-processing-time on estimated cost (strong)")
    ap.add_argument("--config5-problems", type=int, default=1024)
    ap.add_argument("--config2-problems", type=int, default=1000)
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ----------------------------------------------------------------------------- workload

def make_workload(n, rank, checker, split="weak", world=1):
    """The uneven batch of `n` problems: rank r's own seeds (weak scaling), or
    rank r's longest-processing-time share of one common batch (strong), the
    cost of a problem estimated by its collision work times its tree capacity."""
    from prrtc_b200 import scenes
    from prrtc_b200.shard import lpt_partition

    robot = scenes.arm(0)
    if split == "weak":
        return [scenes.make_problem("uneven", 100000 * (rank + 1) + i, checker, robot=robot) for i in range(n)]
    allp = [scenes.make_problem("uneven", 100000 + i, checker, robot=robot) for i in range(n)]
    return [allp[i] for i in lpt_partition([problem_cost(p) for p in allp], world)[rank]]


def problem_cost(p):
    c = p.context
    work = sum(w * (0 if c.get(k) is None else len(c[k])) for k, w in (
        ("world_spheres", 1.0), ("world_capsules", 2.0), ("world_boxes", 3.0), ("world_halfspaces", 1.0)))
    return (1.0 + work) * p.max_nodes / 4096.0


def oracle_checker(configs, ctx):
    from oracle import oracle as O

    return O.Scene(ctx, np.asarray(configs).shape[1]).check_configs(configs, 0)


# ----------------------------------------------------------------------------- clocks

class ClockSampler:
    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "100"], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------------------------- CPU baseline

def _cpu_solve(args):
    import numpy as _np
    from oracle import oracle as O

    ctx, dim, start, goals, lo, hi, seed = args
    sc = O.Scene(ctx, dim)
    r = O.rrtc_host_plan(sc, start, goals, lo, hi, max_iterations=1000, step_size=0.5, num_new_samples=128,
                         granularity=16, max_nodes=65536, connect_max_steps=32, seed=seed, collision_mode=0)
    return bool(r.solved), int(r.config_checks)


def cpu_baseline(problems, seconds, processes):
    """Solve problems in order until the budget is spent; plans/s over the solved sample."""
    import multiprocessing as mp

    args = [(p.context, p.dim, p.start, p.goals, p.lower, p.upper, i) for i, p in enumerate(problems)]
    t0 = time.perf_counter()
    solved = done = checks = 0
    if processes <= 1:
        for a in args:
            s, c = _cpu_solve(a)
            solved += s
            done += 1
            checks += c
            if time.perf_counter() - t0 > seconds:
                break
    else:
        ctx = mp.get_context("spawn")
        with ctx.Pool(processes) as pool:
            for s, c in pool.imap(_cpu_solve, args, chunksize=1):
                solved += s
                done += 1
                checks += c
                if time.perf_counter() - t0 > seconds:
                    pool.terminate()
                    break
    dt = time.perf_counter() - t0
    return {"solved": solved, "done": done, "seconds": dt, "plans_per_s": solved / dt, "checks_per_s": checks / dt}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ----------------------------------------------------------------------------- reference arm

def run_reference(a):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import oracle as O

    O.build()
    problems = make_workload(a.problems, 0, oracle_checker)
    procs = O.cpu_count()
    per_step = []
    sample = min(len(problems), 96)
    for i in range(a.warmup + a.steps):
        st = cpu_baseline(problems[(i * sample) % len(problems):][:sample], a.cpu_seconds, procs)
        if i >= a.warmup:
            per_step.append(st)
    solved = sum(s["solved"] for s in per_step)
    secs = sum(s["seconds"] for s in per_step)
    value = solved / secs if secs > 0 else 0.0
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "plans/s", "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * secs / max(1, len(per_step)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(problems),
        "arm": {"sample_per_step": sample, "parallelism": f"{procs} host processes",
                "planner": "host-driven RRT-Connect (its defaults: binary checker, 16 waypoints per edge, "
                           "128 samples per iteration, 1000 iterations, 65536 nodes)"},
        "cpu_baseline": {"value": value, "unit": "plans/s", "cores": procs, "kind": "port",
                         "sample": f"<= {sample} problems per step (budget {a.cpu_seconds:.0f} s), host-driven "
                                   f"RRT-Connect restated in C (prrtc_robogpu.py:103-298), {cpu_model()}"},
        "e2e": {"value": value, "unit": "plans/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "success_rate": sum(s["solved"] for s in per_step) / max(1, sum(s["done"] for s in per_step)),
    }
    print(json.dumps(line))
    return 0


# ----------------------------------------------------------------------------- our arm

def fp32_probe_rates(torch, lib, dev):
    """FP32 FMA throughput of the two probes: scalar FFMA chains and packed
    fma.rn.f32x2 chains (TFLOP/s, best of five launches each)."""
    from prrtc_b200 import _lib as L

    sm = torch.cuda.get_device_properties(dev).multi_processor_count
    sink = torch.zeros(sm * 8, device=dev)
    blocks, threads, iters = sm * 8, 256, 4096
    s = torch.cuda.current_stream().cuda_stream
    rates = {}
    for name, fn, per_iter in (("ffma", lib.prrtc_b200_fp32_probe, 2.0 * 8 * 16),
                               ("ffma2", lib.prrtc_b200_fp32x2_probe, 4.0 * 8 * 16)):
        L.check(fn(blocks, threads, 64, sink.data_ptr(), s), "probe")
        torch.cuda.synchronize()
        best = 0.0
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            L.check(fn(blocks, threads, iters, sink.data_ptr(), s), "probe")
            e1.record()
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            best = max(best, per_iter * iters * blocks * threads / (ms * 1e-3) / 1e12)
        rates[name] = best
    return rates


def fp32_peak_tflops(torch, lib, dev):
    """FP32 roofline denominator: the faster of the scalar and packed FMA probes."""
    return max(fp32_probe_rates(torch, lib, dev).values())


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except json.JSONDecodeError:
            pass
    return {"hbm_gbs": 6650.0, "_fallback": True}


def run_ours(a):
    import torch
    import torch.distributed as dist

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        dist.init_process_group("nccl", init_method="env://", device_id=dev,
                                timeout=__import__("datetime").timedelta(seconds=120))

    from prrtc_b200 import _lib, build
    from prrtc_b200.batch import STAT_CONFIGS, STAT_EDGES, STAT_FLOPS, STAT_NN_NODES, BatchPlanner, PlanSettings, bucket_problems
    from prrtc_b200.collision import CollisionChecker, gpu_checker
    from prrtc_b200.prrtc import prrtc_plan_batch

    build.build()
    lib = _lib.load()
    problems = make_workload(a.problems, rank, gpu_checker(dev), a.split, ws)
    settings = PlanSettings()
    from prrtc_b200.autotune import choose, choose_joint

    buckets = bucket_problems(problems)
    if a.launch == "merged":
        # every problem in one launch and one work queue (tail join reaches all
        # of them), each tree bounded by its own bucket's capacity
        groups = {"all": problems}
        cap_of = {"all": [p.max_nodes for p in problems]}
    else:
        groups = dict(buckets)
        cap_of = {N: N for N in buckets}
    if a.tuning:
        v_ = [int(x) for x in a.tuning.split(",")] + [0]
        tuned = {k: {"num_new_samples": v_[0], "threads_per_explorer": v_[1], "waypoint_chunk": v_[2],
                     "ctas_per_sm": v_[3]} for k in groups}
    else:
        tuned = {k: choose(ps, cap_of[k], settings, dev) for k, ps in groups.items()}
    # optional: settle the explorer counts with the buckets running together
    if a.tune == "joint" and a.launch == "buckets":
        tuned = choose_joint(buckets, tuned, settings, dev)
    planners = {}
    for k, ps in groups.items():
        s = PlanSettings(**{**settings.__dict__, **tuned[k]})
        planners[k] = BatchPlanner(ps, cap_of[k], s, dev)
    flush = torch.empty(int(256 * 2**20) // 4, dtype=torch.float32, device=dev)
    # the workload (512 contexts of numpy tables) and the planners live for the
    # whole run: move them out of the collector's generations, as a long-running
    # planning service does after start-up, so that a full collection during the
    # end-to-end leg does not walk them
    gc.collect()
    gc.freeze()
    # buckets run concurrently, one stream each, so one bucket's tail overlaps the others
    streams = [torch.cuda.Stream(device=dev) for _ in planners]
    fork = torch.cuda.Event()

    def step():
        main = torch.cuda.current_stream()
        fork.record(main)
        for st, pl in zip(streams, planners.values()):
            st.wait_event(fork)
            with torch.cuda.stream(st):
                pl.run()
        for st in streams:
            main.wait_stream(st)

    # warm-up: first eager (validates), then capture one graph per planner (one
    # planner for all problems by default, one per bucket with --launch buckets)
    for i in range(max(a.warmup, 1)):
        if i == 1 and not a.eager:
            for pl in planners.values():
                pl.capture()
        step()
    if not a.eager and all(pl.graph is None for pl in planners.values()):
        for pl in planners.values():
            pl.capture()
        step()
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()

    # ---- timed region ----
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    solved_total = 0
    solved_host = []
    with ClockSampler(local) as clk:
        time.sleep(0.5)  # let the sampler start before the timed region
        torch.cuda.synchronize()
        torch.cuda.profiler.start()  # ncu --profile-from-start off captures the timed steps only
        for k in range(a.steps):
            flush.fill_(float(k))  # evict L2 (256 MB > 126 MB) outside the timed events
            starts[k].record()
            step()
            ends[k].record()
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
    if ws > 1:
        dist.barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    for pl in planners.values():
        blk = pl.summary_block().cpu().numpy()
        solved_host.append(blk)
        solved_total += int((blk[:, 8] == 1).sum())
    total_s = sum(step_ms) / 1e3
    t = torch.tensor([total_s, float(solved_total * a.steps)], dtype=torch.float64, device=dev)
    if ws > 1:
        tmax = t[:1].clone()
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
        tsum = t[1:].clone()
        dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
        total_s, all_solved = float(tmax.item()), float(tsum.item())
    else:
        all_solved = float(solved_total * a.steps)
    value = all_solved / total_s
    blk = np.concatenate(solved_host, 0)
    solved_mask = blk[:, 8] == 1
    solve_ms = blk[:, 9].copy().view(np.float32)[solved_mask]
    success = float(solved_mask.mean())

    line = {
        "metric": METRIC, "value": value, "unit": "plans/s", "n_gpus": ws, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": float(np.mean(step_ms)), "higher_is_better": True, "scaling": a.split,
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(problems),
        "arm": {"tuned": {str(N): v for N, v in tuned.items()},
                "collision_checker": settings.collision_checker, "edge_resolution": settings.edge_resolution,
                "l2": "flushed (256 MB write) between steps", "gc": "workload frozen (gc.freeze) after set-up",
                "launch": ("eager" if a.eager else "CUDA graph replay") + (
                    ", one launch for all problems with per-problem tree capacities" if a.launch == "merged"
                    else ", one launch per capacity bucket on concurrent streams"),
                "parallelism": (f"weak scaling, {ws} rank(s), every rank its own {len(problems)} problems"
                                if a.split == "weak" else
                                f"strong scaling, {ws} rank(s), one {a.problems}-problem batch split by "
                                "longest-processing-time on estimated cost")},
        "success_rate": success,
        "p50_solve_ms": float(np.median(solve_ms)) if solve_ms.size else None,
    }
    # per planner: fill, pack, init, explore, finalize, path extraction, result block
    line["gpu_launches"] = 7 * len(planners) * a.steps

    # e2e on every rank (each its own problems), whole job = all ranks' plans
    # over the slowest rank's seconds
    if not a.no_extras:
        if ws > 1:
            dist.barrier()
        e_solved, e_s, e_h2d, e_d2h, e_steps, e_diag = measure_e2e(torch, dev, planners, settings, tuned, cap_of,
                                                                    a.steps)
        if ws > 1:
            v = torch.tensor([e_s, float(e_solved), float(e_h2d), float(e_d2h)], dtype=torch.float64, device=dev)
            vmax = v[:1].clone()
            dist.all_reduce(vmax, op=dist.ReduceOp.MAX)
            vsum = v[1:].clone()
            dist.all_reduce(vsum, op=dist.ReduceOp.SUM)
            e_s, e_solved, e_h2d, e_d2h = float(vmax.item()), *(float(x) for x in vsum.tolist())
        line["e2e"] = {"value": e_solved / e_s, "unit": "plans/s", "h2d_bytes_per_step": int(e_h2d),
                       "d2h_bytes_per_step": int(e_d2h), "steps": e_steps, "rank0_timed_region": e_diag,
                       "api": "prrtc_b200.prrtc_plan_batch_async + .results() (per-problem collision_context "
                              "dicts, host numpy inputs, one call per step for all of a rank's problems, three "
                              "steps in flight on one stream: later steps are packed and copied while the "
                              "oldest plans; paths copied to the host; steady state: the timed window holds "
                              "exactly `steps` calls (enqueue with its host->device copy) and `steps` "
                              "read-backs, after 8 untimed steps of the same loop; whole job: every rank, "
                              "slowest rank's time)"}

    if rank == 0 and not a.no_extras:
        # the planners' buffers still hold the last timed step (e2e plans into its own)
        line.update(revalidate_step(planners))
        if ws == 1:
            # single-GPU side measurements (kernels, CPU baseline, the other
            # workloads) only at N = 1: at N > 1 the other ranks would wait for
            # them at the closing barrier
            line.update(extras(a, torch, lib, dev, problems, planners, settings, tuned, line, cap_of))
            line.update(measure_configs(a, torch, lib, dev, settings, tuned))
        else:
            line.update(planner_roofline(torch, lib, dev, planners, settings, tuned, cap_of))
    if rank == 0:
        line["clocks"] = clk.summary()
        print(json.dumps(line))
    for pl in planners.values():
        pl.graph = None
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def planner_roofline(torch, lib, dev, planners, settings, tuned, cap_of):
    """Roofline of the dominant kernel (explore_kernel) against the FP32 peak
    measured by the FFMA probes, with the planner's device counters."""
    from prrtc_b200.batch import STAT_CONFIGS, STAT_EDGES, STAT_FLOPS, STAT_NN_NODES, BatchPlanner, PlanSettings

    out = {}
    rates = fp32_probe_rates(torch, lib, dev)
    fp32 = max(rates.values())
    out["fp32_peak_tflops_measured"] = fp32
    out["fp32_probe_tflops"] = rates

    # --- planner roofline.  Work per launch from the device counters (stats
    # launches: the counters' atomics slow the kernel, so they are not timed);
    # the planner kernel's own duration from CUDA events that the library
    # records right before and after it (tuning.explore_events), over launches
    # without counters, L2 flushed before each as in the timed region.
    flops = cfgs = edges = nn_nodes = 0
    ms = 0.0
    n_stat, n_time = 3, 10
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    ev1.record()  # creates both events; the library re-records them
    flush = torch.empty(64 * 2**20, dtype=torch.float32, device=dev)
    for N, pl in planners.items():
        s = PlanSettings(**{**settings.__dict__, **tuned[N]})
        ip = BatchPlanner(pl.problems, cap_of[N], s, dev, stats=True)
        ip.launch()
        torch.cuda.synchronize()
        ip.stats.zero_()
        for _ in range(n_stat):
            ip.launch()
        st = ip.stats.cpu().numpy() / n_stat
        flops += st[STAT_FLOPS]; cfgs += st[STAT_CONFIGS]; edges += st[STAT_EDGES]
        nn_nodes += st[STAT_NN_NODES]
        del ip
        tp = BatchPlanner(pl.problems, cap_of[N], s, dev)
        tp.tun.explore_events[0], tp.tun.explore_events[1] = ev0.cuda_event, ev1.cuda_event
        tp.launch()
        torch.cuda.synchronize()
        t_ms = []
        for _ in range(n_time):
            flush.fill_(1.0)
            tp.launch()
            torch.cuda.synchronize()
            t_ms.append(ev0.elapsed_time(ev1))
        ms += float(np.mean(t_ms))
        del tp
    del flush
    achieved = flops / (ms * 1e-3) / 1e12
    out["roofline"] = {"kernel": "explore_kernel (persistent planner)", "bound": "fp32", "achieved": achieved,
                       "peak": fp32, "unit": "TFLOP/s", "frac": achieved / fp32,
                       # DRAM bytes of one planner launch of this workload from one ncu capture
                       # (dram__bytes.sum.per_second x gpu__time_duration, profiles/explore_kernel_uneven512_eager.md):
                       # the trees, radii and scenes live in L1/L2, so the planner hardly touches HBM
                       "traffic": 7.4e6, "traffic_unit": "bytes per launch (ncu)",
                       "peak_source": "measured in bench.py, the faster of the scalar FFMA and packed fma.rn.f32x2 "
                                      "probes (no FP32 entry in MEASURED_PEAKS.json)",
                       "launch_ms": ms, "launches_timed": n_time, "launches_counted": n_stat,
                       "note": "collision FLOPs executed per launch (device counters, mean of 3 launches) / the "
                               "explore_kernel's own duration (CUDA events recorded around it by the library, mean "
                               "of 10 launches without counters, L2 flushed before each); the planner is "
                               "latency-bound by its dependent sample->NN->extend->check iterations"}
    out["planner_collision_checks_per_s"] = cfgs / (ms * 1e-3)
    out["planner_edges_per_s"] = edges / (ms * 1e-3)
    out["planner_nn_gbs"] = nn_nodes * 7 * 4 / (ms * 1e-3) / 1e9

    return out


def extras(a, torch, lib, dev, problems, planners, settings, tuned, line, cap_of):
    """Side measurements on rank 0 at N = 1: roofline of the planner kernel, the
    plain per-problem launch form, standalone CC and NN kernels, and the CPU
    baseline."""
    from prrtc_b200.prrtc import prrtc_plan_batch

    out = planner_roofline(torch, lib, dev, planners, settings, tuned, cap_of)
    peaks = measured_peaks()
    fp32 = out["fp32_peak_tflops_measured"]

    # --- plain per-problem-launch form (the reference's batch structure) on the same GPU
    from prrtc_b200.batch import bucket_problems

    plain_ms = []

    def plain(ps_all):
        solved = 0
        plain_ms.clear()
        for N, ps in bucket_problems(ps_all).items():
            G = max(p.goals.shape[0] for p in ps)
            goals = np.zeros((len(ps), G, ps[0].dim), np.float32)
            for i, p in enumerate(ps):
                goals[i, : p.goals.shape[0]] = p.goals
            res = prrtc_plan_batch(np.stack([p.start for p in ps]), goals, max_iterations=settings.max_iterations,
                                   num_new_samples=128, max_nodes=N, min_vals=ps[0].lower, max_vals=ps[0].upper,
                                   collision_context=[p.context for p in ps],
                                   collision_checker=settings.collision_checker,
                                   goal_counts=[p.goals.shape[0] for p in ps],
                                   edge_resolution=settings.edge_resolution, launch="per_problem",
                                   return_trees=False)
            solved += sum(r.solved for r in res)
            plain_ms.extend(r.kernel_time_ms for r in res if r.solved and r.kernel_time_ms is not None)
        return solved

    plain(problems)  # warm: first-call stream and workspace set-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    solved_plain = plain(problems)
    torch.cuda.synchronize()
    dtp = time.perf_counter() - t0
    out["plain_per_problem_e2e"] = {"plans_per_s": solved_plain / dtp, "success_rate": solved_plain / len(problems),
                                    "p50_solve_ms": float(np.median(plain_ms)) if plain_ms else None,
                                    "note": "one plain planner launch per problem over 8 streams, 128 explorers "
                                            "each, host-timed incl. per-problem set-up (the reference's batch "
                                            "form); second of two passes"}
    out["plain_per_problem"] = measure_plain_device(torch, dev, problems, settings)
    out["batched_vs_plain"] = line["value"] / max(out["plain_per_problem"]["plans_per_s"], 1e-9)
    out["batched_vs_plain_e2e"] = line["value"] / max(out["plain_per_problem_e2e"]["plans_per_s"], 1e-9)

    out.update(measure_cc(torch, dev, fp32))
    out.update(measure_checkers(torch, dev))
    out.update(measure_nn(torch, dev, peaks))
    out.update(measure_smooth(torch, dev))

    # --- CPU baseline (the reference's host loop restated): Run A on one pinned
    # core; Run B with a thread pool over each iteration's edge checks on every core
    from oracle import oracle as O

    O.build()
    ra = _cpu_run(problems, 1, a.cpu_seconds, True)
    rb = _cpu_run(problems, O.cpu_count(), a.cpu_seconds / 2, False)
    out["cpu_baseline"] = {"value": ra["plans_per_s"], "unit": "plans/s", "cores": 1, "kind": "port",
                           "sample": f"first {ra['problems']} problems of the workload ({a.cpu_seconds:.0f} s budget), "
                                     f"one pinned core, host-driven RRT-Connect restated in C "
                                     f"(prrtc_robogpu.py:103-298), {cpu_model()}"}
    out["cpu_baseline_threads"] = {"value": rb["plans_per_s"], "unit": "plans/s", "cores": rb["threads"],
                                   "sample": f"first {rb['problems']} problems, a thread pool over each iteration's "
                                             f"edge checks on every core", "p50_solve_ms": rb["p50_solve_ms"],
                                   "success_rate": rb["success_rate"]}
    return out


# ----------------------------------------------------------------------------- path re-validation

def _validate_path(args):
    """0: free at an independent 0.01 rad grid; 1: a graze between the planner's
    own waypoints (free on those, less than 1 mm deep); 2: failed."""
    ctx, dim, path = args
    from oracle import oracle as O

    sc = O.Scene(ctx, dim)
    if sc.validate_path(path, 0.01)[0]:
        return 0
    return 1 if sc.validate_planned_path(path)[0] else 2


def revalidate_step(planners):
    """Every path of the last timed step, re-validated after the timed region by
    the float64 binary checker (the oracle, used here as the checker only) at
    0.01 rad joint-space resolution, in a pool of spawned host processes."""
    import multiprocessing as mp

    from oracle import oracle as O

    jobs = []
    for pl in planners.values():
        for p, r in zip(pl.problems, pl.res.to_results(trees=False, paths_on_host=True)):
            if r.solved:
                jobs.append((p.context, p.dim, np.asarray(r.path)))
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(max(1, min(32, O.cpu_count()))) as pool:
        codes = pool.map(_validate_path, jobs, chunksize=8)
    return {"paths_revalidated": len(codes), "paths_failed": int(sum(c == 2 for c in codes)),
            "paths_grazing": int(sum(c == 1 for c in codes)),
            "revalidation": f"every solved path of the last timed step, float64 binary checker at 0.01 rad; a path "
                            f"that fails there but is free on the planner's own waypoints, with a graze under 1 mm "
                            f"between them, counts as grazing, not failed; "
                            f"{time.perf_counter() - t0:.1f} s on the host after the timed region"}


def measure_e2e(torch, dev, planners, settings, tuned, cap_of, steps):
    """End to end through the public API on this rank: host numpy inputs copied
    in and results plus paths copied back inside the timed region.  Returns
    (plans solved, seconds, host->device bytes per step, device->host bytes per
    step, steps)."""
    from prrtc_b200 import device as _device
    from prrtc_b200.prrtc import prrtc_plan_batch_async

    # One public call per step for all problems, up to three in flight on one
    # stream: the host packs and copies the next steps while the device plans
    # the current one, then reads back the oldest step's results (queued by the
    # call right behind its own kernels).  Every timed step's inputs go host ->
    # device and its results device -> host inside the timed window.
    calls = []
    for key, pl in planners.items():
        ps = pl.problems
        G = max(p.goals.shape[0] for p in ps)
        goals = np.zeros((len(ps), G, ps[0].dim), np.float32)
        for i, p in enumerate(ps):
            goals[i, : p.goals.shape[0]] = p.goals
        calls.append((key, ps, np.stack([p.start for p in ps]), goals, [p.context for p in ps],
                      [p.goals.shape[0] for p in ps], cap_of[key]))
    depth = 3
    e2e_stream = torch.cuda.Stream(device=dev)

    def enqueue(k):
        pending = []
        with torch.cuda.stream(e2e_stream):
            for key, ps, starts, goals, ctxs, gcounts, cap in calls:
                pending.append((ps, prrtc_plan_batch_async(
                    starts, goals, max_iterations=settings.max_iterations,
                    num_new_samples=tuned[key]["num_new_samples"], waypoint_chunk=tuned[key]["waypoint_chunk"],
                    max_nodes=cap, min_vals=ps[0].lower, max_vals=ps[0].upper, collision_context=ctxs,
                    collision_checker=settings.collision_checker, goal_counts=gcounts,
                    edge_resolution=settings.edge_resolution,
                    threads_per_explorer=tuned[key]["threads_per_explorer"],
                    ctas_per_sm=tuned[key].get("ctas_per_sm", 0), return_trees=False, paths_on_host=True)))
        return pending

    def collect(pending):
        solved, d2h = 0, 0
        for ps, pend in pending:
            res = pend.results()
            solved += sum(r.solved for r in res)
            d2h += pend.d2h_bytes
        return solved, d2h

    k_e2e = max(1, int(steps))
    n_warm = 2 * depth + 2
    # diagnostics of the timed window: host time per step, device allocations
    # (cudaMalloc by the caching allocator) and garbage-collector pauses
    gc_ms = [0.0, 0.0]

    def gc_cb(phase, info):
        if phase == "start":
            gc_ms[1] = time.perf_counter()
        elif gc_ms[1] > 0.0:
            gc_ms[0] += (time.perf_counter() - gc_ms[1]) * 1e3

    # One continuous pipeline: depth calls always in flight, the first n_warm
    # steps untimed (they fill the caching allocators with every device and
    # pinned block the pattern needs, and the pipeline itself), then a window of
    # exactly k_e2e enqueues (each with its host -> device copy) and k_e2e
    # read-backs (each with its device -> host copies), then an untimed drain of
    # the calls still in flight.
    solved = d2h = 0
    marks = []
    inflight = [enqueue(k) for k in range(depth - 1)]
    t0 = allocs0 = None
    for k in range(n_warm + k_e2e):
        inflight.append(enqueue(k + depth - 1))
        s_, d_ = collect(inflight.pop(0))
        if k == n_warm - 1:
            _device.H2D_BYTES[0] = 0
            gc.callbacks.append(gc_cb)
            allocs0 = torch.cuda.memory_stats(dev).get("num_device_alloc", 0)
            t0 = time.perf_counter()
        elif k >= n_warm:
            solved += s_
            d2h += d_
            marks.append(time.perf_counter())
    dt = marks[-1] - t0
    h2d = _device.H2D_BYTES[0]
    gc.callbacks.remove(gc_cb)
    allocs = torch.cuda.memory_stats(dev).get("num_device_alloc", 0) - allocs0
    for pending in inflight:  # drain, untimed
        collect(pending)
    torch.cuda.synchronize()
    step_ms = np.diff(np.asarray([t0] + marks)) * 1e3
    diag = {"step_ms_p50": float(np.median(step_ms)), "step_ms_max": float(step_ms.max()),
            "gc_ms": gc_ms[0], "device_allocs": int(allocs)}
    return solved, dt, h2d // k_e2e, d2h // k_e2e, k_e2e, diag


def _cc_flops(ctx) -> tuple[int, int]:
    """Algorithmic FP32 flops (FFMA = 2) and pair tests of one full-sweep check
    of a configuration against the scene of `ctx`, per the kernel's own
    per-test constants (prrtc_device.cuh kFlop*): FK J*(90+63) + S*18 sphere
    centres + S*(Ns*8 + Nc*23 + Nb*26 + Nh*6) world tests + P*8 self pairs."""
    J = int(np.asarray(ctx["fk_twists"]).reshape(-1, 6).shape[0])
    S = int(np.asarray(ctx["sphere_radius"]).reshape(-1).shape[0])
    P = int(np.asarray(ctx["self_pairs"]).reshape(-1, 2).shape[0])
    ns, nc, nb, nh = (int(np.asarray(ctx[k]).shape[0]) if np.asarray(ctx[k]).size else 0
                      for k in ("world_spheres", "world_capsules", "world_boxes", "world_halfspaces"))
    flops = J * (90 + 63) + S * 18 + S * (ns * 8 + nc * 23 + nb * 26 + nh * 6) + P * 8
    return flops, S * (ns + nc + nb + nh) + P


def _time_cc(torch, dev, ctx, dim, lo, hi, n, reps, rng, profile=False):
    from prrtc_b200.collision import CollisionChecker

    chk = CollisionChecker(ctx, dim, "binary", 0.0, dev)
    q = torch.from_numpy(rng.uniform(lo, hi, (n, dim)).astype(np.float32)).to(dev)
    outv = torch.empty(n, dtype=torch.int32, device=dev)
    chk.check(q, full_sweep=True, out=outv)
    torch.cuda.synchronize()
    best = 1e30
    if profile:
        torch.cuda.profiler.start()
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        chk.check(q, full_sweep=True, out=outv)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    if profile:
        torch.cuda.profiler.stop()
    return best, float(outv.float().mean().item())


def measure_cc(torch, dev, fp32, configs: int = 1 << 20, reps: int = 3):
    """Standalone FK + collision kernel, flat checker, full sweep: FP32 roofline
    on the tabletop scene, on the single-plan scene (arm, 16 world spheres) and
    on the dual-arm scene (120 spheres, 256 spheres + 64 boxes + floor)."""
    from prrtc_b200 import scenes
    from prrtc_b200.context import build_collision_context

    rng = np.random.default_rng(0)
    arm = scenes.arm(0)
    ctx = build_collision_context(arm, scenes.tabletop_world(rng))
    n = configs
    # the profiled launches (ncu --profile-from-start off) are the tabletop ones
    best, _ = _time_cc(torch, dev, ctx, 7, -2.8, 2.8, n, reps, rng, profile=True)
    f_cfg, _ = _cc_flops(ctx)
    ach = n * f_cfg / (best * 1e-3) / 1e12
    out = {"cc_kernel": {"workload": f"tabletop scene (32 spheres, 8 capsules, 20 boxes, 1 halfspace), {n} configs, "
                                     "flat checker, full sweep", "checks_per_s": n / (best * 1e-3),
                         "flops_per_check": f_cfg, "achieved_tflops": ach,
                         "frac_of_fp32_peak": (ach / fp32) if fp32 else None,
                         # one ncu capture (profiles/check_kernel_tabletop_fullsweep.md): the
                         # configurations, read once; the scene lives in shared memory
                         "traffic_bytes_ncu": 29.45e6}}
    dual = scenes.dual_arm(0)
    others = {}
    for key, robot, world, what in (
            ("config1_spheres16", arm, scenes.spheres_world(np.random.default_rng(1), 16),
             "7-DOF arm (56 spheres, 960 self pairs), 16 world spheres"),
            ("config5_dual_arm", dual, scenes.large_world(np.random.default_rng(2)),
             "dual arm (14 DOF + 4 mimic joints, 120 spheres), 256 spheres + 64 boxes + floor")):
        c = build_collision_context(robot, world)
        dim = int(robot.lower.shape[0])
        t, coll = _time_cc(torch, dev, c, dim, robot.lower, robot.upper, n, reps, rng)
        f, pairs = _cc_flops(c)
        a_ = n * f / (t * 1e-3) / 1e12
        others[key] = {"workload": f"{what}, {n} uniform configurations, flat checker, full sweep",
                       "checks_per_s": n / (t * 1e-3), "flops_per_check": f, "pair_tests_per_check": pairs,
                       "achieved_tflops": a_, "frac_of_fp32_peak": (a_ / fp32) if fp32 else None,
                       "in_collision": coll}
    out["cc_kernel_other_scenes"] = others
    return out


def measure_smooth(torch, dev, paths: int = 512, waypoints: int = 64, launches: int = 20, reps: int = 3):
    """Smoothing adjoint (prrtc_b200_smooth_cost_grad: cost and gradient of the
    smooth collision + length cost through FK, link transforms recomputed in
    the backward sweep) on the tabletop scene: `paths` paths of `waypoints`
    waypoints, one gradient evaluation per launch (one smoothing step)."""
    from prrtc_b200 import scenes
    from prrtc_b200.context import build_collision_context
    from prrtc_b200.smoothing import SmoothContext

    rng = np.random.default_rng(1)
    ctx = build_collision_context(scenes.arm(0), scenes.tabletop_world(rng))
    sctx = SmoothContext(ctx, 7, device=dev)
    a = rng.uniform(-2.8, 2.8, (paths, 1, 7))
    b = rng.uniform(-2.8, 2.8, (paths, 1, 7))
    t = np.linspace(0.0, 1.0, waypoints)[None, :, None]
    wp = torch.from_numpy((a + (b - a) * t).astype(np.float32)).to(dev)
    sctx.cost_grad(wp)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(launches):
            sctx.cost_grad(wp)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / launches)
    S, P = 56, 960
    pairs = S * (32 + 8 + 20 + 1) + P  # robot-sphere / primitive pairs + self pairs per waypoint
    n = paths * waypoints
    return {"smooth_adjoint": {"workload": f"tabletop scene, {paths} paths x {waypoints} waypoints x 7 dims, cost + "
                                          "gradient per launch", "ms_per_launch": best,
                               "waypoint_gradients_per_s": n / (best * 1e-3),
                               "pair_terms_per_s": n * pairs / (best * 1e-3),
                               "pairs_per_waypoint": pairs}}


def measure_checkers(torch, dev, configs: int = 1 << 20, reps: int = 3):
    """Batched collision checks per second of each checker the planner offers
    (binary, differentiable, binary_coarse, binary_coarse_coop), with early
    exit as the planner uses them, on the tabletop scene with uniformly
    random configurations (the reference's benchmark_collision_checkers.py
    compares the same checkers)."""
    from prrtc_b200 import scenes
    from prrtc_b200.collision import CollisionChecker
    from prrtc_b200.context import build_collision_context

    rng = np.random.default_rng(0)
    ctx = build_collision_context(scenes.arm(0), scenes.tabletop_world(rng))
    q = torch.from_numpy(rng.uniform(-2.8, 2.8, (configs, 7)).astype(np.float32)).to(dev)
    outv = torch.empty(configs, dtype=torch.int32, device=dev)
    res = {}
    for name in ("binary", "differentiable", "binary_coarse", "binary_coarse_coop"):
        chk = CollisionChecker(ctx, 7, name, 0.02, dev)
        chk.check(q, out=outv)
        torch.cuda.synchronize()
        best = 1e30
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            chk.check(q, out=outv)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        best_full = 1e30
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            chk.check(q, full_sweep=True, out=outv)
            e1.record()
            e1.synchronize()
            best_full = min(best_full, e0.elapsed_time(e1))
        res[name] = {"checks_per_s": configs / (best * 1e-3), "checks_per_s_full_sweep": configs / (best_full * 1e-3),
                     "in_collision": float(outv.float().mean().item())}
        del chk
    return {"cc_checkers": {"workload": f"tabletop scene, {configs} uniform random configurations, early exit",
                            **res}}


def measure_nn(torch, dev, peaks, reps: int = 3, launches: int = 20):
    """Standalone nearest neighbour (the prrtc_b200_nearest_neighbor entry of
    prrtc_nearest_neighbor) in two regimes: one query over a 32M-node tree
    (940 MB, streamed from HBM on every launch: the HBM roofline case) and 64
    queries over a 4M-node tree (117 MB, re-read from L2 by every query).
    Inputs are staged once; `launches` back-to-back calls sit between two
    events so that host time between calls does not count (the 940 MB tree is
    larger than L2, so each launch reads it from HBM again)."""
    from prrtc_b200 import _lib
    from prrtc_b200.device import ptr, stream_handle, workspace

    lib = _lib.load()

    def one(N, B, dim=7):
        tree = torch.rand((dim, N), device=dev)
        qq = torch.rand((B, dim), device=dev)
        ts = torch.tensor([N], dtype=torch.int32, device=dev)
        idx = torch.empty((B,), dtype=torch.int32, device=dev)
        dist = torch.empty((B,), dtype=torch.float32, device=dev)
        ws = workspace(lib.prrtc_b200_nearest_neighbor_workspace_size(B), dev)
        sp = stream_handle()

        def call():
            _lib.check(lib.prrtc_b200_nearest_neighbor(ptr(tree), dim, N, ptr(ts), ptr(qq), B, ptr(idx), ptr(dist),
                                                       ws.data_ptr(), ws.numel(), sp), "prrtc_b200_nearest_neighbor")

        call()
        torch.cuda.synchronize()
        best = 1e30
        flush_buf = torch.empty(64 * 2**20, device=dev)
        torch.cuda.profiler.start()
        for _ in range(reps):
            flush_buf.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(launches):
                call()
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1) / launches)
        torch.cuda.profiler.stop()
        del tree, qq, flush_buf, ws
        return best, B * N * dim * 4

    ms_h, by_h = one(1 << 25, 1)
    ms_l, by_l = one(1 << 22, 64)
    hbm = peaks.get("hbm_gbs")
    gbs_h = by_h / (ms_h * 1e-3) / 1e9
    return {"nn_kernel": {"workload": "1 query x 33554432 nodes x 7 dims (940 MB tree, HBM-streamed)",
                          "ms": ms_h, "achieved_gbs": gbs_h, "hbm_peak_gbs": hbm,
                          "frac": gbs_h / hbm if hbm else None,
                          # one ncu capture (profiles/nn_kernel_1q_32M_hbm.md): 6.34 TB/s x 148.9 us
                          "traffic_bytes_ncu": 944e6,
                          "note": "algorithmic bytes = nodes x dim x 4 per query; per-launch time of 20 "
                                  "back-to-back launches (init of the 64-bit argmin keys, scan, decode)"},
            "nn_kernel_l2": {"workload": "64 queries x 4194304 nodes x 7 dims (117 MB tree, L2-resident)",
                             "ms": ms_l, "achieved_gbs": by_l / (ms_l * 1e-3) / 1e9,
                             "note": "each query re-reads the tree from L2, so the rate exceeds HBM peak"}}


# ----------------------------------------------------------------------------- the other configurations

def _wilson(k, n, z=1.96):
    if n == 0:
        return (0.0, 0.0)
    p = k / n
    d = 1 + z * z / n
    c = (p + z * z / (2 * n)) / d
    h = z * np.sqrt(p * (1 - p) / n + z * z / (4 * n * n)) / d
    return (float(c - h), float(c + h))


def _pad_goals(problems):
    G = max(p.goals.shape[0] for p in problems)
    goals = np.zeros((len(problems), G, problems[0].dim), np.float32)
    for i, p in enumerate(problems):
        goals[i, : p.goals.shape[0]] = p.goals
    return goals, [p.goals.shape[0] for p in problems]


def _timed_replays(torch, dev, pl, steps, warmup=2):
    """Graph replays of one BatchPlanner, L2 flushed before each, CUDA events
    around each replay; returns per-step ms."""
    flush = torch.empty(int(256 * 2**20) // 4, dtype=torch.float32, device=dev)
    for _ in range(warmup):
        pl.run()
    if pl.graph is None:
        pl.capture()
        pl.run()
    torch.cuda.synchronize()
    ms = []
    for k in range(steps):
        flush.fill_(float(k))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        pl.run()
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    del flush
    return ms


def _batch_line(torch, dev, problems, caps, settings, steps, label):
    """plans/s of one persistent batched launch (graph replay) over `problems`,
    with success rate, tree sizes, device solve times and the nearest-neighbour
    scan rate of one instrumented launch."""
    from prrtc_b200.batch import STAT_NN_NODES, BatchPlanner

    pl = BatchPlanner(problems, caps, settings, dev)
    ms = _timed_replays(torch, dev, pl, steps)
    blk = pl.summary_block().cpu().numpy()
    solved = blk[:, 8] == 1
    kt = blk[:, 9].copy().view(np.float32)
    sizes = blk[:, 0:2].astype(np.int64)
    res = pl.res.to_results(trees=False, paths_on_host=True)
    pl.graph = None
    del pl
    ip = BatchPlanner(problems, caps, settings, dev, stats=True)
    ip.launch()
    torch.cuda.synchronize()
    ip.stats.zero_()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    ip.launch()
    e1.record()
    e1.synchronize()
    st = ip.stats.cpu().numpy()
    nn_gbs = int(st[STAT_NN_NODES]) * problems[0].dim * 4 / (e0.elapsed_time(e1) * 1e-3) / 1e9
    del ip
    step_ms = float(np.mean(ms))
    out = {"workload": label, "problems": len(problems), "steps": steps, "ms_per_step": step_ms,
           "plans_per_s": float(solved.sum()) / (step_ms * 1e-3), "success_rate": float(solved.mean()),
           "success_wilson95": _wilson(int(solved.sum()), len(problems)),
           "unsolved": int((~solved).sum()),
           "mean_tree_nodes": float(sizes.sum(1).mean()), "max_tree_nodes": int(sizes.sum(1).max()),
           "p50_solve_ms": float(np.median(kt[solved])) if solved.any() else None,
           "p95_solve_ms": float(np.percentile(kt[solved], 95)) if solved.any() else None,
           "planner_nn_gbs": nn_gbs,
           "tuning": {"num_new_samples": settings.num_new_samples, "threads_per_explorer": settings.threads_per_explorer,
                      "waypoint_chunk": settings.waypoint_chunk, "ctas_per_sm": settings.ctas_per_sm},
           "buckets": {str(c): int(sum(1 for x in caps if x == c)) for c in sorted(set(caps))}}
    return out, res


def _tune_chunk(problems, settings, dev):
    """The headline's explorers, threads and CTAs per SM with the waypoint chunk
    chosen for this workload (dense scenes reject most edges in the first pass
    of a small chunk; sparse ones pass whole edges in one pass of 64)."""
    from prrtc_b200.autotune import choose
    from prrtc_b200.batch import PlanSettings

    s = settings
    cands = [(s.num_new_samples, s.threads_per_explorer, cw, s.ctas_per_sm) for cw in (16, 32, 64)]
    best = choose(problems, [p.max_nodes for p in problems], s, dev, candidates=cands, use_cache=False, finalists=2,
                  final_reps=2)
    return PlanSettings(**{**s.__dict__, **best})


def measure_dense(torch, dev, settings, steps=5, n=512):
    """The 512-problem uneven batch at the 16-sphere scene's density (worlds in
    [-0.8,0.8]^2 x [0,1.2], boxes of half extents up to 0.3 m): trees grow,
    the capacity buckets fill and some problems are unsolvable (they run to
    max_iterations and count as unsolved)."""
    from prrtc_b200 import scenes
    from prrtc_b200.collision import gpu_checker

    robot = scenes.arm(0)
    chk = gpu_checker(dev)
    t0 = time.perf_counter()
    problems = [scenes.make_problem("dense", 300000 + i, chk, robot=robot) for i in range(n)]
    gen_s = time.perf_counter() - t0
    settings = _tune_chunk(problems, settings, dev)
    out, _ = _batch_line(torch, dev, problems, [p.max_nodes for p in problems], settings, steps,
                         "dense512: the uneven counts (4-128 spheres r 0.05-0.15, 0-32 boxes of half extents "
                         "0.02-0.3 m) in [-0.8,0.8]^2 x [0,1.2], 1-8 goals, buckets 4096/16384/65536")
    out["generation_s"] = gen_s
    return {"dense512": out}


def _pin_one_core():
    os.sched_setaffinity(0, {sorted(os.sched_getaffinity(0))[0]})


def _host_plan(args):
    """One problem through the reference's host-driven RRT-Connect loop, restated
    in C (prrtc_robogpu.py:103-298); returns (solved, seconds, config checks)."""
    ctx, dim, start, goals, lo, hi, seed, threads = args
    from oracle import oracle as O

    sc = O.Scene(ctx, dim)
    t0 = time.perf_counter()
    r = O.rrtc_host_plan(sc, start, goals, lo, hi, max_iterations=1000, step_size=0.5, num_new_samples=128,
                         granularity=16, max_nodes=65536, connect_max_steps=32, seed=seed, collision_mode=0,
                         n_threads=threads)
    return bool(r.solved), time.perf_counter() - t0, int(r.config_checks)


def _cpu_run(problems, threads, budget_s, pin):
    """The host loop over problems in order until the budget is spent, in one
    spawned process (pinned to one core with `pin`)."""
    import multiprocessing as mp

    args = [(p.context, p.dim, p.start, p.goals, p.lower, p.upper, i, threads) for i, p in enumerate(problems)]
    solved, secs, checks = [], [], 0
    with mp.get_context("spawn").Pool(1, initializer=_pin_one_core if pin else None) as pool:
        t0 = time.perf_counter()
        for s, dt, c in pool.imap(_host_plan, args):
            solved.append(s)
            secs.append(dt)
            checks += c
            if time.perf_counter() - t0 > budget_s:
                break
    secs = np.asarray(secs)
    ok = np.asarray(solved, bool)
    return {"problems": int(ok.size), "threads": threads, "pinned_to_one_core": pin,
            "success_rate": float(ok.mean()) if ok.size else None,
            "p50_solve_ms": float(np.median(secs[ok]) * 1e3) if ok.any() else None,
            "plans_per_s": float(ok.sum() / secs.sum()) if secs.size else None,
            "checks_per_s": float(checks / secs.sum()) if secs.size else None}


def measure_config1(torch, dev, n=32, cpu_budget_s=10.0):
    """Single plan, 7-DOF arm among 16 spheres (seeds 0..n-1; the configuration
    names seed 0), step 0.5, 128 samples, 10000 iterations, 65536 nodes, the
    reference's defaults otherwise (binary checker, 16 waypoints per edge).  GPU:
    one prrtc_plan call per problem -- device-clock solve time and the host wall
    time of the call (inputs copied in, path read back).  CPU path: the
    reference's host loop restated in C on this host, Run A on one pinned core,
    Run B with a thread pool over each iteration's edge checks on every core."""
    from oracle import oracle as O
    from prrtc_b200 import prrtc_plan, scenes
    from prrtc_b200.collision import gpu_checker

    chk = gpu_checker(dev)
    problems = [scenes.make_problem("spheres16", i, chk) for i in range(n)]
    kw = dict(max_iterations=10000, step_size=0.5, num_new_samples=128, max_nodes=65536)
    p0 = problems[0]
    prrtc_plan(p0.start, p0.goals, min_vals=p0.lower, max_vals=p0.upper, collision_context=p0.context, **kw)
    torch.cuda.synchronize()
    dev_ms, wall_ms, ok = [], [], []
    for p in problems:
        t0 = time.perf_counter()
        r = prrtc_plan(p.start, p.goals, min_vals=p.lower, max_vals=p.upper, collision_context=p.context, **kw)
        path = r.path.cpu() if r.solved else None
        wall_ms.append((time.perf_counter() - t0) * 1e3)
        dev_ms.append(r.kernel_time_ms)
        ok.append(bool(r.solved) and path is not None)
    ok = np.asarray(ok)
    gpu = {"problems": n, "success_rate": float(ok.mean()),
           "p50_solve_ms_device": float(np.median(np.asarray(dev_ms)[ok])),
           "p50_call_ms_host": float(np.median(np.asarray(wall_ms)[ok])),
           "note": "device: globaltimer from the first explorer's start to the solution; host: the whole "
                   "prrtc_plan call including set-up, copies and the path read-back"}
    cores = O.cpu_count()
    run_a = _cpu_run(problems, 1, cpu_budget_s, True)
    run_b = _cpu_run(problems, cores, cpu_budget_s, False)
    return {"config1_single_plan": {"workload": "7-DOF arm, 16 world spheres, 1 goal, seeds 0..%d" % (n - 1),
                                    "gpu": gpu, "cpu_run_a": run_a, "cpu_run_b": run_b, "cpu": cpu_model(),
                                    "cpu_path": "host-driven RRT-Connect (prrtc_robogpu.py:103-298) restated "
                                                "in C: uniform samples, brute-force nearest neighbour, steer, "
                                                "batched edge checks, greedy connect (JAX and PyRoFFI absent)"}}


def measure_config2_4(torch, dev, settings, want4, n=1000, oracle_sample=100, smooth_paths_n=512):
    """n tabletop problems as plain single plans (one launch per problem, 8
    streams): success, path cost, device time to solution; the oracle's
    sequential restatement of the planner on the first problems as the
    reference.  Then smoothing: the first 512 solved paths resampled to 64 waypoints,
    50 projected gradient steps of the adjoint cost (each path in its own
    world, one batched launch per step), exact re-validation at 0.01 rad."""
    import multiprocessing as mp

    from oracle import oracle as O
    from prrtc_b200 import prrtc_plan_batch, scenes
    from prrtc_b200.collision import gpu_checker

    chk = gpu_checker(dev)
    robot = scenes.arm(0)
    t0 = time.perf_counter()
    problems = [scenes.make_problem("tabletop", 200000 + i, chk, robot=robot) for i in range(n)]
    gen_s = time.perf_counter() - t0
    goals, gcount = _pad_goals(problems)
    kw = dict(max_iterations=settings.max_iterations, num_new_samples=128, max_nodes=65536,
              collision_checker=settings.collision_checker, edge_resolution=settings.edge_resolution)
    t0 = time.perf_counter()
    res = prrtc_plan_batch(np.stack([p.start for p in problems]), goals, goal_counts=gcount,
                           min_vals=problems[0].lower, max_vals=problems[0].upper,
                           collision_context=[p.context for p in problems], launch="per_problem",
                           return_trees=False, **kw)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    ok = np.array([r.solved for r in res])
    cost = np.array([r.cost for r in res if r.solved])
    kt = np.array([r.kernel_time_ms for r in res if r.solved])
    # the oracle's sequential restatement (explorers in round-robin) on the first problems
    jobs = [(p.context, p.dim, p.start, p.goals, p.lower, p.upper) for p in problems[:oracle_sample]]
    with mp.get_context("spawn").Pool(max(1, min(32, O.cpu_count()))) as pool:
        ora = pool.map(_oracle_plan_job, jobs, chunksize=2)
    oo = np.array([s for s, _ in ora])
    oc = np.array([c for s, c in ora if s])
    out = {"config2_tabletop": {
        "workload": f"{n} tabletop problems (floor, table + 3-5 shelves + clutter = 20 boxes, 8 capsules, "
                    "32 spheres, 4 goals), plain single-plan launches, 128 explorers, 65536 nodes",
        "problems": n, "generation_s": gen_s, "wall_s": wall, "success_rate": float(ok.mean()),
        "success_wilson95": _wilson(int(ok.sum()), n),
        "cost_mean": float(cost.mean()), "cost_median": float(np.median(cost)),
        "p50_time_to_solution_ms": float(np.median(kt)), "p95_time_to_solution_ms": float(np.percentile(kt, 95)),
        "oracle": {"problems": int(oo.size), "success_rate": float(oo.mean()),
                   "success_wilson95": _wilson(int(oo.sum()), int(oo.size)),
                   "cost_median": float(np.median(oc)) if oc.size else None,
                   "gpu_cost_median_same_problems": float(np.median([r.cost for r in res[:oracle_sample]
                                                                     if r.solved])),
                   "what": "sequential restatement of the same planner (explorers in round-robin), same "
                           "settings, on the first problems"}}}
    if want4:
        out.update(measure_config4(torch, dev, problems, res, smooth_paths_n))
    return out


def _oracle_plan_job(args):
    ctx, dim, start, goals, lo, hi = args
    from oracle import oracle as O

    r = O.plan(O.Scene(ctx, dim), start, goals, lo, hi, max_iterations=10000, num_new_samples=128, max_nodes=65536,
               collision_mode=3, edge_resolution=0.01)
    return r.solved == 1, r.cost


def _smoothing_pass(torch, dev, paths, contexts, lower, upper, waypoints, steps=50):
    """Resample, `steps` projected gradient steps of the batched adjoint
    (CUDA events around the steps), exact re-validation; wall time of the whole
    pass."""
    from prrtc_b200.smoothing import BatchSmoothContext, projected_steps, resample_path, revalidate_batch

    t0 = time.perf_counter()
    dim = int(np.asarray(paths[0]).shape[1])
    init = torch.from_numpy(np.stack([resample_path(np.asarray(p), waypoints) for p in paths])).to(dev)
    sctx = BatchSmoothContext(contexts, dim, device=dev)
    c0, _ = sctx.cost_grad(init, need_grad=False)
    projected_steps(sctx, init, lower, upper, 2, 0.05)  # warm
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    x = projected_steps(sctx, init, lower, upper, steps, 0.05)
    e1.record()
    e1.synchronize()
    c1, _ = sctx.cost_grad(x, need_grad=False)
    accepted = revalidate_batch(x, contexts, 0.01, dev)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    acc = accepted.cpu().numpy()
    c0, c1 = c0.cpu().numpy(), c1.cpu().numpy()
    final = np.where(acc, c1, c0)
    return {"paths": len(paths), "waypoints": waypoints, "dim": dim, "steps": steps,
            "device_ms_steps": e0.elapsed_time(e1), "ms_per_step": e0.elapsed_time(e1) / steps,
            "wall_s_pass": wall, "accepted_rate": float(acc.mean()),
            "cost_before_mean": float(c0.mean()), "cost_after_mean": float(final.mean()),
            "cost_drop_mean": float((c0 - final).mean()),
            "note": "cost = sum softplus_50(0.02 - d) over robot-sphere/world and self pairs + squared path "
                    "length; paths that fail exact re-validation at 0.01 rad revert to the planner's path"}


def measure_config4(torch, dev, problems, res, n=512):
    solved = [(p, r) for p, r in zip(problems, res) if r.solved]
    sel = solved[:n]
    paths = [np.asarray(r.path.cpu() if hasattr(r.path, "cpu") else r.path) for _, r in sel]
    out = _smoothing_pass(torch, dev, paths, [p.context for p, _ in sel], sel[0][0].lower, sel[0][0].upper, 64)
    out["workload"] = f"the first {len(sel)} solved tabletop paths, 64 waypoints x 7 DOF, each in its own world"
    return {"config4_smoothing": out}


def measure_config5(torch, dev, settings, tuned, n=1024, steps=3):
    """1024 dual-arm problems (two 7-DOF arms 0.6 m apart with two mimic finger
    joints each, 120 spheres; 256 spheres + 64 boxes + floor; 1-4 goals; 131072
    nodes) in one persistent batched launch, then the smoothing pass at 96
    waypoints x 14 DOF on the solved paths."""
    from prrtc_b200 import scenes
    from prrtc_b200.batch import PlanSettings
    from prrtc_b200.collision import gpu_checker

    chk = gpu_checker(dev)
    robot = scenes.dual_arm(0)
    t0 = time.perf_counter()
    problems = [scenes.make_problem("large", 400000 + i, chk, robot=robot) for i in range(n)]
    gen_s = time.perf_counter() - t0
    s = _tune_chunk(problems, PlanSettings(**{**settings.__dict__, **tuned}), dev)
    line, res = _batch_line(torch, dev, problems, [p.max_nodes for p in problems], s, steps,
                            f"{n} dual-arm problems (14 DOF + 4 mimic joints, 120 spheres), 256 spheres + 64 boxes "
                            "+ floor, 1-4 goals, 131072 nodes")
    line["generation_s"] = gen_s
    sel = [(p, r) for p, r in zip(problems, res) if r.solved]
    sm = _smoothing_pass(torch, dev, [np.asarray(r.path) for _, r in sel], [p.context for p, _ in sel],
                         sel[0][0].lower, sel[0][0].upper, 96)
    return {"config5_dual_arm": {**line, "smoothing": sm}}


def measure_plain_device(torch, dev, problems, settings, n_streams=8):
    """The plain per-problem form timed on the device: every problem's inputs
    staged on the GPU beforehand, one plain planner launch per problem (128
    explorers, its own tree capacity) over `n_streams` streams, all launches
    captured in one CUDA graph and replayed between CUDA events -- host set-up
    excluded, as for the batched value."""
    import ctypes as C

    from prrtc_b200 import _lib
    from prrtc_b200.device import DeviceContext, workspace
    from prrtc_b200.prrtc import _attrs, _outputs_struct, _resolve_collision_mode, _tuning

    lib = _lib.load()
    keep, calls = [], []
    mode = _resolve_collision_mode(settings.collision_checker)
    for p in problems:
        N = int(p.max_nodes)
        ctx = DeviceContext(p.context, dev)
        st = torch.from_numpy(p.start).to(dev)
        gl = torch.from_numpy(np.ascontiguousarray(p.goals)).to(dev)
        lo, hi = torch.from_numpy(p.lower).to(dev), torch.from_numpy(p.upper).to(dev)
        inp = _lib.Inputs()
        inp.start_config, inp.goal_configs, inp.num_goals = st.data_ptr(), gl.data_ptr(), gl.shape[0]
        inp.min_vals, inp.max_vals = lo.data_ptr(), hi.data_ptr()
        inp.robot, inp.world = ctx.robot(), ctx.world()
        t = {k: torch.empty(shape, dtype=dt, device=dev) for k, shape, dt in (
            ("ta", (p.dim, N), torch.float32), ("tb", (p.dim, N), torch.float32), ("pa", (N,), torch.int32),
            ("pb", (N,), torch.int32), ("sz", (2,), torch.int32), ("cp", (2,), torch.int32),
            ("it", (1,), torch.int32), ("cn", (3,), torch.int32), ("sv", (1,), torch.int32),
            ("kt", (1,), torch.float32))}
        outs = _outputs_struct(t["ta"], t["tb"], t["pa"], t["pb"], t["sz"], t["cp"], t["it"], t["cn"], t["sv"],
                               t["kt"])
        attrs = _attrs(settings.max_iterations, settings.step_size, 128, settings.balance_mode, settings.tree_ratio,
                       settings.dynamic_domain, settings.dd_alpha, settings.dd_radius, settings.dd_min_radius, p.dim,
                       N, settings.granularity, mode, settings.collision_margin)
        tun = _tuning(settings.edge_resolution, 128, 16)
        ws = workspace(lib.prrtc_b200_plan_workspace_size(C.byref(inp), C.byref(attrs), C.byref(tun)), dev)
        keep.append((ctx, st, gl, lo, hi, t, ws))
        calls.append((inp, outs, attrs, tun, ws, t))
    streams = [torch.cuda.Stream(device=dev) for _ in range(n_streams)]

    def launch_all():
        main = torch.cuda.current_stream()
        for s in streams:
            s.wait_stream(main)
        for i, (inp, outs, attrs, tun, ws, _) in enumerate(calls):
            s = streams[i % n_streams]
            _lib.check(lib.prrtc_b200_plan(C.byref(inp), C.byref(outs), C.byref(attrs), C.byref(tun), ws.data_ptr(),
                                           ws.numel(), s.cuda_stream), "prrtc_b200_plan")
        for s in streams:
            main.wait_stream(s)

    launch_all()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        launch_all()
    flush = torch.empty(int(256 * 2**20) // 4, dtype=torch.float32, device=dev)
    ms = []
    for k in range(4):
        flush.fill_(float(k))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g.replay()
        e1.record()
        e1.synchronize()
        if k:
            ms.append(e0.elapsed_time(e1))
    solved = np.array([int(c[5]["sv"].item()) == 1 for c in calls])
    kt = np.array([float(c[5]["kt"].item()) for c in calls])
    del g
    step = float(np.mean(ms))
    return {"plans_per_s": float(solved.sum()) / (step * 1e-3), "ms_per_step": step,
            "success_rate": float(solved.mean()), "p50_solve_ms": float(np.median(kt[solved])),
            "note": f"one plain planner launch per problem (128 explorers, per-problem tree capacity) over "
                    f"{n_streams} streams, inputs resident, all launches in one CUDA graph replayed between "
                    f"CUDA events, L2 flushed before each replay; mean of 3 replays"}


def measure_configs(a, torch, lib, dev, settings, tuned):
    """The other workloads (single plan, 1000 tabletop plans, smoothing, dual arm, dense batch), rank 0,
    after the headline."""
    from prrtc_b200.batch import PlanSettings

    want = set(x.strip() for x in a.configs.split(",")) - {"none", ""}
    out = {}
    tuned_one = next(iter(tuned.values()))
    jobs = [("dense", "dense512", lambda: measure_dense(torch, dev, PlanSettings(**{**settings.__dict__, **tuned_one}))),
            ("1", "config1_single_plan", lambda: measure_config1(torch, dev)),
            ("2", "config2_tabletop", lambda: measure_config2_4(torch, dev, settings, "4" in want,
                                                                 n=a.config2_problems)),
            ("5", "config5_dual_arm", lambda: measure_config5(torch, dev, settings, tuned_one,
                                                               n=a.config5_problems))]
    for key, name, fn in jobs:
        if key in want or (key == "2" and "4" in want):
            try:  # one configuration failing is reported in the line instead of losing the headline
                out.update(fn())
            except Exception as exc:  # noqa: BLE001
                out[name] = {"error": f"{type(exc).__name__}: {exc}"[:500]}
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
    return out


def run_kernel(a):
    import torch

    from prrtc_b200 import _lib, build

    build.build()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    lib = _lib.load()
    if a.kernel == "cc":
        out = measure_cc(torch, dev, fp32_peak_tflops(torch, lib, dev))
    elif a.kernel == "smooth":
        out = measure_smooth(torch, dev)
    elif a.kernel == "checkers":
        out = measure_checkers(torch, dev)
    else:
        out = measure_nn(torch, dev, measured_peaks())
    print(json.dumps(out))
    return 0


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)
    if a.kernel:
        return run_kernel(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())
