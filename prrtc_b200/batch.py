"""Preallocated batched planner: problems packed once, buffers static, the whole
plan (scene packing, output initialisation, persistent planner, path
extraction) replayable as one captured CUDA graph.

Problems of different tree capacities share one planner when ``max_nodes`` is
a per-problem list (row stride = the largest capacity, each tree bounded by its
own); separate ``BatchPlanner`` instances per capacity bucket, each with its
own graph (problems grouped by ``bucket_problems``), remain available.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .device import DeviceContext, cuda_device, workspace
from .prrtc import PRRTCResult, _attrs, _pack_worlds, _resolve_collision_mode, _Results, _tuning, lpt_order

STAT_EDGES, STAT_CONFIGS, STAT_FLOPS, STAT_NN_NODES = range(4)


@dataclass
class PlanSettings:
    max_iterations: int = 10000
    step_size: float = 0.5
    num_new_samples: int = 128
    granularity: int = 16
    balance_mode: int = 1
    tree_ratio: float = 0.5
    dynamic_domain: bool = True
    dd_alpha: float = 1e-4
    dd_radius: float = 4.0
    dd_min_radius: float = 1.0
    collision_checker: str = "binary_coarse_coop"
    collision_margin: float = 0.02
    edge_resolution: float = 0.01
    threads_per_explorer: int = 128
    waypoint_chunk: int = 16
    resident_ctas: int = 0
    tail_explorers: bool = True
    ctas_per_sm: int = 0


class BatchPlanner:
    """B problems sharing one robot, each with its own world and goals, planned by
    the persistent batched kernel with ``max_nodes`` tree slots per problem."""

    def __init__(self, problems, max_nodes: int, settings: PlanSettings, device=None, stats: bool = False,
                 order: str | None = "lpt"):
        self.lib = _lib.load()
        self.dev = cuda_device(device)
        self.settings = settings
        self.problems = list(problems)
        B = self.B = len(self.problems)
        dim = self.dim = self.problems[0].dim
        # an int, or one capacity per problem (one launch; row stride = the largest)
        caps = None
        if isinstance(max_nodes, (list, tuple, np.ndarray)):
            caps = np.asarray(max_nodes, dtype=np.int32).reshape(B)
            max_nodes = int(caps.max())
        self.N = int(max_nodes)
        G = max(p.goals.shape[0] for p in self.problems)
        # ---- host staging (pinned) ----
        starts = np.stack([p.start for p in self.problems]).astype(np.float32)
        goals = np.zeros((B, G, dim), np.float32)
        gcount = np.zeros((B,), np.int32)
        for i, p in enumerate(self.problems):
            goals[i, : p.goals.shape[0]] = p.goals
            gcount[i] = p.goals.shape[0]
        contexts = [p.context for p in self.problems]
        packed, counts = _pack_worlds(contexts, B)
        order_np = lpt_order(contexts) if order == "lpt" else np.arange(B, dtype=np.int32)
        self.host = {
            "starts": starts, "goals": goals, "goal_counts": gcount, "order": order_np,
            "lo": self.problems[0].lower.astype(np.float32), "hi": self.problems[0].upper.astype(np.float32),
        }
        for k in packed:
            self.host[k] = packed[k]
            self.host[k + "_count"] = counts[k]
        if caps is not None:
            self.host["caps"] = caps
        self.pinned = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k, v in self.host.items()}
        self.d = {k: torch.empty_like(v, device=self.dev) for k, v in self.pinned.items()}
        self.upload()
        # ---- robot tables (shared) ----
        self.robot_ctx = DeviceContext(contexts[0], self.dev, world_keys=False)
        # ---- C structs ----
        d = self.d
        bi = _lib.BatchInputs()
        bi.batch = B
        bi.start_configs, bi.goal_configs, bi.num_goals = d["starts"].data_ptr(), d["goals"].data_ptr(), G
        bi.goal_counts = d["goal_counts"].data_ptr()
        bi.min_vals, bi.max_vals = d["lo"].data_ptr(), d["hi"].data_ptr()
        bi.robot = self.robot_ctx.robot()
        for key in ("world_spheres", "world_capsules", "world_boxes", "world_halfspaces", "self_pairs"):
            n = int(self.host[key].shape[1])
            setattr(bi, key, d[key].data_ptr() if d[key].numel() else None)
            setattr(bi, "max_" + key, n)
            setattr(bi, key + "_count", d[key + "_count"].data_ptr())
        bi.problem_order = d["order"].data_ptr()
        if caps is not None:
            bi.problem_capacity = d["caps"].data_ptr()
        self.bi = bi
        s = settings
        self.attrs = _attrs(s.max_iterations, s.step_size, s.num_new_samples, s.balance_mode, s.tree_ratio,
                            s.dynamic_domain, s.dd_alpha, s.dd_radius, s.dd_min_radius, dim, self.N, s.granularity,
                            _resolve_collision_mode(s.collision_checker), s.collision_margin)
        self.tun = _tuning(s.edge_resolution, s.threads_per_explorer, s.waypoint_chunk, s.resident_ctas,
                           s.tail_explorers, s.ctas_per_sm)
        self.stats = torch.zeros(4, dtype=torch.int64, device=self.dev) if stats else None
        if self.stats is not None:
            self.tun.stats = self.stats.data_ptr()
        self.res = _Results(B, dim, self.N, self.dev, (B,))
        self.outs = self.res.outputs()
        self.ws = workspace(self.lib.prrtc_b200_plan_batch_workspace_size(C.byref(bi), C.byref(self.attrs),
                                                                         C.byref(self.tun)), self.dev)
        self.graph = None

    # -- data movement --
    def upload(self, stream: torch.cuda.Stream | None = None) -> int:
        """Host->device copy of every input; returns the bytes copied."""
        n = 0
        with torch.cuda.stream(stream) if stream is not None else _null():
            for k, v in self.pinned.items():
                self.d[k].copy_(v, non_blocking=True)
                n += v.numel() * v.element_size()
        return n

    def h2d_bytes(self) -> int:
        return sum(v.numel() * v.element_size() for v in self.pinned.values())

    # -- execution --
    def launch(self) -> None:
        sp = torch.cuda.current_stream().cuda_stream
        _lib.check(self.lib.prrtc_b200_plan_batch(C.byref(self.bi), C.byref(self.outs), C.byref(self.attrs),
                                                  C.byref(self.tun), self.ws.data_ptr(), self.ws.numel(), sp),
                   "prrtc_b200_plan_batch")
        self.res.extract(sp)

    def capture(self) -> None:
        """Capture launch() as a CUDA graph (warm up once first).  Replays go to
        the caller's current stream."""
        s = torch.cuda.Stream(device=self.dev)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.launch()
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize(self.dev)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.launch()
        self.graph = g

    def run(self) -> None:
        if self.graph is not None:
            self.graph.replay()
        else:
            self.launch()

    # -- results --
    def results(self, trees: bool = False) -> list[PRRTCResult]:
        return self.res.to_results(trees=trees)

    def summary_block(self) -> torch.Tensor:
        """Device tensor [B, 16] of packed scalars (sizes, iterations, connection,
        solved, device solve ms, path length, cost) -- one small read-back."""
        return self.res.block

    def d2h_bytes(self) -> int:
        return self.res.block.numel() * 4


class _null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def bucket_problems(problems):
    """Group problems by tree capacity: {max_nodes: [problems]} (largest first)."""
    out: dict[int, list] = {}
    for p in problems:
        out.setdefault(int(p.max_nodes), []).append(p)
    return dict(sorted(out.items(), key=lambda kv: -kv[0]))
