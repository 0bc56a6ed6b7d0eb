"""Autotuner for the persistent batched planner.

For one capacity bucket, times a plan of the bucket's problems with each
candidate number of explorers per problem (samples per iteration) and keeps the
fastest by solved plans per second; ties within 3% go to fewer explorers.
Results are cached per (device, bucket, problem count, shape) in
``~/.cache/prrtc_b200/autotune.json``.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

import torch

CANDIDATES = (32, 64, 128, 256)
CACHE = Path(os.environ.get("PRRTC_B200_CACHE", Path.home() / ".cache" / "prrtc_b200")) / "autotune.json"


def _key(dev, N, problems, settings) -> str:
    p = problems[0]
    name = torch.cuda.get_device_name(dev)
    return (f"{name}|N{N}|B{len(problems)}|dim{p.dim}|S{p.context['sphere_radius'].shape[0]}|"
            f"{settings.collision_checker}|res{settings.edge_resolution}|T{settings.threads_per_explorer}")


def _load() -> dict:
    try:
        return json.loads(CACHE.read_text())
    except (OSError, json.JSONDecodeError):
        return {}


def choose_samples(problems, N: int, settings, dev, candidates=CANDIDATES, use_cache: bool = True) -> int:
    from .batch import BatchPlanner, PlanSettings

    key = _key(dev, N, problems, settings)
    cache = _load() if use_cache else {}
    if key in cache:
        return int(cache[key])
    best, best_rate = candidates[0], -1.0
    for E in candidates:
        s = PlanSettings(**{**settings.__dict__, "num_new_samples": E})
        pl = BatchPlanner(problems, N, s, dev)
        pl.launch()  # warm
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        pl.launch()
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        solved = int((pl.summary_block()[:, 8] == 1).sum().item())
        rate = solved / (ms * 1e-3)
        if rate > best_rate * 1.03:
            best, best_rate = E, rate
        del pl
    if use_cache:
        cache[key] = best
        try:
            CACHE.parent.mkdir(parents=True, exist_ok=True)
            CACHE.write_text(json.dumps(cache, indent=1))
        except OSError:
            pass
    return best
