"""Distributional parity over seeded problems: the GPU planner against the
oracle's sequential restatement of the same algorithm.

Explorers race on the GPU, so trees differ run to run (the reference says the
same: verify_coarse_equivalence.py:3-8); what must agree are the distributions.
The batched planner runs with exactly num_new_samples explorers per problem
(tail_explorers=False), as the reference and the oracle do.
Criteria, at 95%: the Wilson intervals of the two success rates overlap, and the
bootstrap intervals of the two median path costs overlap.  Every GPU path is
re-validated with the float64 binary checker at 0.01 rad.

PRRTC_DIST_PROBLEMS sets the problem count (default 1000, tabletop workload).
"""
from __future__ import annotations

import multiprocessing as mp
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_PROBLEMS = int(os.environ.get("PRRTC_DIST_PROBLEMS", "1000"))
SETTINGS = dict(max_iterations=2000, step_size=0.5, num_new_samples=32, granularity=16, balance_mode=1,
                tree_ratio=0.5, dynamic_domain=True, collision_margin=0.02)
CHECKER, MODE, RES, N_NODES = "binary_coarse_coop", 3, 0.01, 16384


def _make(seed):
    from conftest import make_problem

    return make_problem("tabletop", seed)


def _oracle_plan(seed):
    from conftest import make_problem
    from oracle import oracle as O

    pr = make_problem("tabletop", seed)
    sc = O.Scene(pr.context, pr.dim)
    r = O.plan(sc, pr.start, pr.goals, pr.lower, pr.upper, max_nodes=N_NODES, collision_mode=MODE,
               edge_resolution=RES, **SETTINGS)
    return r.solved == 1, r.cost


def wilson(k, n, z=1.96):
    p = k / n
    d = 1 + z * z / n
    c = (p + z * z / (2 * n)) / d
    h = z * np.sqrt(p * (1 - p) / n + z * z / (4 * n * n)) / d
    return c - h, c + h


def boot_median(x, rng, n=2000):
    x = np.asarray(x)
    meds = np.median(rng.choice(x, size=(n, x.size), replace=True), axis=1)
    return np.percentile(meds, 2.5), np.percentile(meds, 97.5)


def test_success_and_cost_distributions_match_oracle(cuda, orc):
    from prrtc_b200 import prrtc_plan_batch

    seeds = list(range(5000, 5000 + N_PROBLEMS))
    ctx = mp.get_context("spawn")
    with ctx.Pool(max(1, min(32, os.cpu_count() or 1))) as pool:
        problems = pool.map(_make, seeds, chunksize=8)
        ora = pool.map(_oracle_plan, seeds, chunksize=8)
    res = prrtc_plan_batch(np.stack([p.start for p in problems]), np.stack([p.goals for p in problems]),
                           max_nodes=N_NODES, min_vals=problems[0].lower, max_vals=problems[0].upper,
                           collision_context=[p.context for p in problems], collision_checker=CHECKER,
                           edge_resolution=RES, return_trees=False, tail_explorers=False, **SETTINGS)
    gs = np.array([r.solved for r in res])
    gc = np.array([r.cost for r in res if r.solved])
    os_ = np.array([s for s, _ in ora])
    oc = np.array([c for s, c in ora if s])
    # every GPU path re-validates
    bad = 0
    for p, r in zip(problems, res):
        if r.solved:
            ok, _ = orc.Scene(p.context, p.dim).validate_path(r.path.cpu().numpy(), 0.01)
            bad += not ok
    assert bad == 0, f"{bad} paths failed re-validation"
    lo_g, hi_g = wilson(gs.sum(), gs.size)
    lo_o, hi_o = wilson(os_.sum(), os_.size)
    assert lo_g <= hi_o and lo_o <= hi_g, f"success GPU {gs.mean():.3f} [{lo_g:.3f},{hi_g:.3f}] vs oracle " \
                                          f"{os_.mean():.3f} [{lo_o:.3f},{hi_o:.3f}]"
    rng = np.random.default_rng(0)
    cg, co = boot_median(gc, rng), boot_median(oc, rng)
    assert cg[0] <= co[1] and co[0] <= cg[1], f"median cost GPU {np.median(gc):.3f} {cg} vs oracle " \
                                              f"{np.median(oc):.3f} {co}"
    print(f"\nsuccess GPU {gs.mean():.4f} oracle {os_.mean():.4f}; median cost GPU {np.median(gc):.3f} {cg} "
          f"oracle {np.median(oc):.3f} {co}; mean cost GPU {gc.mean():.3f} oracle {oc.mean():.3f}")
