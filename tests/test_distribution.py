"""Distributional parity over seeded problems: the GPU planner against the
oracle's sequential restatement of the same algorithm.

Explorers race on the GPU, so trees differ run to run (the reference says the
same: verify_coarse_equivalence.py:3-8); what must agree are the distributions.
The batched planner runs with exactly num_new_samples explorers per problem
(tail_explorers=False), as the reference and the oracle do.

Workload: the dense uneven scenes (4-128 spheres and 0-32 boxes of half extents
up to 0.3 m in [-0.8,0.8]^2 x [0,1.2]), where 2-25% of configuration space is
free and some start / goal pairs are disconnected, with a small tree capacity
(512 nodes) and an iteration limit that is never reached: a problem ends when
it connects or when a tree overflows, both planners solve well under all
problems (about 90%), and the success rate measures the search, not the
easiness of the scenes.  (Ending problems by the iteration limit instead would
compare unlike things: on the GPU the first explorer to pass the limit ends the
problem while its racing peers have run fewer iterations, where the round-robin
restatement gives every explorer the full count.)
Criteria, at 95%: the Wilson intervals of the two success rates overlap, and a
one-sided two-sample Kolmogorov-Smirnov test does not find the GPU's path costs
stochastically larger than the oracle's.  The cost test is one-sided on
purpose: on the GPU the explorers race, and while one explorer walks a long
connection (several checked sub-edges) the others keep inserting nodes, so the
first connection to complete -- which ends the search -- is more often a short
one than in the round-robin restatement, where each explorer's whole connect
runs as one step.  GPU paths come out shorter (measured on this workload:
median cost 6.84 against 8.73, KS D = 0.21), as they would for the
reference's own CTA explorers; a longer GPU path would be a defect.  Every GPU
path is re-validated with the float64 binary checker at 0.01 rad.

test_single_explorer_plans_match_oracle removes the race: with one explorer
per problem the planner is deterministic and must retrace the oracle's
sequence -- the same samples, trees, connection and path, bit for bit --
except where a configuration checked along the way lies so close to contact
that the float32 and float64 verdicts can differ.

PRRTC_DIST_PROBLEMS sets the problem count (default 1000).
"""
from __future__ import annotations

import multiprocessing as mp
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_PROBLEMS = int(os.environ.get("PRRTC_DIST_PROBLEMS", "1000"))
SETTINGS = dict(max_iterations=5000, step_size=0.5, num_new_samples=32, granularity=16, balance_mode=1,
                tree_ratio=0.5, dynamic_domain=True, collision_margin=0.02)
CHECKER, MODE, RES, N_NODES = "binary_coarse_coop", 3, 0.01, 512
KIND = "dense"


def _make(seed):
    from conftest import make_problem

    return make_problem(KIND, seed)


def _oracle_plan(seed):
    from conftest import make_problem
    from oracle import oracle as O

    pr = make_problem(KIND, seed)
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
    G = max(p.goals.shape[0] for p in problems)
    goals = np.zeros((len(problems), G, problems[0].dim), np.float32)
    for i, p in enumerate(problems):
        goals[i, : p.goals.shape[0]] = p.goals
    res = prrtc_plan_batch(np.stack([p.start for p in problems]), goals, goal_counts=[p.goals.shape[0] for p in problems],
                           max_nodes=N_NODES, min_vals=problems[0].lower, max_vals=problems[0].upper,
                           collision_context=[p.context for p in problems], collision_checker=CHECKER,
                           edge_resolution=RES, return_trees=False, tail_explorers=False, **SETTINGS)
    gs = np.array([r.solved for r in res])
    gc = np.array([r.cost for r in res if r.solved])
    os_ = np.array([s for s, _ in ora])
    oc = np.array([c for s, c in ora if s])
    # Every GPU path re-validates on the planner's own waypoints (granularity 16
    # and 0.01 rad, t = (k+1)/G per edge): a waypoint there that the oracle finds
    # in collision would be a checker miss.  An independent 0.01 rad grid (t =
    # k/n, n = ceil(len/res)) may still land in a graze that lies between the
    # planner's waypoints -- the resolution limit of any sampled edge check, which
    # the reference's own evaluation shows as solved paths that are not valid --
    # so those are counted and bounded: shallow, and rare.
    misses, slivers = [], []
    n_paths = 0
    for seed, p, r in zip(seeds, problems, res):
        if not r.solved:
            continue
        n_paths += 1
        path = r.path.cpu().numpy()
        sc = orc.Scene(p.context, p.dim)
        ok, md = sc.validate_path(path, RES)
        if ok:
            continue
        grid = np.concatenate([orc.edge_waypoints(path[i], path[i + 1], SETTINGS["granularity"], RES)
                               for i in range(path.shape[0] - 1)] + [path[:1]])
        md_grid = float(sc.min_distances(grid).min())
        _, md_fine = sc.validate_path(path, 0.0005)
        (misses if md_grid < -1e-5 else slivers).append((seed, md_grid, float(md), float(md_fine)))
    assert not misses, f"{len(misses)} paths collide on the planner's own waypoints (seed, min distance there / " \
                       f"at 0.01 / at 0.0005 rad): {misses}"
    assert len(slivers) <= max(2, n_paths // 200) and all(f > -1e-3 for *_, f in slivers), \
        f"grazes between the planner's waypoints (seed, min distance on its waypoints / 0.01 / 0.0005 rad): {slivers}"
    lo_g, hi_g = wilson(gs.sum(), gs.size)
    lo_o, hi_o = wilson(os_.sum(), os_.size)
    summary = (f"success GPU {gs.mean():.4f} [{lo_g:.3f},{hi_g:.3f}] oracle {os_.mean():.4f} [{lo_o:.3f},{hi_o:.3f}]; "
               f"median cost GPU {np.median(gc):.3f} oracle {np.median(oc):.3f}; "
               f"mean cost GPU {gc.mean():.3f} oracle {oc.mean():.3f}")
    print("\n" + summary)
    # the workload discriminates: neither planner solves (almost) everything
    assert 0.5 < os_.mean() < 0.97, summary
    assert lo_g <= hi_o and lo_o <= hi_g, summary
    from scipy.stats import ks_2samp

    # alternative="less": H1 = the GPU's cost CDF lies below the oracle's somewhere (GPU costs larger)
    ks = ks_2samp(gc, oc, alternative="less")
    assert ks.pvalue > 0.05, f"{summary}; one-sided KS D = {ks.statistic:.4f}, p = {ks.pvalue:.4f}"
    rng = np.random.default_rng(0)
    cg, co = boot_median(gc, rng), boot_median(oc, rng)
    assert cg[0] <= co[1], f"{summary}; median cost intervals GPU {cg} oracle {co}"
    print(f"one-sided KS D = {ks.statistic:.4f}, p = {ks.pvalue:.4f}; median cost intervals GPU {cg} oracle {co}")


SINGLE = dict(SETTINGS, num_new_samples=1)


def _oracle_single(seed):
    from conftest import make_problem
    from oracle import oracle as O

    pr = make_problem(KIND, seed)
    r = O.plan(O.Scene(pr.context, pr.dim), pr.start, pr.goals, pr.lower, pr.upper, max_nodes=N_NODES,
               collision_mode=MODE, edge_resolution=RES, **SINGLE)
    return r.solved, r.iter_count, tuple(r.tree_sizes), r.path


def test_single_explorer_plans_match_oracle(cuda, orc):
    from prrtc_b200 import prrtc_plan_batch

    seeds = list(range(7000, 7200))
    ctx = mp.get_context("spawn")
    with ctx.Pool(max(1, min(32, os.cpu_count() or 1))) as pool:
        problems = pool.map(_make, seeds, chunksize=4)
        ora = pool.map(_oracle_single, seeds, chunksize=4)
    G = max(p.goals.shape[0] for p in problems)
    goals = np.zeros((len(problems), G, problems[0].dim), np.float32)
    for i, p in enumerate(problems):
        goals[i, : p.goals.shape[0]] = p.goals
    res = prrtc_plan_batch(np.stack([p.start for p in problems]), goals, goal_counts=[p.goals.shape[0] for p in problems],
                           max_nodes=N_NODES, min_vals=problems[0].lower, max_vals=problems[0].upper,
                           collision_context=[p.context for p in problems], collision_checker=CHECKER,
                           edge_resolution=RES, return_trees=False, tail_explorers=False, **SINGLE)
    same = 0
    for r, (o_solved, o_iters, o_sizes, o_path) in zip(res, ora):
        if bool(r.solved) != (o_solved == 1) or (r.tree_a_size, r.tree_b_size) != o_sizes:
            continue
        if r.solved:
            p = r.path.cpu().numpy()
            if r.iterations != o_iters or p.shape != o_path.shape or not np.array_equal(p.view(np.uint32),
                                                                                        o_path.view(np.uint32)):
                continue
        same += 1
    print(f"\nsingle explorer: {same} of {len(res)} plans identical to the oracle's; solved GPU "
          f"{sum(r.solved for r in res)} oracle {sum(o[0] == 1 for o in ora)}")
    assert same >= 0.85 * len(res)
