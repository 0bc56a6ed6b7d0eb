"""Property tests (hypothesis, CPU) of the oracle and the host-side helpers.

Where the fixed-case tests of test_oracle.py pin the oracle on chosen inputs,
these draw the inputs: Halton values against the exact radical inverse at any
index, the nearest-neighbour scan against a float64 argmin over trees with NaN
slots and duplicate nodes, the extend step and the edge waypoints against their
geometric definitions, float32 FK against float64 FK on random arms, the
coarse-gated checkers against the flat checker on random arms and worlds, the
coarse model's enclosure of its fine spheres and its self-pair blocks, the
float64 autograd restatement of the smoothing cost against the C oracle's cost
and its central differences, the paths of the two CPU planners (the
sequential restatement and the host-driven loop of the CPU baseline), and the
longest-processing-time split used to shard a batch over ranks.  The draws are derandomized: every run
tests the same examples.
"""
from __future__ import annotations

from fractions import Fraction

import numpy as np
from hypothesis import given, settings
from hypothesis import strategies as st

from prrtc_b200 import scenes
from prrtc_b200.context import build_collision_context
from prrtc_b200.shard import lpt_partition

PRIMES = [3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59]
FAST = settings(max_examples=150, deadline=None, derandomize=True)
SLOW = settings(max_examples=40, deadline=None, derandomize=True)
seeds = st.integers(0, 2**31 - 1)


def radical_inverse(n: int, b: int) -> Fraction:
    r, f = Fraction(0), Fraction(1, b)
    while n > 0:
        r += f * (n % b)
        n //= b
        f /= b
    return r


@FAST
@given(base=st.sampled_from(PRIMES), n=st.integers(1, 4_000_000))
def test_halton_value_is_the_radical_inverse(orc, base, n):
    v, nxt = orc.halton_next(base, n)
    assert nxt == n + 1
    assert 0.0 <= v < 1.0
    assert abs(v - float(radical_inverse(n, base))) <= 2e-6


@FAST
@given(explorer=st.integers(0, 2**31 - 1))
def test_prime_order_is_a_permutation_of_the_16_primes(orc, explorer):
    assert sorted(orc.prime_order(explorer).tolist()) == PRIMES


@FAST
@given(seed=seeds, dim=st.integers(1, 16), n=st.integers(1, 200), spare=st.integers(0, 8),
       dups=st.integers(0, 6), nan_frac=st.floats(0.0, 0.5))
def test_nearest_is_the_float64_argmin_lowest_index_first(orc, seed, dim, n, spare, dups, nan_frac):
    rng = np.random.default_rng(seed)
    pts = rng.uniform(-3, 3, (n, dim)).astype(np.float32)
    for _ in range(dups if n > 1 else 0):  # later copies of earlier nodes
        i, j = sorted(rng.choice(n, 2, replace=False))
        pts[j] = pts[i]
    nan = rng.random(n) < nan_frac
    tree = np.full((dim, n + spare), np.nan, np.float32)  # slots past n are never scanned
    tree[:, :n] = pts.T
    tree[:, np.flatnonzero(nan)] = np.nan
    q = rng.uniform(-3, 3, dim).astype(np.float32)
    idx, dsq = orc.nearest(tree, n, q)
    if nan.all():
        assert idx == -1
        return
    d64 = ((tree[:, :n].astype(np.float64) - q.astype(np.float64)[:, None]) ** 2).sum(0)
    d64[nan] = np.inf
    best = d64.min()
    assert 0 <= idx < n and not nan[idx]
    assert d64[idx] <= best * (1 + 1e-5) + 1e-9
    assert abs(dsq - d64[idx]) <= 1e-5 * max(1.0, d64[idx])
    same = np.flatnonzero((tree[:, :n] == tree[:, idx:idx + 1]).all(0))
    assert same.min() == idx  # of identical nodes the lowest index wins


@FAST
@given(seed=seeds, dim=st.integers(1, 16), step=st.floats(0.01, 2.0), scale=st.floats(0.001, 4.0))
def test_extend_moves_at_most_one_step_along_the_segment(orc, seed, dim, step, scale):
    rng = np.random.default_rng(seed)
    b = rng.uniform(-2, 2, dim).astype(np.float32)
    s = (b + rng.normal(size=dim) * scale).astype(np.float32)
    seg = s.astype(np.float64) - b.astype(np.float64)
    L = float(np.linalg.norm(seg))
    nd = float(np.float32(L))
    cand = orc.extend(b, s, nd, step)
    d = cand.astype(np.float64) - b.astype(np.float64)
    assert np.linalg.norm(d) <= step * (1 + 1e-5) + 1e-6
    if L > 1e-6:
        t = float(d @ seg) / (L * L)
        assert -1e-5 <= t <= 1 + 1e-5
        assert np.linalg.norm(d - t * seg) <= 1e-5 * max(1.0, L)
    if L <= step:
        assert np.abs(cand - s).max() <= 1e-5 * max(1.0, float(np.abs(s).max()))


@FAST
@given(seed=seeds, dim=st.integers(1, 16), granularity=st.integers(1, 32),
       resolution=st.sampled_from([0.0, 0.005, 0.01, 0.05, 0.1]), scale=st.floats(0.0, 2.0))
def test_edge_waypoints_end_at_the_target_and_respect_the_resolution(orc, seed, dim, granularity, resolution,
                                                                     scale):
    rng = np.random.default_rng(seed)
    b = rng.uniform(-2, 2, dim).astype(np.float32)
    e = (b + rng.normal(size=dim) * scale).astype(np.float32)
    w = orc.edge_waypoints(b, e, granularity, resolution)
    G = w.shape[0]
    L = float(np.linalg.norm(e.astype(np.float64) - b.astype(np.float64)))
    assert G >= granularity
    if resolution > 0:
        assert G >= int(np.ceil(L / resolution * (1 - 1e-5)))
        steps = np.linalg.norm(np.diff(np.vstack([b[None], w]).astype(np.float64), axis=0), axis=1)
        assert steps.max() <= resolution * (1 + 1e-4) + 1e-6
    else:
        assert G == granularity
    assert np.abs(w[-1] - e).max() <= 1e-5 * max(1.0, float(np.abs(e).max()))


@SLOW
@given(seed=st.integers(0, 10**6), n_joints=st.integers(1, 12), qseed=seeds)
def test_fk_float32_within_1e5_of_float64_on_random_arms(orc, seed, n_joints, qseed):
    robot = scenes.arm(seed, n_joints)
    sc = orc.Scene(build_collision_context(robot, None), robot.dim)
    rng = np.random.default_rng(qseed)
    for q in rng.uniform(robot.lower, robot.upper, (8, robot.dim)).astype(np.float32):
        assert np.abs(sc.fk(q, f64=True) - sc.fk(q, f64=False)).max() < 1e-5


@SLOW
@given(qseed=seeds)
def test_fk_float32_within_1e5_of_float64_on_the_mimic_dual_arm(orc, dual, qseed):
    sc = orc.Scene(build_collision_context(dual, None), dual.dim)
    rng = np.random.default_rng(qseed)
    for q in rng.uniform(dual.lower, dual.upper, (8, dual.dim)).astype(np.float32):
        assert np.abs(sc.fk(q, f64=True) - sc.fk(q, f64=False)).max() < 1e-5


@SLOW
@given(seed=st.integers(0, 10**6), n_joints=st.integers(2, 9), wseed=seeds,
       kind=st.sampled_from(["spheres", "tabletop", "uneven"]))
def test_gated_checkers_agree_with_the_flat_checker_on_random_arms_and_worlds(orc, seed, n_joints, wseed, kind):
    robot = scenes.arm(seed, n_joints)
    rng = np.random.default_rng(wseed)
    world = {"spheres": lambda: scenes.spheres_world(rng, 16), "tabletop": lambda: scenes.tabletop_world(rng),
             "uneven": lambda: scenes.uneven_world(rng)}[kind]()
    ctx = build_collision_context(robot, world)
    sc = orc.Scene(ctx, robot.dim)
    q = rng.uniform(robot.lower, robot.upper, (48, robot.dim)).astype(np.float32)
    v0 = sc.check_configs(q, 0)
    md = sc.min_distances(q)
    far = np.abs(md) > 1e-5
    assert np.array_equal(v0[far], (md[far] <= 0).astype(np.int32))
    for mode in (2, 3):  # the coarse gate never changes a verdict
        assert np.array_equal(sc.check_configs(q, mode), v0)


@SLOW
@given(seed=st.integers(0, 10**6), n_joints=st.integers(1, 12))
def test_coarse_spheres_enclose_their_fine_spheres_on_random_arms(seed, n_joints):
    ctx = build_collision_context(scenes.arm(seed, n_joints), None)
    off = ctx["fine_link_offsets"]
    assert off[0] == 0 and off[-1] == ctx["sphere_radius"].shape[0]
    for k in range(ctx["coarse_sphere_link_idx"].shape[0]):
        s, e = off[k], off[k + 1]
        assert (ctx["sphere_link_idx"][s:e] == ctx["coarse_sphere_link_idx"][k]).all()
        # exactly (float64 arithmetic on the stored float32 values): the gate's soundness
        reach = np.linalg.norm(ctx["sphere_local"][s:e].astype(np.float64) -
                               ctx["coarse_sphere_local"][k].astype(np.float64), axis=1) + \
            ctx["sphere_radius"][s:e].astype(np.float64)
        assert (reach <= float(ctx["coarse_sphere_radius"][k])).all()
    pairs = ctx["self_pairs"]
    expect = sum(8 * 8 for i in range(n_joints) for j in range(i + 2, n_joints))
    assert pairs.shape[0] == expect
    if pairs.shape[0]:
        links = ctx["sphere_link_idx"][pairs]
        assert (np.abs(links[:, 0] - links[:, 1]) >= 2).all()


@SLOW
@given(seed=st.integers(0, 10**6), n_joints=st.integers(1, 12))
def test_self_pair_ranges_are_complete_blocks_of_their_coarse_pairs(seed, n_joints):
    """Range q of the self-pair list holds exactly the pairs (fine spheres of
    coarse group a) x (fine spheres of coarse group b) for coarse pair q = (a, b),
    and the ranges tile the list: the layout the packed checker reads as dense
    blocks gated by one coarse pair each."""
    ctx = build_collision_context(scenes.arm(seed, n_joints), None)
    pairs, cp, rng_ = ctx["self_pairs"], ctx["coarse_self_pairs"], ctx["self_pair_ranges"]
    off = ctx["fine_link_offsets"]
    assert cp.shape[0] == rng_.shape[0]
    cursor = 0
    for q in range(cp.shape[0]):
        lo, hi = int(rng_[q, 0]), int(rng_[q, 1])
        assert lo == cursor and hi >= lo
        a, b = int(cp[q, 0]), int(cp[q, 1])
        want = {(i, j) for i in range(off[a], off[a + 1]) for j in range(off[b], off[b + 1])}
        got = {(int(i), int(j)) for i, j in pairs[lo:hi]}
        assert got == want and hi - lo == len(want)
        cursor = hi
    assert cursor == pairs.shape[0]


@SLOW
@given(seed=st.integers(0, 10**6), n_joints=st.integers(2, 9), wseed=seeds,
       kind=st.sampled_from(["spheres", "tabletop", "uneven"]), n_wp=st.integers(3, 8),
       margin=st.sampled_from([0.0, 0.02, 0.05]), beta=st.sampled_from([20.0, 50.0]))
def test_autodiff_smoothing_cost_matches_the_oracle_on_random_arms_worlds_and_paths(orc, seed, n_joints, wseed,
                                                                                    kind, n_wp, margin, beta):
    """The float64 autograd restatement of the smoothing cost -- the reference
    the GPU adjoint is checked against -- equals the C oracle's cost, and its
    gradient equals central differences of that cost."""
    from oracle.smooth_autodiff import smooth_grad

    robot = scenes.arm(seed, n_joints)
    rng = np.random.default_rng(wseed)
    world = {"spheres": lambda: scenes.spheres_world(rng, 16), "tabletop": lambda: scenes.tabletop_world(rng),
             "uneven": lambda: scenes.uneven_world(rng)}[kind]()
    ctx = build_collision_context(robot, world)
    sc = orc.Scene(ctx, robot.dim)
    ends = rng.uniform(robot.lower, robot.upper, (2, robot.dim))
    w = np.linspace(ends[0], ends[1], n_wp) + rng.normal(0, 0.05, (n_wp, robot.dim))
    c, g = smooth_grad(ctx, w, margin, beta, 1.0)
    c64 = sc.smooth_cost(w, margin, beta, 1.0)
    assert abs(c - c64) <= 1e-9 * max(1.0, abs(c64))
    h = 1e-5
    for _ in range(4):
        i, d = int(rng.integers(0, n_wp)), int(rng.integers(0, robot.dim))
        wp, wm = w.copy(), w.copy()
        wp[i, d] += h
        wm[i, d] -= h
        fd = (sc.smooth_cost(wp, margin, beta, 1.0) - sc.smooth_cost(wm, margin, beta, 1.0)) / (2 * h)
        assert abs(g[i, d] - fd) <= 1e-5 * max(1.0, abs(fd)), (i, d, g[i, d], fd)


PLANS = settings(max_examples=12, deadline=None, derandomize=True)


@PLANS
@given(kind=st.sampled_from(["spheres16", "tabletop", "uneven"]), seed=st.integers(0, 10**6))
def test_oracle_planner_paths_join_start_to_goal_and_revalidate(orc, kind, seed):
    """Whenever the sequential restatement of the planner solves a random
    problem, its path runs from the start to one of the goals and re-validates
    at 0.01 rad under the rules the GPU planner's paths are held to."""
    from conftest import make_problem

    pr = make_problem(kind, seed)
    sc = orc.Scene(pr.context, pr.dim)
    r = orc.plan(sc, pr.start, pr.goals, pr.lower, pr.upper, max_iterations=1000, num_new_samples=16,
                 max_nodes=pr.max_nodes, collision_mode=3, edge_resolution=0.01)
    if r.solved != 1:
        assert r.path is None
        return
    assert np.array_equal(r.path[0], pr.start) and any(np.array_equal(r.path[-1], g) for g in pr.goals)
    ok, md = sc.validate_planned_path(r.path, 16, 0.01)
    assert ok, md


@PLANS
@given(kind=st.sampled_from(["spheres16", "tabletop", "uneven"]), seed=st.integers(0, 10**6),
       rseed=st.integers(0, 2**31 - 1))
def test_host_loop_paths_are_free_on_their_own_edge_waypoints(orc, kind, seed, rseed):
    """Whenever the host-driven loop (the CPU baseline) solves a random problem,
    its path runs from the start to the goal, and every vertex and every one of
    the 16 waypoints per edge it checked is free (within 1e-5 m: float32
    against float64)."""
    from conftest import make_problem

    pr = make_problem(kind, seed)
    sc = orc.Scene(pr.context, pr.dim)
    r = orc.rrtc_host_plan(sc, pr.start, pr.goals[0], pr.lower, pr.upper, max_iterations=300,
                           num_new_samples=32, seed=rseed)
    if not r.solved:
        return
    p = r.path
    assert np.array_equal(p[0], pr.start) and np.array_equal(p[-1], pr.goals[0])
    pts = np.concatenate([p] + [orc.edge_waypoints(p[i], p[i + 1], 16, 0.0) for i in range(p.shape[0] - 1)])
    assert sc.min_distances(pts).min() >= -1e-5


@FAST
@given(costs=st.lists(st.floats(0.0, 1e3, allow_nan=False), max_size=300), world=st.integers(1, 8))
def test_lpt_split_takes_every_problem_once_within_the_list_scheduling_bound(costs, world):
    parts = lpt_partition(costs, world)
    assert len(parts) == world
    got = np.sort(np.concatenate(parts)) if parts else np.zeros(0, np.int64)
    assert np.array_equal(got, np.arange(len(costs)))
    if costs:
        c = np.asarray(costs, np.float64)
        loads = [c[p].sum() for p in parts]
        assert max(loads) <= c.sum() / world + c.max() + 1e-9
