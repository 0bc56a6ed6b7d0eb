"""CPU tests of the oracle: sampling, nearest neighbour, extend, FK, primitive
distances, checker equivalences and the two planner restatements."""
from __future__ import annotations

from fractions import Fraction

import numpy as np
import pytest

from conftest import make_problem
from prrtc_b200.context import RobotModel, build_collision_context, empty_world

PRIMES = [3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59]


def radical_inverse(n: int, b: int) -> Fraction:
    r, f = Fraction(0), Fraction(1, b)
    while n > 0:
        r += f * (n % b)
        n //= b
        f /= b
    return r


@pytest.mark.parametrize("base", [3, 5, 7, 59])
def test_halton_matches_radical_inverse(orc, base):
    state = 1
    for n in range(1, 400):
        v, state = orc.halton_next(base, state)
        assert state == n + 1
        assert abs(v - float(radical_inverse(n, base))) <= 4e-7


def test_prime_order_restates_lcg_shuffle(orc):
    assert orc.prime_order(0).tolist() == PRIMES
    for e in (1, 2, 3, 100, 127, 4095):
        p = list(PRIMES)
        rng = (e * 1664525 + 1013904223) & 0xFFFFFFFF
        for i in range(15, 0, -1):
            rng = (rng * 1664525 + 1013904223) & 0xFFFFFFFF
            j = rng % (i + 1)
            p[i], p[j] = p[j], p[i]
        got = orc.prime_order(e).tolist()
        assert got == p and sorted(got) == PRIMES


def test_halton_samples_shape_and_range(orc):
    lo = np.full(7, -2.8, np.float32)
    hi = np.full(7, 2.8, np.float32)
    s = orc.halton_samples(3, 500, lo, hi)
    assert s.shape == (500, 7) and (s >= lo).all() and (s <= hi).all()
    # one shared index stream: dimension d of sample k is radical_inverse(k+1, prime_order[d])
    po = orc.prime_order(3)
    for k in (0, 10, 499):
        for d in range(7):
            want = float(lo[d]) + float(radical_inverse(k + 1, int(po[d]))) * (float(hi[d]) - float(lo[d]))
            assert abs(s[k, d] - want) < 2e-6


def test_nearest_lowest_index_and_nan_skip(orc):
    rng = np.random.default_rng(0)
    dim, N = 7, 1000
    t = rng.uniform(-1, 1, (dim, N)).astype(np.float32)
    q = rng.uniform(-1, 1, dim).astype(np.float32)
    i, d = orc.nearest(t, N, q)
    dd = ((t - q[:, None]) ** 2).sum(0)
    assert i == int(np.argmin(dd)) and abs(d - dd[i]) < 1e-5
    t2 = np.concatenate([t[:, :10]] * 3, 1)
    i2, _ = orc.nearest(t2, 30, t[:, 7])
    assert i2 == 7
    t3 = t.copy()
    t3[:, i] = np.nan
    i3, _ = orc.nearest(t3, N, q)
    assert i3 != i and i3 == int(np.argmin(np.where(np.isnan(dd * 0 + t3[0]), np.inf, dd)))


def test_extend_and_waypoints(orc):
    base = np.zeros(7, np.float32)
    sample = np.full(7, 1.0, np.float32)
    nd = float(np.sqrt(np.float32(7.0)))
    cand = orc.extend(base, sample, nd, 0.5)
    assert abs(np.linalg.norm(cand) - 0.5) < 1e-6
    cand2 = orc.extend(base, sample, nd, 100.0)
    assert np.array_equal(cand2, sample)
    w = orc.edge_waypoints(base, cand, 16)
    assert w.shape == (16, 7) and np.allclose(w[-1], cand) and np.allclose(w[0], cand / 16)
    w2 = orc.edge_waypoints(base, cand, 16, 0.01)
    assert w2.shape == (50, 7)


def _fk_numpy(rob: RobotModel, q: np.ndarray) -> np.ndarray:
    """Independent product-of-exponentials FK (scalar loops, float64)."""
    def quat(wxyz):
        w, x, y, z = wxyz / np.linalg.norm(wxyz)
        return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                         [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                         [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])

    def expm_twist(tw, v):
        # 4x4 matrix exponential by scaling and squaring of the twist matrix
        X = np.zeros((4, 4))
        w = np.asarray(tw[3:], float) * v
        X[:3, :3] = [[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]]
        X[:3, 3] = np.asarray(tw[:3], float) * v
        E, term = np.eye(4), np.eye(4)
        Xs = X / 64.0
        for k in range(1, 30):
            term = term @ Xs / k
            E = E + term
        for _ in range(6):
            E = E @ E
        return E

    J = rob.n_joints
    W = [None] * J
    for j in range(J):
        P = np.eye(4)
        P[:3, :3] = quat(rob.parent_tf[j, :4].astype(float))
        P[:3, 3] = rob.parent_tf[j, 4:]
        if rob.mimic_act_idx[j] >= 0:
            v = rob.mimic_mul[j] * q[rob.mimic_act_idx[j]] + rob.mimic_off[j]
        elif rob.act_idx[j] >= 0:
            v = q[rob.act_idx[j]]
        else:
            v = 0.0
        L = P @ expm_twist(rob.twists[j], v)
        W[j] = L if rob.parent_idx[j] < 0 else W[rob.parent_idx[j]] @ L
    return np.stack([np.concatenate([W[rob.topo_inv[k]][:3, :3].ravel(), W[rob.topo_inv[k]][:3, 3]])
                     for k in range(J)])


@pytest.mark.parametrize("which", ["arm", "dual"])
def test_fk_f64_matches_independent_expm(orc, which, arm, dual):
    rob = arm if which == "arm" else dual
    ctx = build_collision_context(rob, None)
    sc = orc.Scene(ctx, rob.dim)
    rng = np.random.default_rng(1)
    for _ in range(20):
        q = rng.uniform(rob.lower, rob.upper).astype(np.float64)
        assert np.abs(sc.fk(q) - _fk_numpy(rob, q)).max() < 1e-9
        f32 = sc.fk(q.astype(np.float32), f64=False)
        assert np.abs(f32 - sc.fk(q.astype(np.float32).astype(np.float64))).max() < 1e-5


def _one_sphere_scene(centre, r, world):
    rob = RobotModel(
        twists=np.zeros((1, 6), np.float32), parent_tf=np.array([[1, 0, 0, 0, *centre]], np.float32),
        parent_idx=np.array([-1], np.int32), act_idx=np.array([-1], np.int32),
        mimic_mul=np.ones(1, np.float32), mimic_off=np.zeros(1, np.float32),
        mimic_act_idx=np.array([-1], np.int32), topo_inv=np.array([0], np.int32),
        lower=np.array([-1.0], np.float32), upper=np.array([1.0], np.float32),
        sphere_frame=np.array([0], np.int32), sphere_local=np.zeros((1, 3), np.float32),
        sphere_radius=np.array([r], np.float32), link_pairs=[])
    return build_collision_context(rob, world)


def _box_distance_bruteforce(p, box):
    c, R, h = box[:3], np.stack([box[3:6], box[6:9], box[9:12]], 1), box[12:15]
    local = R.T @ (p - c)
    q = np.abs(local) - h
    return np.linalg.norm(np.maximum(q, 0)) + min(q.max(), 0.0)


def test_primitive_distances_against_geometry(orc):
    rng = np.random.default_rng(2)
    for _ in range(200):
        p = rng.uniform(-1, 1, 3)
        r = float(rng.uniform(0.01, 0.1))
        # sphere
        o = np.concatenate([rng.uniform(-1, 1, 3), [rng.uniform(0.05, 0.3)]]).astype(np.float32)
        w = empty_world(); w["world_spheres"] = o[None]
        d = orc.Scene(_one_sphere_scene(p, r, w), 1).min_distance([0.0])
        pf = p.astype(np.float32).astype(np.float64)
        assert abs(d - (np.linalg.norm(pf - o[:3]) - r - o[3])) < 1e-5
        # capsule: brute force over the segment
        a, b = rng.uniform(-1, 1, 3), rng.uniform(-1, 1, 3)
        rc = rng.uniform(0.01, 0.2)
        cap = np.array([*a, *b, rc], np.float32)
        w = empty_world(); w["world_capsules"] = cap[None]
        d = orc.Scene(_one_sphere_scene(p, r, w), 1).min_distance([0.0])
        ts = np.linspace(0, 1, 20001)
        seg = cap[:3][None] + ts[:, None] * (cap[3:6] - cap[:3])[None]
        bf = np.linalg.norm(seg - pf, axis=1).min() - r - rc
        assert abs(d - bf) < 1e-4
        # oriented box
        yaw = rng.uniform(-np.pi, np.pi)
        cy, sy = np.cos(yaw), np.sin(yaw)
        box = np.array([*rng.uniform(-1, 1, 3), cy, sy, 0, -sy, cy, 0, 0, 0, 1, *rng.uniform(0.02, 0.3, 3)],
                       np.float32)
        w = empty_world(); w["world_boxes"] = box[None]
        d = orc.Scene(_one_sphere_scene(p, r, w), 1).min_distance([0.0])
        assert abs(d - (_box_distance_bruteforce(pf, box.astype(np.float64)) - r)) < 1e-5
        # halfspace
        n = rng.normal(size=3); n /= np.linalg.norm(n)
        hs = np.array([*n, *rng.uniform(-1, 1, 3)], np.float32)
        w = empty_world(); w["world_halfspaces"] = hs[None]
        d = orc.Scene(_one_sphere_scene(p, r, w), 1).min_distance([0.0])
        assert abs(d - (hs[:3].astype(float) @ (pf - hs[3:6]) - r)) < 1e-5


@pytest.mark.parametrize("kind", ["spheres16", "tabletop", "uneven"])
def test_checker_modes_agree(orc, kind):
    pr = make_problem(kind, 3)
    sc = orc.Scene(pr.context, pr.dim)
    rng = np.random.default_rng(4)
    q = rng.uniform(pr.lower, pr.upper, (400, pr.dim)).astype(np.float32)
    md = sc.min_distances(q)
    v0 = sc.check_configs(q, 0)
    assert np.array_equal(v0, (md <= 0).astype(np.int32))
    for mode in (2, 3):
        assert np.array_equal(sc.check_configs(q, mode), v0)
    v1 = sc.check_configs(q, 1, 0.02)
    band = np.abs(md - 0.02) > 1e-6
    assert np.array_equal(v1[band], (md[band] < 0.02).astype(np.int32))


def test_coarse_model_encloses_fine(arm, dual):
    for rob in (arm, dual):
        ctx = build_collision_context(rob, None)
        off = ctx["fine_link_offsets"]
        assert off[0] == 0 and off[-1] == ctx["sphere_radius"].shape[0]
        for k in range(ctx["coarse_sphere_link_idx"].shape[0]):
            s, e = off[k], off[k + 1]
            assert (ctx["sphere_link_idx"][s:e] == ctx["coarse_sphere_link_idx"][k]).all()
            # exactly: float64 arithmetic on the stored float32 values
            d = np.linalg.norm(ctx["sphere_local"][s:e].astype(np.float64) -
                               ctx["coarse_sphere_local"][k].astype(np.float64), axis=1) + \
                ctx["sphere_radius"][s:e].astype(np.float64)
            assert (d <= float(ctx["coarse_sphere_radius"][k])).all()
        rng = ctx["self_pair_ranges"]
        assert rng[0, 0] == 0 and (rng[1:, 0] == rng[:-1, 1]).all() and rng[-1, 1] == ctx["self_pairs"].shape[0]


def test_workload_shapes(arm, dual):
    c1 = build_collision_context(arm, None)
    assert c1["sphere_radius"].shape == (56,) and c1["self_pairs"].shape == (960, 2)
    assert c1["coarse_sphere_link_idx"].shape == (7,) and c1["coarse_self_pairs"].shape == (15, 2)
    c5 = build_collision_context(dual, None)
    assert dual.n_joints == 18 and dual.dim == 14 and c5["sphere_radius"].shape == (120,)
    assert (dual.mimic_act_idx >= 0).sum() == 4
    p2 = make_problem("tabletop", 0)
    assert p2.context["world_boxes"].shape == (20, 15) and p2.context["world_capsules"].shape == (8, 7)
    assert p2.context["world_spheres"].shape == (32, 4) and p2.context["world_halfspaces"].shape == (1, 6)
    assert p2.goals.shape == (4, 7)


@pytest.mark.parametrize("kind,seed", [("spheres16", 0), ("tabletop", 1), ("uneven", 2)])
def test_sequential_prrtc_solves_and_revalidates(orc, kind, seed):
    pr = make_problem(kind, seed)
    sc = orc.Scene(pr.context, pr.dim)
    r = orc.plan(sc, pr.start, pr.goals, pr.lower, pr.upper, max_iterations=3000, num_new_samples=32,
                 max_nodes=pr.max_nodes, collision_mode=3, edge_resolution=0.01)
    assert r.solved == 1
    assert np.array_equal(r.path[0], pr.start) and any(np.array_equal(r.path[-1], g) for g in pr.goals)
    ok, md = sc.validate_path(r.path, 0.01)
    assert ok, md
    r2 = orc.plan(sc, pr.start, pr.goals, pr.lower, pr.upper, max_iterations=3000, num_new_samples=32,
                  max_nodes=pr.max_nodes, collision_mode=3, edge_resolution=0.01)
    assert r2.tree_sizes == r.tree_sizes and r2.connection == r.connection  # sequential => deterministic


def test_validate_planned_path_rules(orc, arm):
    """validate_planned_path.  A 0.12 rad edge: the planner checks it at 16
    waypoints (t = k/16, granularity 16), an independent 0.01 rad grid at 12 (t =
    k/12).  A small world sphere grazing the fastest robot sphere at t = 5/12 by
    20 um -- free at every planner waypoint -- fails the independent grid, passes
    as a shallow graze, and fails when graze_depth is below its depth; a sphere
    on the path fails outright."""
    from prrtc_b200.context import build_collision_context

    dim = arm.dim
    empty = build_collision_context(arm, {})
    sc0 = orc.Scene(empty, dim)
    q0 = np.zeros(dim, np.float32)
    q0[1], q0[3] = 1.2, -0.5  # arm stretched out: the base joint sweeps its far spheres
    q1 = q0.copy()
    q1[0] = np.float32(0.12)
    sli, sloc, srad = empty["sphere_link_idx"], empty["sphere_local"], empty["sphere_radius"]

    def centres(q):
        F = sc0.fk(np.asarray(q, np.float32))
        return np.stack([F[l, :9].reshape(3, 3) @ sloc[i] + F[l, 9:12] for i, l in enumerate(sli)])

    def at(t):
        return q0 + np.float32(t) * (q1 - q0)

    s = int(np.argmax(np.linalg.norm(centres(q1) - centres(q0), axis=1)))
    tg, rho, depth = 5.0 / 12.0, 0.01, 2e-5
    cg = centres(at(tg))[s]
    v = centres(at(tg + 1e-3))[s] - centres(at(tg - 1e-3))[s]
    u = np.cross(v, [0.0, 0.0, 1.0])
    u /= np.linalg.norm(u)
    o = cg + u * (srad[s] + rho - depth)
    sc = orc.Scene(build_collision_context(arm, {"world_spheres": np.array([[*o, rho]], np.float32)}), dim)
    path = np.stack([q0, q1])
    planner = orc.edge_waypoints(q0, q1, 16, 0.01)
    assert planner.shape[0] == 16 and sc.min_distances(planner).min() > 0.0
    assert sc.min_distances(at(tg)[None])[0] < -depth / 2
    assert sc0.validate_planned_path(path)[0]
    assert not sc.validate_path(path, 0.01)[0]
    ok, md = sc.validate_planned_path(path)
    assert ok and -2 * depth < md < 0.0
    assert not sc.validate_planned_path(path, graze_depth=depth / 2)[0]
    hit = orc.Scene(build_collision_context(arm, {"world_spheres": np.array([[*cg, 0.05]], np.float32)}), dim)
    assert not hit.validate_planned_path(path)[0]


def test_sequential_prrtc_overflow_and_iteration_limit(orc):
    pr = make_problem("tabletop", 5)
    sc = orc.Scene(pr.context, pr.dim)
    r = orc.plan(sc, pr.start, pr.goals, pr.lower, pr.upper, max_iterations=2, num_new_samples=1,
                 max_nodes=65536, collision_mode=0)
    assert r.solved in (1, -1)
    if r.solved == -1:
        assert r.iter_count == 3
    r = orc.plan(sc, pr.start, pr.goals, pr.lower, pr.upper, max_iterations=1000, num_new_samples=8,
                 max_nodes=6, collision_mode=0)
    assert r.solved in (1, -1)
    if r.solved == -1:
        assert r.tree_sizes[0] > 6 or r.tree_sizes[1] > 6


def test_host_rrtc_solves(orc):
    pr = make_problem("spheres16", 0)
    sc = orc.Scene(pr.context, pr.dim)
    r = orc.rrtc_host_plan(sc, pr.start, pr.goals, pr.lower, pr.upper, max_iterations=200, num_new_samples=32,
                           seed=0)
    assert r.solved and r.path is not None
    assert np.array_equal(r.path[0], pr.start) and np.array_equal(r.path[-1], pr.goals[0])
    r4 = orc.rrtc_host_plan(sc, pr.start, pr.goals, pr.lower, pr.upper, max_iterations=200, num_new_samples=32,
                            seed=0, n_threads=4)
    assert r4.solved == r.solved and r4.iterations == r.iterations and abs(r4.cost - r.cost) < 1e-6


def test_smooth_cost_finite_difference_consistency(orc):
    pr = make_problem("spheres16", 0)
    sc = orc.Scene(pr.context, pr.dim)
    w = np.linspace(pr.start, pr.goals[0], 8).astype(np.float64)
    c = sc.smooth_cost(w, 0.02, 50.0, 1.0)
    assert np.isfinite(c) and c > 0
    w2 = w.copy(); w2[3, 2] += 1e-3
    assert sc.smooth_cost(w2, 0.02, 50.0, 1.0) != c


def test_point_cloud_stage_brute_force(orc, arm):
    """The oracle's point-cloud stage: a sphere hits a point iff |c - p| <= r + r_env."""
    from prrtc_b200.scenes import box_surface_points

    rng = np.random.default_rng(3)
    boxes = np.array([[0.5, 0.0, 0.5, 1, 0, 0, 0, 1, 0, 0, 0, 1, 0.2, 0.3, 0.1]], np.float32)
    pts = box_surface_points(rng, boxes, 3000)
    # every point on the box surface: one local coordinate at +-half-length
    loc = np.abs(pts - boxes[0, :3]) / boxes[0, 12:15]
    assert np.allclose(loc.max(1), 1.0, atol=1e-5) and (loc <= 1.0 + 1e-5).all()
    ctx = build_collision_context(arm, empty_world())
    for k in ("self_pairs",):
        ctx.pop(k, None)
    ctx["point_cloud"], ctx["r_env"] = pts, 0.02
    sc = orc.Scene(ctx, arm.dim)
    q = rng.uniform(arm.lower, arm.upper, (60, arm.dim)).astype(np.float32)
    v = sc.check_configs(q, 0)
    md = sc.min_distances(q)
    for i in range(q.shape[0]):
        F = sc.fk(q[i])  # [J, 12]
        c = np.einsum("sij,sj->si", F[ctx["sphere_link_idx"], :9].reshape(-1, 3, 3), ctx["sphere_local"]) + \
            F[ctx["sphere_link_idx"], 9:]
        d = np.linalg.norm(c[:, None, :] - pts[None].astype(np.float64), axis=-1) - ctx["sphere_radius"][:, None] - 0.02
        assert abs(d.min() - md[i]) < 1e-6
        if abs(d.min()) > 1e-6:
            assert v[i] == int(d.min() <= 0)
    assert 0 < v.sum() < q.shape[0]


@pytest.mark.parametrize("kind,seed", [("tabletop", 3), ("spheres16", 1), ("uneven", 7), ("large", 5)])
def test_autodiff_reference_matches_oracle_cost_and_differences(orc, kind, seed):
    """The autograd restatement of the smoothing cost (the stand-in for a
    jax.grad reference) agrees with the C oracle's cost, and its gradient with
    central differences of that cost."""
    from oracle.smooth_autodiff import smooth_grad

    pr = make_problem(kind, seed)
    sc = orc.Scene(pr.context, pr.dim)
    rng = np.random.default_rng(seed)
    w = np.linspace(pr.start, pr.goals[0], 6).astype(np.float64) + rng.normal(0, 0.05, (6, pr.dim))
    c, g = smooth_grad(pr.context, w, 0.02, 50.0, 1.0)
    c64 = sc.smooth_cost(w, 0.02, 50.0, 1.0)
    assert abs(c - c64) <= 1e-9 * max(1.0, abs(c64))
    h = 1e-5
    for i, d in [(1, 0), (2, 3), (4, 6), (3, 1), (2, pr.dim - 1)]:
        wp, wm = w.copy(), w.copy()
        wp[i, d] += h
        wm[i, d] -= h
        fd = (sc.smooth_cost(wp, 0.02, 50.0, 1.0) - sc.smooth_cost(wm, 0.02, 50.0, 1.0)) / (2 * h)
        assert abs(g[i, d] - fd) <= 1e-5 * max(1.0, abs(fd)), (i, d, g[i, d], fd)
