"""Point-cloud collision checking (the point-cloud edge validation of
cuda-rrtc/jax/prrtc_robogpu.py:183-191): the device hash grid against the
oracle's brute-force sphere-vs-point test, in the edge checker, the batched
checker and both planners."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import make_problem

pytestmark = pytest.mark.gpu


def _cloud_only(ctx, pts, r_env):
    """The robot of ctx with only a point cloud as its world (no self pairs)."""
    c = {k: v for k, v in ctx.items() if k.startswith(("fk_", "sphere_", "coarse_", "fine_", "self_pair_ranges"))}
    c["point_cloud"], c["r_env"] = pts, r_env
    return c


def _exclusion(sc, q, thr=0.0):
    md = sc.min_distances(q)
    return np.abs(md - thr) > 1e-4


@pytest.mark.parametrize("n_buckets", [0, 1024])
def test_edges_cloud_only_match_oracle(cuda, orc, n_buckets):
    from prrtc_b200.pointcloud import PointCloud, PointCloudChecker

    pr = make_problem("pointcloud", 3)
    rng = np.random.default_rng(5)
    pts = pr.context["point_cloud"]
    ctx = _cloud_only(pr.context, pts, 0.015)
    sc = orc.Scene(ctx, pr.dim)
    S, G = 96, 8
    a = rng.uniform(pr.lower, pr.upper, (S, pr.dim)).astype(np.float32)
    b = (a + rng.normal(0, 0.15, (S, pr.dim))).astype(np.float32)
    ts = np.linspace(0.0, 1.0, G, dtype=np.float32)
    edges = (a[:, None] * (1 - ts)[None, :, None] + b[:, None] * ts[None, :, None]).astype(np.float32)
    chk = PointCloudChecker(ctx, pr.dim)
    cloud = PointCloud(pts, 0.015, n_buckets=n_buckets)
    free = chk.check_edges_collision_free(edges, point_cloud=cloud, r_env=0.015).cpu().numpy()
    w = edges.reshape(-1, pr.dim)
    ora = sc.check_configs(w, 0).reshape(S, G)
    far = _exclusion(sc, w).reshape(S, G).all(1)
    assert far.mean() > 0.9
    assert np.array_equal(free[far], (ora[far].sum(1) == 0).astype(np.int32))
    assert 0.05 < free.mean() < 0.95  # both outcomes occur


@pytest.mark.parametrize("mode", [0, 1, 3])
def test_configs_with_world_and_cloud_match_oracle(cuda, orc, mode):
    from prrtc_b200.collision import CollisionChecker

    pr = make_problem("pointcloud", 4)
    rng = np.random.default_rng(6)
    q = rng.uniform(pr.lower, pr.upper, (600, pr.dim)).astype(np.float32)
    names = ["binary", "differentiable", "binary_coarse", "binary_coarse_coop"]
    mine = CollisionChecker(pr.context, pr.dim, names[mode], 0.02).check(q).cpu().numpy()
    sc = orc.Scene(pr.context, pr.dim)
    ora = sc.check_configs(q, mode, 0.02)
    far = _exclusion(sc, q, 0.02 if mode == 1 else 0.0)
    assert far.mean() > 0.95
    assert np.array_equal(mine[far], ora[far])


def test_cloud_edge_cases(cuda, orc):
    """Points beyond +-1e4 m are ignored; an empty cloud is no cloud; one bucket
    for every point (all hash collisions) gives the same verdicts."""
    from prrtc_b200.pointcloud import PointCloud, PointCloudChecker

    pr = make_problem("pointcloud", 5)
    rng = np.random.default_rng(8)
    pts = pr.context["point_cloud"][:4000]
    far_pts = np.concatenate([pts, np.array([[2e4, 0, 0], [0, -3e4, 0], [np.inf, 0, 0]], np.float32)])
    ctx = _cloud_only(pr.context, pts, 0.02)
    chk = PointCloudChecker(ctx, pr.dim)
    q = rng.uniform(pr.lower, pr.upper, (400, 1, pr.dim)).astype(np.float32)
    base = chk.check_edges_collision_free(q, point_cloud=PointCloud(pts, 0.02)).cpu().numpy()
    extra = chk.check_edges_collision_free(q, point_cloud=PointCloud(far_pts, 0.02)).cpu().numpy()
    assert np.array_equal(base, extra)
    one = chk.check_edges_collision_free(q, point_cloud=PointCloud(pts, 0.02, n_buckets=1)).cpu().numpy()
    assert np.array_equal(base, one)
    fine = chk.check_edges_collision_free(q, point_cloud=PointCloud(pts, 0.02, cell=0.04)).cpu().numpy()
    assert np.array_equal(base, fine)
    empty = chk.check_edges_collision_free(q, point_cloud=PointCloud(np.zeros((0, 3), np.float32), 0.02))
    assert empty.cpu().numpy().tolist() == [1] * q.shape[0]  # nothing else in this world
    sc = orc.Scene(ctx, pr.dim)
    ora = sc.check_configs(q.reshape(-1, pr.dim), 0)
    far = _exclusion(sc, q.reshape(-1, pr.dim))
    assert np.array_equal(base[far], 1 - ora[far])


def test_plan_against_point_cloud_revalidates(cuda, orc):
    """The single-kernel planner with the cloud checked inside the kernel."""
    from prrtc_b200 import prrtc_plan

    pr = make_problem("pointcloud", 6)
    r = prrtc_plan(pr.start, pr.goals, max_iterations=10000, num_new_samples=64, max_nodes=65536,
                   min_vals=pr.lower, max_vals=pr.upper, collision_context=pr.context,
                   collision_checker="binary_coarse_coop", edge_resolution=0.01)
    assert r.solved
    path = r.path.cpu().numpy()
    ok, md = orc.Scene(pr.context, pr.dim).validate_path(path, 0.01)
    assert ok, md


def test_batch_plan_shared_cloud(cuda, orc):
    from prrtc_b200 import prrtc_plan_batch
    from prrtc_b200.pointcloud import PointCloud

    probs = [make_problem("pointcloud", 20 + i) for i in range(4)]
    # one shared cloud: plan every problem in problem 0's scene
    ctx = probs[0].context
    sc = orc.Scene(ctx, probs[0].dim)
    starts, goals = [], []
    for p in probs:
        if sc.in_collision(p.start) or sc.in_collision(p.goals[0]):
            continue
        starts.append(p.start)
        goals.append(p.goals[:1])
    starts.append(probs[0].start)
    goals.append(probs[0].goals[:1])
    cloud = PointCloud(ctx["point_cloud"], ctx["r_env"])
    world = {k: v for k, v in ctx.items() if k not in ("point_cloud", "r_env")}
    res = prrtc_plan_batch(np.stack(starts), np.stack(goals), max_iterations=10000, num_new_samples=32,
                           max_nodes=32768, min_vals=probs[0].lower, max_vals=probs[0].upper,
                           collision_context=[world] * len(starts), collision_checker="binary_coarse_coop",
                           edge_resolution=0.01, point_cloud=cloud)
    assert sum(r.solved for r in res) >= len(starts) - 1
    for r in res:
        if r.solved:
            ok, md = sc.validate_path(r.path.cpu().numpy(), 0.01)
            assert ok, md


def test_host_driven_planner_with_point_cloud(cuda, orc):
    """prrtc_plan_robogpu: host loop, batched edge checks on the device."""
    from prrtc_b200.pointcloud import PointCloudChecker, prrtc_plan_robogpu

    pr = make_problem("pointcloud", 7)
    world = {k: v for k, v in pr.context.items() if k not in ("point_cloud", "r_env")}
    chk = PointCloudChecker(world, pr.dim)
    r = prrtc_plan_robogpu(pr.start, pr.goals, world, chk, point_cloud=pr.context["point_cloud"],
                           r_env=pr.context["r_env"], max_iterations=400, num_new_samples=64, granularity=32,
                           max_nodes=50000, min_vals=pr.lower, max_vals=pr.upper, seed=1)
    assert r.solved
    path = r.path.numpy()
    assert np.array_equal(path[0], pr.start) and np.array_equal(path[-1], pr.goals[0])
    # every vertex of the path is collision free in the oracle (the edges were
    # checked at the host planner's own 32 waypoints, not at a fixed resolution)
    sc = orc.Scene(pr.context, pr.dim)
    assert not sc.check_configs(path.astype(np.float32), 0).any()
