"""Seeded synthetic robots, worlds and planning problems.

The reference evaluates on MotionBenchMaker / VAMP problem sets loaded from
PyRoFFI resources (evaluate_mbm.py:251-263), which are not available.  These
generators stand in for them with the shapes, counts and value ranges of the
benchmark workloads:

* ``arm``       -- 7 revolute joints, axes alternating z / y, parent offsets
                   U(0.08, 0.33) m along z, limits +-2.8 rad, 8 spheres per link
                   (r ~ U(0.04, 0.08), centres within +-0.05 m of the link
                   segment), self pairs between every two links >= 2 apart.
* ``dual_arm``  -- two such chains on a shared base 0.6 m apart, each with two
                   mimic finger joints (mimic_mul 1, mimic_off 0): 18 joints,
                   14 actuated, 120 spheres, within-arm and cross-arm self pairs.
* worlds        -- ``spheres_world`` (16 spheres in [-.8,.8]^2 x [0,1.2]),
                   ``tabletop_world`` (floor halfspace, table + 3-5 shelf slabs +
                   clutter boxes, capsules, spheres), ``uneven_world`` (4-128
                   spheres, 0-32 boxes), ``dense_world`` (the same counts at the
                   16-sphere scene's density, larger boxes), ``large_world`` (256 spheres, 64 boxes,
                   floor).

Start and goal configurations are rejection-sampled collision free by a caller
supplied ``checker(configs [n,dim]) -> verdicts [n]`` (the GPU checker in
production, the oracle in CPU tests), so the generators carry no checker of
their own.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable

import numpy as np

from .context import RobotModel, build_collision_context, empty_world

Checker = Callable[[np.ndarray, dict], np.ndarray]

ARM_LIMIT = 2.8


def _arm_tables(rng, n_joints, base_xyz, first_offset_min=0.0):
    offs = rng.uniform(0.08, 0.33, size=n_joints + 1).astype(np.float64)
    offs[0] = max(offs[0], first_offset_min)
    twists = np.zeros((n_joints, 6), np.float32)
    ptf = np.zeros((n_joints, 7), np.float32)
    for j in range(n_joints):
        twists[j, 3:] = (0.0, 0.0, 1.0) if j % 2 == 0 else (0.0, 1.0, 0.0)
        ptf[j, 0] = 1.0
        ptf[j, 6] = offs[j]
    ptf[0, 4:7] = np.asarray(base_xyz, np.float64) + np.array([0.0, 0.0, offs[0]])
    return offs, twists, ptf


def _link_spheres(rng, length, n=8, jitter=0.05):
    """n spheres whose centres lie within `jitter` of the segment (0,0,0)-(0,0,length)."""
    s = rng.uniform(0.0, length, size=n)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    off = d * (jitter * rng.uniform(0.0, 1.0, size=(n, 1)) ** (1.0 / 3.0))
    centres = np.stack([np.zeros(n), np.zeros(n), s], 1) + off
    radii = rng.uniform(0.04, 0.08, size=n)
    return centres.astype(np.float32), radii.astype(np.float32)


def _floor_clear_offset(rng_state_offsets, centres0, radii0):
    """Height the base must be raised so link-0 spheres stay above z = 0."""
    low = float(np.min(centres0[:, 2] - radii0))
    return max(0.0, 0.01 - low)


def _straight_pose_clearance(robot: RobotModel) -> float:
    """Smallest self-pair distance with every joint at 0 (all frames translate along z)."""
    z = np.cumsum(robot.parent_tf[:, 6].astype(np.float64))
    centres = robot.sphere_local.astype(np.float64).copy()
    centres[:, 2] += z[robot.sphere_frame]
    centres[:, :2] += robot.parent_tf[0, 4:6]
    best = np.inf
    for fi, fj in robot.link_pairs:
        a, b = robot.sphere_frame == fi, robot.sphere_frame == fj
        d = np.linalg.norm(centres[a][:, None] - centres[b][None], axis=-1)
        d -= robot.sphere_radius[a][:, None] + robot.sphere_radius[b][None]
        best = min(best, float(d.min()))
    return best


def arm(seed: int = 0, n_joints: int = 7) -> RobotModel:
    """Synthetic serial arm (the robot of the single-arm workloads).

    Draws robots from seeds ``seed, seed+1000, ...`` and keeps the first whose
    straight pose (q = 0) has every self pair at least 2 cm apart, the same
    structural requirement the reference's evaluation applies to its robots
    (no self pair in collision at q = 0, evaluate_mbm.py:70-224).
    """
    for attempt in range(1000):
        rob = _arm_draw(seed + 1000 * attempt, n_joints)
        if _straight_pose_clearance(rob) >= 0.02:
            return rob
    raise RuntimeError("no self-collision-free arm found")


def _arm_draw(seed: int, n_joints: int) -> RobotModel:
    rng = np.random.default_rng(seed)
    offs, twists, ptf = _arm_tables(rng, n_joints, (0.0, 0.0, 0.0))
    centres, radii, frames = [], [], []
    for j in range(n_joints):
        c, r = _link_spheres(rng, offs[j + 1])
        centres.append(c)
        radii.append(r)
        frames.append(np.full(8, j, np.int32))
    # keep the base link clear of a floor at z = 0 (link 0 only spins about z)
    lift = _floor_clear_offset(None, centres[0] + np.array([0, 0, offs[0]], np.float32), radii[0])
    ptf[0, 6] += lift
    pairs = [(i, j) for i in range(n_joints) for j in range(i + 2, n_joints)]
    J = n_joints
    return RobotModel(
        twists=twists, parent_tf=ptf,
        parent_idx=np.arange(-1, J - 1, dtype=np.int32),
        act_idx=np.arange(J, dtype=np.int32),
        mimic_mul=np.ones(J, np.float32), mimic_off=np.zeros(J, np.float32),
        mimic_act_idx=np.full(J, -1, np.int32), topo_inv=np.arange(J, dtype=np.int32),
        lower=np.full(J, -ARM_LIMIT, np.float32), upper=np.full(J, ARM_LIMIT, np.float32),
        sphere_frame=np.concatenate(frames), sphere_local=np.concatenate(centres),
        sphere_radius=np.concatenate(radii), link_pairs=pairs,
    )


def dual_arm(seed: int = 0) -> RobotModel:
    """Two 7-DOF arm chains 0.6 m apart, each with two mimic finger joints (the dual-arm workload)."""
    single = arm(seed)
    J1 = single.n_joints
    twists, ptf, parent, act, mm, mo, mact = [], [], [], [], [], [], []
    centres, radii, frames = [], [], []
    pairs = []
    rng = np.random.default_rng(seed + 1000)
    arm_frames = []
    for a, y in enumerate((-0.3, 0.3)):
        base = len(parent)
        for j in range(J1):
            twists.append(single.twists[j])
            t = single.parent_tf[j].copy()
            if j == 0:
                t[5] += y
            ptf.append(t)
            parent.append(-1 if j == 0 else base + j - 1)
            act.append(a * J1 + j)
            mm.append(1.0); mo.append(0.0); mact.append(-1)
        # two fingers on the last link, revolute about the link's x axis, mimicking the wrist joint
        tool = float(np.max(single.sphere_local[single.sphere_frame == J1 - 1][:, 2]))
        for f, sx in enumerate((0.03, -0.03)):
            twists.append(np.array([0, 0, 0, 1.0, 0, 0], np.float32))
            ptf.append(np.array([1, 0, 0, 0, sx, 0.0, tool], np.float32))
            parent.append(base + J1 - 1)
            act.append(-1)
            mm.append(1.0); mo.append(0.0); mact.append(a * J1 + J1 - 1)
        frames_this = list(range(base, base + J1 + 2))
        arm_frames.append(frames_this)
        for j in range(J1):
            sel = single.sphere_frame == j
            centres.append(single.sphere_local[sel]); radii.append(single.sphere_radius[sel])
            frames.append(np.full(int(sel.sum()), base + j, np.int32))
        for f in range(2):
            c = np.stack([np.zeros(2), np.zeros(2), rng.uniform(0.0, 0.08, 2)], 1) + rng.uniform(-0.01, 0.01, (2, 3))
            centres.append(c.astype(np.float32))
            radii.append(rng.uniform(0.02, 0.03, 2).astype(np.float32))
            frames.append(np.full(2, base + J1 + f, np.int32))
        # within-arm pairs: links >= 2 apart along the chain (fingers count as link J1)
        for i in range(J1):
            for j in range(i + 2, J1):
                pairs.append((base + i, base + j))
        for f in range(2):
            for i in range(J1 - 2):
                pairs.append((base + i, base + J1 + f))
    for fa in arm_frames[0]:
        for fb in arm_frames[1]:
            pairs.append((fa, fb))
    J = len(parent)
    dim = 2 * J1
    return RobotModel(
        twists=np.asarray(twists, np.float32), parent_tf=np.asarray(ptf, np.float32),
        parent_idx=np.asarray(parent, np.int32), act_idx=np.asarray(act, np.int32),
        mimic_mul=np.asarray(mm, np.float32), mimic_off=np.asarray(mo, np.float32),
        mimic_act_idx=np.asarray(mact, np.int32), topo_inv=np.arange(J, dtype=np.int32),
        lower=np.full(dim, -ARM_LIMIT, np.float32), upper=np.full(dim, ARM_LIMIT, np.float32),
        sphere_frame=np.concatenate(frames), sphere_local=np.concatenate(centres),
        sphere_radius=np.concatenate(radii), link_pairs=pairs,
    )


# ----------------------------------------------------------------------------- worlds

BASE_KEEPOUT = 0.3  # obstacles never intersect the column |xy| < 0.3 m around the arm base


def _centres(rng, n, lo, hi, clearance, keepout=BASE_KEEPOUT):
    """n points uniform in [lo, hi] whose xy distance to a base column exceeds keep-out + clearance."""
    bases = _BASES
    out = np.zeros((0, 3))
    while out.shape[0] < n:
        c = rng.uniform(lo, hi, size=(max(4 * n, 16), 3))
        ok = np.ones(c.shape[0], bool)
        for bx, by in bases:
            ok &= np.hypot(c[:, 0] - bx, c[:, 1] - by) > keepout + clearance
        out = np.concatenate([out, c[ok]], 0)
    return out[:n]


_BASES = [(0.0, 0.0)]


def _spheres(rng, n, lo=(-0.8, -0.8, 0.0), hi=(0.8, 0.8, 1.2), r=(0.05, 0.15)):
    rr = rng.uniform(*r, size=(n, 1))
    c = _centres(rng, n, lo, hi, r[1])
    return np.concatenate([c, rr], 1).astype(np.float32)


def _yaw_box(c, yaw, hl):
    cy, sy = np.cos(yaw), np.sin(yaw)
    a1, a2, a3 = (cy, sy, 0.0), (-sy, cy, 0.0), (0.0, 0.0, 1.0)
    return np.array([*c, *a1, *a2, *a3, *hl], np.float32)


def _random_boxes(rng, n, lo, hi, hl=(0.02, 0.1)):
    cs = _centres(rng, n, lo, hi, float(np.sqrt(2.0)) * hl[1])
    out = [_yaw_box(c, rng.uniform(-np.pi, np.pi), rng.uniform(hl[0], hl[1], 3)) for c in cs]
    return np.asarray(out, np.float32).reshape(-1, 15)


def _capsules(rng, n, lo=(0.2, -0.6, 0.0), hi=(0.9, 0.6, 1.0)):
    out = []
    for c in _centres(rng, n, lo, hi, 0.26):
        axis = rng.normal(size=3)
        axis /= np.linalg.norm(axis)
        h = rng.uniform(0.1, 0.4)
        r = rng.uniform(0.02, 0.06)
        out.append([*(c - axis * h / 2), *(c + axis * h / 2), r])
    return np.asarray(out, np.float32).reshape(-1, 7)


def spheres_world(rng, n=16) -> dict:
    w = empty_world()
    w["world_spheres"] = _spheres(rng, n)
    return w


def tabletop_world(rng) -> dict:
    """Floor + table top + 3-5 shelf slabs + clutter (20 boxes), 8 capsules, 32 spheres."""
    w = empty_world()
    boxes = []
    yaw = rng.uniform(-0.3, 0.3)
    cx, cy = rng.uniform(0.5, 0.7), rng.uniform(-0.2, 0.2)
    table_h = rng.uniform(0.25, 0.45)
    boxes.append(_yaw_box((cx, cy, table_h), yaw, (rng.uniform(0.15, 0.3), rng.uniform(0.2, 0.3), 0.02)))
    n_shelf = int(rng.integers(3, 6))
    for k in range(n_shelf):
        z = table_h + 0.15 + k * rng.uniform(0.12, 0.2)
        boxes.append(_yaw_box((cx + rng.uniform(-0.05, 0.05), cy, min(z, 1.0)), yaw,
                              (rng.uniform(0.1, 0.2), rng.uniform(0.2, 0.3), 0.02)))
    n_clutter = 20 - len(boxes)
    for c in _centres(rng, n_clutter, (0.2, -0.6, 0.0), (0.9, 0.6, 1.0), 0.12):
        boxes.append(_yaw_box(c, rng.uniform(-np.pi, np.pi), rng.uniform(0.02, 0.08, 3)))
    w["world_boxes"] = np.asarray(boxes, np.float32)
    w["world_capsules"] = _capsules(rng, 8)
    w["world_spheres"] = _spheres(rng, 32, lo=(0.2, -0.6, 0.0), hi=(0.9, 0.6, 1.0), r=(0.02, 0.06))
    w["world_halfspaces"] = np.array([[0, 0, 1, 0, 0, 0]], np.float32)
    return w


UNEVEN_LO, UNEVEN_HI = (-1.6, -1.6, 0.0), (1.6, 1.6, 1.8)


def uneven_world(rng) -> dict:
    """4-128 spheres and 0-32 boxes; the larger region keeps 128-obstacle scenes solvable."""
    w = empty_world()
    w["world_spheres"] = _spheres(rng, int(rng.integers(4, 129)), lo=UNEVEN_LO, hi=UNEVEN_HI)
    nb = int(rng.integers(0, 33))
    if nb:
        w["world_boxes"] = _random_boxes(rng, nb, UNEVEN_LO, UNEVEN_HI)
    return w


DENSE_LO, DENSE_HI = (-0.8, -0.8, 0.0), (0.8, 0.8, 1.2)
DENSE_KEEPOUT = 0.15  # just clear of the arm's first link: any obstacle there blocks every configuration


def dense_world(rng) -> dict:
    """The uneven counts (4-128 spheres, 0-32 boxes) at the density of the
    16-sphere scene: spheres (r 0.05-0.15) and boxes (half extents 0.02-0.3,
    random yaw) in [-0.8,0.8]^2 x [0,1.2], clear only of a 0.15 m column around
    the base.  About 2-25% of the configuration space is free, and some start /
    goal pairs lie in different free components (unsolvable problems)."""
    w = empty_world()
    n = int(rng.integers(4, 129))
    r = rng.uniform(0.05, 0.15, size=(n, 1))
    c = _centres(rng, n, DENSE_LO, DENSE_HI, 0.15, DENSE_KEEPOUT)
    w["world_spheres"] = np.concatenate([c, r], 1).astype(np.float32)
    nb = int(rng.integers(0, 33))
    if nb:
        cs = _centres(rng, nb, DENSE_LO, DENSE_HI, float(np.sqrt(2.0)) * 0.3, DENSE_KEEPOUT)
        boxes = [_yaw_box(ci, rng.uniform(-np.pi, np.pi), rng.uniform(0.02, 0.3, 3)) for ci in cs]
        w["world_boxes"] = np.asarray(boxes, np.float32).reshape(-1, 15)
    return w


def box_surface_points(rng, boxes: np.ndarray, n: int) -> np.ndarray:
    """n points uniform over the surfaces of oriented boxes [Nb, 15] (c, a1, a2, a3, half-lengths)."""
    boxes = np.asarray(boxes, np.float64).reshape(-1, 15)
    hl = boxes[:, 12:15]
    # faces of box b: axis k at +-hl[k], spanned by the two other axes
    area = np.stack([4 * hl[:, 1] * hl[:, 2], 4 * hl[:, 0] * hl[:, 2], 4 * hl[:, 0] * hl[:, 1]], 1)  # [Nb, 3]
    w = np.repeat(area, 2, axis=1).reshape(-1)
    face = rng.choice(w.shape[0], size=n, p=w / w.sum())
    b, k, sign = face // 6, (face % 6) // 2, np.where(face % 2 == 0, 1.0, -1.0)
    u = rng.uniform(-1.0, 1.0, size=(n, 3))
    u[np.arange(n), k] = sign
    local = u * hl[b]
    axes = boxes[b, 3:12].reshape(n, 3, 3)  # rows a1, a2, a3
    return (boxes[b, :3] + np.einsum("nk,nkj->nj", local, axes)).astype(np.float32)


def pointcloud_world(rng, n_points: int = 20000) -> tuple[dict, np.ndarray]:
    """Tabletop scene whose 20 boxes are seen only as a scanned point cloud
    (n_points on their surfaces); floor, capsules and spheres stay analytic."""
    base = tabletop_world(rng)
    pts = box_surface_points(rng, base["world_boxes"], n_points)
    w = empty_world()
    for k in ("world_spheres", "world_capsules", "world_halfspaces"):
        w[k] = base[k]
    return w, pts


LARGE_LO, LARGE_HI = (-2.4, -2.6, 0.0), (2.4, 2.6, 2.0)


def large_world(rng) -> dict:
    """256 spheres, 64 boxes and a floor around the dual arm."""
    global _BASES
    saved, _BASES = _BASES, [(0.0, -0.3), (0.0, 0.3)]
    try:
        w = empty_world()
        w["world_spheres"] = _spheres(rng, 256, lo=LARGE_LO, hi=LARGE_HI)
        w["world_boxes"] = _random_boxes(rng, 64, LARGE_LO, LARGE_HI)
        w["world_halfspaces"] = np.array([[0, 0, 1, 0, 0, 0]], np.float32)
    finally:
        _BASES = saved
    return w


# ----------------------------------------------------------------------------- problems

@dataclass
class Problem:
    seed: int
    context: dict
    start: np.ndarray
    goals: np.ndarray
    lower: np.ndarray
    upper: np.ndarray
    max_nodes: int = 65536

    @property
    def dim(self) -> int:
        return int(self.start.shape[0])


def sample_free(rng, ctx, lo, hi, n, checker: Checker, max_tries: int = 200, batch: int = 256):
    """n collision-free configurations drawn uniform in [lo, hi]."""
    out = []
    for _ in range(max_tries):
        cand = rng.uniform(lo, hi, size=(batch, lo.shape[0])).astype(np.float32)
        v = np.asarray(checker(cand, ctx)).reshape(-1)
        out.extend(cand[v == 0])
        if len(out) >= n:
            return np.asarray(out[:n], np.float32)
    raise RuntimeError("could not sample collision-free configurations")


BUCKETS = (4096, 16384, 65536)


def make_problem(kind: str, seed: int, checker: Checker, robot: RobotModel | None = None) -> Problem:
    """Problem ``seed`` of workload ``kind``: spheres16 | tabletop | uneven | dense | large | pointcloud."""
    rng = np.random.default_rng(seed)
    if kind == "large":
        robot = robot or dual_arm(0)
    else:
        robot = robot or arm(0)
    if kind == "spheres16":
        world, n_goals, max_nodes = spheres_world(rng, 16), 1, 65536
    elif kind == "tabletop":
        world, n_goals, max_nodes = tabletop_world(rng), 4, 65536
    elif kind in ("uneven", "dense"):
        world = uneven_world(rng) if kind == "uneven" else dense_world(rng)
        n_goals = int(rng.integers(1, 9))
        n_obs = world["world_spheres"].shape[0] + world["world_boxes"].shape[0]
        max_nodes = BUCKETS[0] if n_obs < 48 else (BUCKETS[1] if n_obs < 112 else BUCKETS[2])
    elif kind == "large":
        world = large_world(rng)
        n_goals = int(rng.integers(1, 5))
        max_nodes = 131072
    elif kind == "pointcloud":
        world, cloud = pointcloud_world(rng)
        n_goals, max_nodes = 2, 65536
    else:
        raise ValueError(f"unknown workload {kind!r}")
    ctx = build_collision_context(robot, world)
    if kind == "pointcloud":
        ctx["point_cloud"], ctx["r_env"] = cloud, 0.01
    lo, hi = robot.lower.astype(np.float32), robot.upper.astype(np.float32)
    qs = sample_free(rng, ctx, lo, hi, 1 + n_goals, checker)
    return Problem(seed, ctx, qs[0], qs[1:], lo, hi, max_nodes)
