"""Collision-context construction: the ``collision_context`` key contract.

Restates ``build_prrtc_collision_context`` (cuda-rrtc/jax/utils.py:119-252) and
``world_obstacles_to_exact`` (utils.py:58-116) for robot models described by plain
arrays (PyRoFFI's Robot / RobotCollisionSpherized are not available):

* fine spheres with radius > 0, stably sorted by their FK frame (utils.py:130-157);
* one coarse bounding sphere per contiguous frame group, centred on the AABB
  midpoint of the group's sphere centres, radius max(|p - c| + r) (utils.py:159-182);
* self pairs: every fine-sphere combination of each active link pair, row-major,
  grouped by coarse pair with ``[start, end)`` ranges (utils.py:186-227);
* world rows: sphere (x,y,z,r), capsule (p1,p2,r), box (c, R[:,0], R[:,1], R[:,2],
  half_lengths), halfspace (n, p) (utils.py:58-116).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

WORLD_KEYS = {"world_spheres": 4, "world_capsules": 7, "world_boxes": 15, "world_halfspaces": 6}
ROBOT_KEYS = (
    "fk_twists", "fk_parent_tf", "fk_parent_idx", "fk_act_idx", "fk_mimic_mul",
    "fk_mimic_off", "fk_mimic_act_idx", "fk_topo_inv", "sphere_link_idx", "sphere_local",
    "sphere_radius",
)
COARSE_KEYS = (
    "coarse_sphere_link_idx", "coarse_sphere_local", "coarse_sphere_radius",
    "fine_link_offsets", "coarse_self_pairs", "self_pair_ranges",
)


@dataclass
class RobotModel:
    """Kinematic tree + spherised collision model.

    Joint tables follow the FK convention of this library: joints are stored in
    topological order (``parent_idx[j] < j``, -1 for the root); the local
    transform of joint j is ``parent_tf[j] o exp(twist[j] * v_j)`` with twist
    order (v, w) and parent_tf ``[qw,qx,qy,qz,tx,ty,tz]``; the joint value is
    ``mimic_mul*q[mimic_act_idx] + mimic_off`` for a mimic joint, ``q[act_idx]``
    for an actuated joint, 0 for a fixed joint; output frame k is sorted joint
    ``topo_inv[k]``.
    """

    twists: np.ndarray
    parent_tf: np.ndarray
    parent_idx: np.ndarray
    act_idx: np.ndarray
    mimic_mul: np.ndarray
    mimic_off: np.ndarray
    mimic_act_idx: np.ndarray
    topo_inv: np.ndarray
    lower: np.ndarray
    upper: np.ndarray
    sphere_frame: np.ndarray       # raw FK frame per sphere (any order)
    sphere_local: np.ndarray       # [S,3]
    sphere_radius: np.ndarray      # [S]
    link_pairs: list = field(default_factory=list)  # active (frame_i, frame_j) self pairs

    @property
    def dim(self) -> int:
        return int(self.lower.shape[0])

    @property
    def n_joints(self) -> int:
        return int(self.parent_idx.shape[0])


def empty_world() -> dict:
    return {k: np.zeros((0, c), dtype=np.float32) for k, c in WORLD_KEYS.items()}


def build_collision_context(robot: RobotModel, world: dict | None = None) -> dict:
    """Produce every collision_context key for ``robot`` in ``world``."""
    radius_full = np.asarray(robot.sphere_radius, dtype=np.float32)
    valid = radius_full > 0.0
    frame = np.asarray(robot.sphere_frame, dtype=np.int32)[valid]
    local = np.asarray(robot.sphere_local, dtype=np.float32)[valid]
    radius = radius_full[valid]
    old_index = np.flatnonzero(valid)

    order = np.argsort(frame, kind="stable")
    sphere_link_idx = frame[order].astype(np.int32)
    sphere_local = local[order].astype(np.float32)
    sphere_radius = radius[order].astype(np.float32)
    new_of_valid = np.empty(order.shape[0], dtype=np.int32)
    new_of_valid[order] = np.arange(order.shape[0], dtype=np.int32)

    if sphere_link_idx.shape[0] > 0:
        bounds = np.flatnonzero(np.diff(sphere_link_idx)) + 1
        starts = np.concatenate(([0], bounds)).astype(np.int64)
        ends = np.concatenate((bounds, [sphere_link_idx.shape[0]])).astype(np.int64)
    else:
        starts = np.zeros((0,), dtype=np.int64)
        ends = np.zeros((0,), dtype=np.int64)
    coarse_link = sphere_link_idx[starts].astype(np.int32)
    fine_offsets = np.concatenate((starts, [sphere_link_idx.shape[0]])).astype(np.int32)
    coarse_local = np.zeros((starts.shape[0], 3), dtype=np.float32)
    coarse_radius = np.zeros((starts.shape[0],), dtype=np.float32)
    for k, (s, e) in enumerate(zip(starts, ends)):
        locs = sphere_local[s:e].astype(np.float64)
        rads = sphere_radius[s:e].astype(np.float64)
        # the centre as stored (float32); the reach is measured from it, in
        # float64, and the radius rounded up, so that the float32 sphere
        # encloses every fine sphere exactly
        c = (0.5 * (locs.min(axis=0) + locs.max(axis=0))).astype(np.float32)
        coarse_local[k] = c
        r = float(np.max(np.linalg.norm(locs - c.astype(np.float64), axis=1) + rads))
        coarse_radius[k] = np.nextafter(np.float32(r), np.float32(np.inf))
    group_of_frame = {int(f): k for k, f in enumerate(coarse_link)}

    # raw sphere index -> new sorted index (-1 when filtered)
    new_of_raw = np.full(radius_full.shape[0], -1, dtype=np.int32)
    new_of_raw[old_index] = new_of_valid
    raw_frame = np.asarray(robot.sphere_frame, dtype=np.int32)
    blocks, cpairs, ranges = [], [], []
    cursor = 0
    for fi, fj in robot.link_pairs:
        a = np.sort(new_of_raw[(raw_frame == fi) & valid])
        b = np.sort(new_of_raw[(raw_frame == fj) & valid])
        if a.size == 0 or b.size == 0:
            continue
        gi, gj = group_of_frame.get(int(fi), -1), group_of_frame.get(int(fj), -1)
        if gi < 0 or gj < 0:
            continue
        blk = np.stack(np.meshgrid(a, b, indexing="ij"), axis=-1).reshape(-1, 2)
        blocks.append(blk)
        cpairs.append((gi, gj))
        ranges.append((cursor, cursor + blk.shape[0]))
        cursor += blk.shape[0]
    self_pairs = np.concatenate(blocks, 0).astype(np.int32) if blocks else np.zeros((0, 2), np.int32)

    ctx = {
        "fk_twists": np.asarray(robot.twists, np.float32),
        "fk_parent_tf": np.asarray(robot.parent_tf, np.float32),
        "fk_parent_idx": np.asarray(robot.parent_idx, np.int32),
        "fk_act_idx": np.asarray(robot.act_idx, np.int32),
        "fk_mimic_mul": np.asarray(robot.mimic_mul, np.float32),
        "fk_mimic_off": np.asarray(robot.mimic_off, np.float32),
        "fk_mimic_act_idx": np.asarray(robot.mimic_act_idx, np.int32),
        "fk_topo_inv": np.asarray(robot.topo_inv, np.int32),
        "sphere_link_idx": sphere_link_idx,
        "sphere_local": sphere_local,
        "sphere_radius": sphere_radius,
        "self_pairs": self_pairs,
        "coarse_sphere_link_idx": coarse_link,
        "coarse_sphere_local": coarse_local,
        "coarse_sphere_radius": coarse_radius,
        "fine_link_offsets": fine_offsets,
        "coarse_self_pairs": np.asarray(cpairs, np.int32).reshape(-1, 2),
        "self_pair_ranges": np.asarray(ranges, np.int32).reshape(-1, 2),
    }
    w = empty_world()
    if world:
        for k, c in WORLD_KEYS.items():
            if k in world and world[k] is not None:
                w[k] = np.asarray(world[k], np.float32).reshape(-1, c)
    ctx.update(w)
    return ctx


def with_world(ctx: dict, world: dict) -> dict:
    """Copy of ``ctx`` whose world keys are replaced by ``world``'s."""
    out = dict(ctx)
    for k, c in WORLD_KEYS.items():
        out[k] = np.asarray(world.get(k, np.zeros((0, c))), np.float32).reshape(-1, c)
    return out
