"""Property test (hypothesis, GPU) of the batched checker on random arms and worlds.

The fixed-case parity tests use the 7-joint arm and the 18-joint dual arm.  Here
hypothesis draws serial arms of 2-16 joints (16-128 spheres, self pairs between
links two or more apart), a world (16 spheres, the tabletop scene, or an uneven
scene of 4-128 spheres and 0-32 boxes) and a checker, and the GPU verdicts --
early exit and full sweep -- must equal the oracle's for every configuration
more than 1e-4 m from contact.  The arm's size moves the checker's pass size:
32 configurations per pass up to about 8 joints, 16 or 8 beyond, where the
pass buffers of 32 configurations would leave fewer than four CTAs per SM.
The draws are derandomized: every run tests the same examples.
"""
from __future__ import annotations

import numpy as np
import pytest
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

from prrtc_b200 import scenes
from prrtc_b200.context import build_collision_context

pytestmark = pytest.mark.gpu

CHECKERS = ["binary", "differentiable", "binary_coarse", "binary_coarse_coop"]


@settings(max_examples=24, deadline=None, derandomize=True,
          suppress_health_check=[HealthCheck.function_scoped_fixture])
@given(seed=st.integers(0, 10**6), n_joints=st.integers(2, 16), wseed=st.integers(0, 2**31 - 1),
       kind=st.sampled_from(["spheres", "tabletop", "uneven"]), mode=st.integers(0, 3))
def test_batched_checker_matches_oracle_on_random_arms_and_worlds(cuda, orc, seed, n_joints, wseed, kind, mode):
    from prrtc_b200.collision import CollisionChecker

    robot = scenes.arm(seed, n_joints)
    rng = np.random.default_rng(wseed)
    world = {"spheres": lambda: scenes.spheres_world(rng, 16), "tabletop": lambda: scenes.tabletop_world(rng),
             "uneven": lambda: scenes.uneven_world(rng)}[kind]()
    ctx = build_collision_context(robot, world)
    q = rng.uniform(robot.lower, robot.upper, (700, robot.dim)).astype(np.float32)
    chk = CollisionChecker(ctx, robot.dim, CHECKERS[mode], 0.02, device=cuda)
    early = chk.check(q).cpu().numpy()
    full = chk.check(q, full_sweep=True).cpu().numpy()
    assert np.array_equal(early, full)
    sc = orc.Scene(ctx, robot.dim)
    want = sc.check_configs(q, mode, 0.02)
    thr = 0.02 if mode == 1 else 0.0
    far = np.abs(sc.min_distances(q) - thr) > 1e-4
    assert np.array_equal(early[far], want[far]), f"{(early[far] != want[far]).sum()} verdicts differ"
