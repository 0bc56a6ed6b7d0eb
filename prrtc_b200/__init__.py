"""prrtc_b200 -- B200-native (sm_100a) pRRTC motion planner.

Drop-in for P-RRAX's ``prrtc_plan`` path: the same API and collision_context
contract, computed by hand-written CUDA kernels in ``libprrtc_b200.so``.
"""
from .prrtc import (  # noqa: F401
    PRRTCResult,
    lpt_order,
    prrtc_extend,
    prrtc_iteration,
    prrtc_nearest_neighbor,
    prrtc_plan,
    prrtc_plan_batch,
    prrtc_plan_batch_async,
)
from .pointcloud import PointCloud, PointCloudChecker, prrtc_plan_robogpu  # noqa: E402,F401
from ._lib import PrrtcError, PrrtcTimeout  # noqa: E402,F401

__all__ = [
    "PRRTCResult",
    "prrtc_plan",
    "prrtc_plan_batch",
    "prrtc_plan_batch_async",
    "prrtc_nearest_neighbor",
    "prrtc_extend",
    "prrtc_iteration",
    "lpt_order",
    "PointCloud",
    "PointCloudChecker",
    "prrtc_plan_robogpu",
    "PrrtcError",
    "PrrtcTimeout",
]
