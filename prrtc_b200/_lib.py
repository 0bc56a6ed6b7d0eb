"""ctypes bindings of libprrtc_b200.so (the C-ABI in include/prrtc_b200.h).

The library is built in-tree by ``prrtc_b200.build``; loading fails loudly when
it is missing or when no CUDA device is present -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import time
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libprrtc_b200.so"

OK, EARG, EWORKSPACE, ECUDA, EUNSUPPORTED = 0, -1, -2, -3, -4

P = C.c_void_p
I32 = C.c_int32
F32 = C.c_float


class Robot(C.Structure):
    _fields_ = [
        ("fk_twists", P), ("fk_parent_tf", P), ("fk_parent_idx", P), ("fk_act_idx", P),
        ("fk_mimic_mul", P), ("fk_mimic_off", P), ("fk_mimic_act_idx", P), ("fk_topo_inv", P),
        ("n_joints", I32),
        ("sphere_link_idx", P), ("sphere_local", P), ("sphere_radius", P), ("n_spheres", I32),
        ("coarse_sphere_link_idx", P), ("coarse_sphere_local", P), ("coarse_sphere_radius", P),
        ("fine_link_offsets", P), ("n_coarse", I32),
        ("coarse_self_pairs", P), ("self_pair_ranges", P), ("n_coarse_self_pairs", I32),
    ]


class World(C.Structure):
    _fields_ = [
        ("world_spheres", P), ("n_world_spheres", I32),
        ("world_capsules", P), ("n_world_capsules", I32),
        ("world_boxes", P), ("n_world_boxes", I32),
        ("world_halfspaces", P), ("n_world_halfspaces", I32),
        ("self_pairs", P), ("n_self_pairs", I32),
    ]


class Inputs(C.Structure):
    _fields_ = [
        ("start_config", P), ("goal_configs", P), ("num_goals", I32),
        ("min_vals", P), ("max_vals", P), ("robot", Robot), ("world", World),
    ]


class Outputs(C.Structure):
    _fields_ = [
        ("tree_a_configs", P), ("tree_b_configs", P), ("tree_a_parents", P), ("tree_b_parents", P),
        ("tree_sizes", P), ("completed", P), ("iter_count", P), ("connection_info", P),
        ("solved_flag", P), ("kernel_time_ms", P),
    ]


class Attrs(C.Structure):
    _fields_ = [
        ("max_iterations", I32), ("step_size", F32), ("num_new_samples", I32), ("balance_mode", I32),
        ("tree_ratio", F32), ("dynamic_domain", I32), ("dd_alpha", F32), ("dd_radius", F32),
        ("dd_min_radius", F32), ("dim", I32), ("max_nodes", I32), ("granularity", I32),
        ("collision_mode", I32), ("collision_margin", F32),
    ]


class PointCloud(C.Structure):
    _fields_ = [
        ("points", P), ("bucket_start", P), ("n_points", I32), ("n_buckets", I32), ("cell", F32), ("r_env", F32),
    ]


class Tuning(C.Structure):
    _fields_ = [
        ("edge_resolution", F32), ("threads_per_explorer", I32), ("waypoint_chunk", I32),
        ("resident_ctas", I32), ("stats", P), ("point_cloud", P), ("tail_explorers", I32),
        ("staging_wait_polls", I32), ("ctas_per_sm", I32), ("explore_events", P * 2),
    ]


class BatchInputs(C.Structure):
    _fields_ = [
        ("batch", I32), ("start_configs", P), ("goal_configs", P), ("num_goals", I32), ("goal_counts", P),
        ("min_vals", P), ("max_vals", P), ("robot", Robot),
        ("world_spheres", P), ("max_world_spheres", I32), ("world_spheres_count", P),
        ("world_capsules", P), ("max_world_capsules", I32), ("world_capsules_count", P),
        ("world_boxes", P), ("max_world_boxes", I32), ("world_boxes_count", P),
        ("world_halfspaces", P), ("max_world_halfspaces", I32), ("world_halfspaces_count", P),
        ("self_pairs", P), ("max_self_pairs", I32), ("self_pairs_count", P),
        ("problem_order", P), ("problem_capacity", P),
    ]


EXPORTS = (
    "prrtc_b200_plan_workspace_size", "prrtc_b200_plan",
    "prrtc_b200_plan_batch_workspace_size", "prrtc_b200_plan_batch",
    "prrtc_b200_nearest_neighbor_workspace_size", "prrtc_b200_nearest_neighbor",
    "prrtc_b200_extend",
    "prrtc_b200_check_configs_workspace_size", "prrtc_b200_check_configs",
    "prrtc_b200_iteration",
    "prrtc_b200_point_cloud_workspace_size", "prrtc_b200_point_cloud_build",
    "prrtc_b200_check_edges_workspace_size", "prrtc_b200_check_edges",
    "prrtc_b200_fk", "prrtc_b200_halton", "prrtc_b200_extract_paths", "prrtc_b200_result_block",
    "prrtc_b200_smooth_workspace_size", "prrtc_b200_smooth_cost_grad",
    "prrtc_b200_smooth_batch_workspace_size", "prrtc_b200_smooth_cost_grad_batch",
    "prrtc_b200_choose_tree", "prrtc_b200_radius_update",
    "prrtc_b200_fp32_probe", "prrtc_b200_fp32x2_probe",
    "prrtc_b200_error_string", "prrtc_b200_last_cuda_error", "prrtc_b200_version",
)

_SIGS = {
    "prrtc_b200_plan_workspace_size": (C.c_size_t, [P, P, P]),
    "prrtc_b200_plan": (C.c_int, [P, P, P, P, P, C.c_size_t, P]),
    "prrtc_b200_plan_batch_workspace_size": (C.c_size_t, [P, P, P]),
    "prrtc_b200_plan_batch": (C.c_int, [P, P, P, P, P, C.c_size_t, P]),
    "prrtc_b200_nearest_neighbor_workspace_size": (C.c_size_t, [I32]),
    "prrtc_b200_nearest_neighbor": (C.c_int, [P, I32, I32, P, P, I32, P, P, P, C.c_size_t, P]),
    "prrtc_b200_extend": (C.c_int, [P, I32, I32, P, P, I32, P, P, P, P, P]),
    "prrtc_b200_check_configs_workspace_size": (C.c_size_t, [P, P]),
    "prrtc_b200_check_configs": (C.c_int, [P, P, I32, P, I32, I32, F32, I32, P, P, C.c_size_t, P]),
    "prrtc_b200_iteration": (C.c_int, [P, P, P, P, I32, I32, P, I32, P, P, P, P, P, P, P, P]),
    "prrtc_b200_point_cloud_workspace_size": (C.c_size_t, [I32, I32]),
    "prrtc_b200_point_cloud_build": (C.c_int, [P, I32, F32, F32, I32, P, C.c_size_t, P, P]),
    "prrtc_b200_check_edges_workspace_size": (C.c_size_t, [P, P, I32, I32]),
    "prrtc_b200_check_edges": (C.c_int, [P, P, P, I32, P, I32, I32, I32, F32, P, P, C.c_size_t, P]),
    "prrtc_b200_fk": (C.c_int, [P, I32, P, I32, P, P]),
    "prrtc_b200_halton": (C.c_int, [I32, I32, I32, P, P, P, P]),
    "prrtc_b200_extract_paths": (C.c_int, [I32, I32, I32, P, P, P, P, P, P, I32, P, P, P, P]),
    "prrtc_b200_result_block": (C.c_int, [I32, I32, I32, P, P, P, P, P, P, P, P, P, P, P, C.c_int64, P]),
    "prrtc_b200_smooth_workspace_size": (C.c_size_t, [P, P]),
    "prrtc_b200_smooth_cost_grad": (C.c_int, [P, P, I32, P, I32, I32, F32, F32, F32, P, P, P, C.c_size_t, P]),
    "prrtc_b200_smooth_batch_workspace_size": (C.c_size_t, [P]),
    "prrtc_b200_smooth_cost_grad_batch": (C.c_int, [P, I32, P, I32, F32, F32, F32, P, P, P, C.c_size_t, P]),
    "prrtc_b200_choose_tree": (C.c_int, [I32, I32, P, P, P, I32, F32, P, P, P]),
    "prrtc_b200_radius_update": (C.c_int, [P, P, P, I32, F32, F32, F32, I32, P, P]),
    "prrtc_b200_fp32_probe": (C.c_int, [I32, I32, I32, P, P]),
    "prrtc_b200_fp32x2_probe": (C.c_int, [I32, I32, I32, P, P]),
    "prrtc_b200_error_string": (C.c_char_p, [C.c_int]),
    "prrtc_b200_last_cuda_error": (C.c_int, []),
    "prrtc_b200_version": (C.c_int, []),
}

_lib = None


def load(build_if_missing: bool = True) -> C.CDLL:
    """Load the shared library (building it first if absent and nvcc is available)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists() and build_if_missing:
        from . import build as _build
        _build.build()
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m prrtc_b200.build`")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


_hostpack = None


def hostpack():
    """The native host packer module (csrc/hostpack.cc), built on first use."""
    global _hostpack
    if _hostpack is None:
        from . import build as _build

        _build.build_hostpack()
        from . import _hostpack as hp

        _hostpack = hp
    return _hostpack


class PrrtcError(RuntimeError):
    pass


class PrrtcTimeout(PrrtcError):
    """A host wait for a call's results ran past its timeout.  The call's work is
    still queued or running on the GPU; its buffers stay referenced, and the
    wait can be repeated."""


def wait_event(event, timeout_s: float | None, what: str) -> None:
    """Wait for a CUDA event (an object with ``synchronize()`` and ``query()``):
    blocking when ``timeout_s`` is None; otherwise polling ``query()``
    (cudaEventQuery) until the event completes or ``timeout_s`` seconds have
    passed, then raising PrrtcTimeout.  The poll sleeps 20 us, doubling up to
    1 ms, so a GPU that stops answering leaves the host with an error instead
    of a thread blocked for good."""
    if timeout_s is None:
        event.synchronize()
        return
    deadline = time.monotonic() + max(0.0, float(timeout_s))
    nap = 20e-6
    while not event.query():
        if time.monotonic() >= deadline:
            raise PrrtcTimeout(f"{what}: not complete after {float(timeout_s):g} s")
        time.sleep(nap)
        nap = min(2.0 * nap, 1e-3)


def check(rc: int, what: str) -> None:
    if rc != OK:
        lib = load()
        msg = lib.prrtc_b200_error_string(rc).decode()
        if rc == EARG:
            raise ValueError(f"{what}: {msg}")
        raise PrrtcError(f"{what} failed ({rc}): {msg}")
