"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE).

Only the test suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.  It wraps ``liboracle.so`` (built from
``prrtc_oracle.c`` by ``oracle/Makefile``), a C restatement of the reference's
pRRTC arithmetic; see ``prrtc_oracle.h`` for the reference lines each function
follows.  Parity at the PyRoFFI boundary (FK, primitive distances) is unpinned;
Halton / nearest-neighbour / extend arithmetic is pinned on the GPU against the
reference's own device code (``oracle/ref``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "liboracle.so"

DIM_MAX = 16


def build() -> Path:
    """Compile liboracle.so with the committed Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _LIB_PATH


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            build()
        _lib = C.CDLL(str(_LIB_PATH))
        _declare(_lib)
    return _lib


class OrcScene(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("n_joints", C.c_int),
        ("twists", C.c_void_p), ("parent_tf", C.c_void_p), ("parent_idx", C.c_void_p),
        ("act_idx", C.c_void_p), ("mimic_mul", C.c_void_p), ("mimic_off", C.c_void_p),
        ("mimic_act_idx", C.c_void_p), ("topo_inv", C.c_void_p),
        ("n_spheres", C.c_int), ("sphere_link_idx", C.c_void_p), ("sphere_local", C.c_void_p),
        ("sphere_radius", C.c_void_p),
        ("n_ws", C.c_int), ("world_spheres", C.c_void_p),
        ("n_wc", C.c_int), ("world_capsules", C.c_void_p),
        ("n_wb", C.c_int), ("world_boxes", C.c_void_p),
        ("n_wh", C.c_int), ("world_halfspaces", C.c_void_p),
        ("n_self", C.c_int), ("self_pairs", C.c_void_p),
        ("n_coarse", C.c_int), ("coarse_link", C.c_void_p), ("coarse_local", C.c_void_p),
        ("coarse_radius", C.c_void_p), ("fine_offsets", C.c_void_p),
        ("n_coarse_self", C.c_int), ("coarse_self_pairs", C.c_void_p), ("self_pair_ranges", C.c_void_p),
        ("n_points", C.c_int), ("points", C.c_void_p), ("r_env", C.c_float),
    ]


class OrcPlanParams(C.Structure):
    _fields_ = [
        ("max_iterations", C.c_int), ("step_size", C.c_float), ("num_new_samples", C.c_int),
        ("balance_mode", C.c_int), ("tree_ratio", C.c_float), ("dynamic_domain", C.c_int),
        ("dd_alpha", C.c_float), ("dd_radius", C.c_float), ("dd_min_radius", C.c_float),
        ("dim", C.c_int), ("max_nodes", C.c_int), ("granularity", C.c_int),
        ("collision_mode", C.c_int), ("collision_margin", C.c_float), ("edge_resolution", C.c_float),
    ]


class OrcPlanOut(C.Structure):
    _fields_ = [
        ("tree_a", C.c_void_p), ("tree_b", C.c_void_p), ("parents_a", C.c_void_p), ("parents_b", C.c_void_p),
        ("tree_sizes", C.c_int * 2), ("completed", C.c_int * 2), ("iter_count", C.c_int),
        ("connection", C.c_int * 3), ("solved", C.c_int),
        ("edge_checks", C.c_int64), ("config_checks", C.c_int64),
    ]


class OrcHostOut(C.Structure):
    _fields_ = [
        ("solved", C.c_int), ("iterations", C.c_int), ("size_a", C.c_int), ("size_b", C.c_int),
        ("path_len", C.c_int), ("cost", C.c_float), ("config_checks", C.c_int64),
    ]


def _declare(L: C.CDLL) -> None:
    P, I, F, D = C.c_void_p, C.c_int, C.c_float, C.c_double
    sig = {
        "orc_halton_next": (F, [I, P]),
        "orc_prime_order": (None, [I, P]),
        "orc_halton_sample": (None, [P, P, I, P, P, P]),
        "orc_nearest": (I, [P, I, I, I, P, P]),
        "orc_dist_sq": (F, [P, I, I, I, P]),
        "orc_extend": (None, [P, P, I, F, F, P]),
        "orc_edge_waypoints": (I, [P, I, I, F]),
        "orc_waypoint": (None, [P, P, I, I, I, P]),
        "orc_choose_tree": (I, [I, I, I, I, I, I, F, P]),
        "orc_radius_shrink": (None, [P, I, F, F, F]),
        "orc_radius_grow": (None, [P, I, F]),
        "orc_fk_f64": (None, [P, P, P]),
        "orc_fk_f32": (None, [P, P, P]),
        "orc_config_in_collision": (I, [P, P, I, F]),
        "orc_min_distance": (D, [P, P]),
        "orc_edge_in_collision": (I, [P, P, P, I, F, I, F]),
        "orc_check_configs": (None, [P, P, I, I, F, P]),
        "orc_prrtc_plan": (I, [P, P, P, I, P, P, P, P]),
        "orc_trace_path": (I, [P, P, P, P, I, I, P, P, I]),
        "orc_path_cost": (F, [P, I, I]),
        "orc_rrtc_host_plan": (I, [P, P, P, P, P, I, F, I, I, I, I, C.c_uint64, I, F, I, P, I, P]),
        "orc_validate_path": (I, [P, P, I, F, P]),
        "orc_smooth_cost": (D, [P, P, I, F, F, F]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data if a is not None and a.size > 0 else 0


_CTX_SPEC = {
    "fk_twists": (np.float32, (-1, 6)), "fk_parent_tf": (np.float32, (-1, 7)),
    "fk_parent_idx": (np.int32, (-1,)), "fk_act_idx": (np.int32, (-1,)),
    "fk_mimic_mul": (np.float32, (-1,)), "fk_mimic_off": (np.float32, (-1,)),
    "fk_mimic_act_idx": (np.int32, (-1,)), "fk_topo_inv": (np.int32, (-1,)),
    "sphere_link_idx": (np.int32, (-1,)), "sphere_local": (np.float32, (-1, 3)),
    "sphere_radius": (np.float32, (-1,)),
    "world_spheres": (np.float32, (-1, 4)), "world_capsules": (np.float32, (-1, 7)),
    "world_boxes": (np.float32, (-1, 15)), "world_halfspaces": (np.float32, (-1, 6)),
    "self_pairs": (np.int32, (-1, 2)),
    "coarse_sphere_link_idx": (np.int32, (-1,)), "coarse_sphere_local": (np.float32, (-1, 3)),
    "coarse_sphere_radius": (np.float32, (-1,)), "fine_link_offsets": (np.int32, (-1,)),
    "coarse_self_pairs": (np.int32, (-1, 2)), "self_pair_ranges": (np.int32, (-1, 2)),
    "point_cloud": (np.float32, (-1, 3)),
}


class Scene:
    """A collision_context dict held as contiguous numpy arrays plus its OrcScene view."""

    def __init__(self, ctx: dict, dim: int):
        self.arrays = {}
        for key, (dt, shape) in _CTX_SPEC.items():
            if key in ctx and ctx[key] is not None:
                a = np.ascontiguousarray(np.asarray(ctx[key], dtype=dt)).reshape(shape)
            else:
                a = np.zeros((0,) + tuple(s for s in shape[1:]), dtype=dt)
            self.arrays[key] = a
        A = self.arrays
        self.dim = int(dim)
        s = OrcScene()
        s.dim = self.dim
        s.n_joints = A["fk_parent_idx"].shape[0]
        s.twists, s.parent_tf = _ptr(A["fk_twists"]), _ptr(A["fk_parent_tf"])
        s.parent_idx, s.act_idx = _ptr(A["fk_parent_idx"]), _ptr(A["fk_act_idx"])
        s.mimic_mul, s.mimic_off = _ptr(A["fk_mimic_mul"]), _ptr(A["fk_mimic_off"])
        s.mimic_act_idx, s.topo_inv = _ptr(A["fk_mimic_act_idx"]), _ptr(A["fk_topo_inv"])
        s.n_spheres = A["sphere_link_idx"].shape[0]
        s.sphere_link_idx, s.sphere_local, s.sphere_radius = (
            _ptr(A["sphere_link_idx"]), _ptr(A["sphere_local"]), _ptr(A["sphere_radius"]))
        s.n_ws, s.world_spheres = A["world_spheres"].shape[0], _ptr(A["world_spheres"])
        s.n_wc, s.world_capsules = A["world_capsules"].shape[0], _ptr(A["world_capsules"])
        s.n_wb, s.world_boxes = A["world_boxes"].shape[0], _ptr(A["world_boxes"])
        s.n_wh, s.world_halfspaces = A["world_halfspaces"].shape[0], _ptr(A["world_halfspaces"])
        s.n_self, s.self_pairs = A["self_pairs"].shape[0], _ptr(A["self_pairs"])
        s.n_coarse = A["coarse_sphere_link_idx"].shape[0]
        s.coarse_link, s.coarse_local, s.coarse_radius = (
            _ptr(A["coarse_sphere_link_idx"]), _ptr(A["coarse_sphere_local"]), _ptr(A["coarse_sphere_radius"]))
        s.fine_offsets = _ptr(A["fine_link_offsets"])
        s.n_coarse_self = A["coarse_self_pairs"].shape[0]
        s.coarse_self_pairs, s.self_pair_ranges = _ptr(A["coarse_self_pairs"]), _ptr(A["self_pair_ranges"])
        s.n_points, s.points = A["point_cloud"].shape[0], _ptr(A["point_cloud"])
        s.r_env = float(ctx.get("r_env", 0.0) or 0.0)
        self.c = s
        self.ref = C.byref(self.c)

    # --- FK / collision ---
    def fk(self, q, f64: bool = True) -> np.ndarray:
        J = self.c.n_joints
        if f64:
            qd = np.ascontiguousarray(q, dtype=np.float64)
            out = np.zeros((J, 12), dtype=np.float64)
            lib().orc_fk_f64(self.ref, _ptr(qd), _ptr(out))
        else:
            qf = np.ascontiguousarray(q, dtype=np.float32)
            out = np.zeros((J, 12), dtype=np.float32)
            lib().orc_fk_f32(self.ref, _ptr(qf), _ptr(out))
        return out

    def in_collision(self, q, mode: int = 0, margin: float = 0.02) -> bool:
        qf = np.ascontiguousarray(q, dtype=np.float32)
        return bool(lib().orc_config_in_collision(self.ref, _ptr(qf), int(mode), float(margin)))

    def check_configs(self, configs, mode: int = 0, margin: float = 0.02) -> np.ndarray:
        cf = np.ascontiguousarray(configs, dtype=np.float32).reshape(-1, self.dim)
        out = np.zeros(cf.shape[0], dtype=np.int32)
        if cf.shape[0]:
            lib().orc_check_configs(self.ref, _ptr(cf), cf.shape[0], int(mode), float(margin), _ptr(out))
        return out

    def min_distance(self, q) -> float:
        qf = np.ascontiguousarray(q, dtype=np.float32)
        return float(lib().orc_min_distance(self.ref, _ptr(qf)))

    def min_distances(self, configs) -> np.ndarray:
        cf = np.ascontiguousarray(configs, dtype=np.float32).reshape(-1, self.dim)
        return np.array([self.min_distance(c) for c in cf], dtype=np.float64)

    def edge_in_collision(self, base, end, granularity=16, resolution=0.0, mode=0, margin=0.02) -> bool:
        b = np.ascontiguousarray(base, dtype=np.float32)
        e = np.ascontiguousarray(end, dtype=np.float32)
        return bool(lib().orc_edge_in_collision(self.ref, _ptr(b), _ptr(e), int(granularity),
                                                float(resolution), int(mode), float(margin)))

    def validate_path(self, path, resolution: float = 0.01):
        p = np.ascontiguousarray(path, dtype=np.float32).reshape(-1, self.dim)
        md = C.c_double(0.0)
        ok = lib().orc_validate_path(self.ref, _ptr(p), p.shape[0], float(resolution), C.byref(md))
        return bool(ok), float(md.value)

    def validate_planned_path(self, path, granularity: int = 16, resolution: float = 0.01,
                              graze_depth: float = 1e-3):
        """Re-validation of a path a sampling planner returned: (ok, min distance).

        The path passes when it is free at an independent `resolution` grid.
        Otherwise it must be free on the planner's own waypoints -- each edge at
        max(granularity, ceil(len/resolution)) points t = (k+1)/G, as the planner
        checked it, within 1e-5 m of contact (float32 against float64) -- and any
        graze between those waypoints, found at resolution/20, must be shallower
        than `graze_depth`: a sampled edge check cannot see a graze that lies
        between its samples, in this planner as in the reference's."""
        p = np.ascontiguousarray(path, dtype=np.float32).reshape(-1, self.dim)
        ok, md = self.validate_path(p, resolution)
        if ok:
            return True, md
        grid = np.concatenate([edge_waypoints(p[i], p[i + 1], granularity, resolution)
                               for i in range(p.shape[0] - 1)] + [p[:1]])
        md_grid = float(self.min_distances(grid).min())
        _, md_fine = self.validate_path(p, resolution / 20.0)
        return (md_grid >= -1e-5 and md_fine > -graze_depth), min(md_grid, md_fine)

    def smooth_cost(self, waypoints, margin=0.02, beta=50.0, w_len=1.0) -> float:
        w = np.ascontiguousarray(waypoints, dtype=np.float64).reshape(-1, self.dim)
        return float(lib().orc_smooth_cost(self.ref, _ptr(w), w.shape[0], float(margin), float(beta), float(w_len)))


# --- sampling / NN / extend (restated reference arithmetic) ---

def halton_next(base: int, state: int) -> tuple[float, int]:
    st = C.c_int(state)
    v = lib().orc_halton_next(int(base), C.byref(st))
    return float(np.float32(v)), st.value


def prime_order(explorer: int) -> np.ndarray:
    out = np.zeros(16, dtype=np.int32)
    lib().orc_prime_order(int(explorer), _ptr(out))
    return out


def halton_samples(explorer: int, n: int, lo, hi) -> np.ndarray:
    """First n Halton samples of one explorer: float32 [n, dim]."""
    lo = np.ascontiguousarray(lo, dtype=np.float32)
    hi = np.ascontiguousarray(hi, dtype=np.float32)
    dim = lo.shape[0]
    po = prime_order(explorer)
    st = np.ones(DIM_MAX, dtype=np.int32)
    out = np.zeros((n, dim), dtype=np.float32)
    row = np.zeros(dim, dtype=np.float32)
    for i in range(n):
        lib().orc_halton_sample(_ptr(po), _ptr(st), dim, _ptr(lo), _ptr(hi), _ptr(row))
        out[i] = row
    return out


def nearest(tree: np.ndarray, n: int, q) -> tuple[int, float]:
    """tree: float32 [dim, max_nodes] SoA."""
    t = np.ascontiguousarray(tree, dtype=np.float32)
    qf = np.ascontiguousarray(q, dtype=np.float32)
    d = C.c_float(0.0)
    idx = lib().orc_nearest(_ptr(t), t.shape[1], t.shape[0], int(n), _ptr(qf), C.byref(d))
    return int(idx), float(np.float32(d.value))


def nearest_batch(tree: np.ndarray, n: int, queries) -> tuple[np.ndarray, np.ndarray]:
    q = np.ascontiguousarray(queries, dtype=np.float32)
    idx = np.zeros(q.shape[0], dtype=np.int32)
    dsq = np.zeros(q.shape[0], dtype=np.float32)
    for i in range(q.shape[0]):
        idx[i], dsq[i] = nearest(tree, n, q[i])
    return idx, dsq


def extend(base, sample, nd: float, step: float) -> np.ndarray:
    b = np.ascontiguousarray(base, dtype=np.float32)
    s = np.ascontiguousarray(sample, dtype=np.float32)
    out = np.zeros_like(b)
    lib().orc_extend(_ptr(b), _ptr(s), b.shape[0], float(np.float32(nd)), float(step), _ptr(out))
    return out


def choose_tree(mode: int, sizes, local_iter, vamp_in, nblocks: int, tree_ratio: float):
    """Tree side of every explorer bid < nblocks for n cases (sizes [n,2],
    local_iter [n], vamp_in [n,nblocks]) -> (tree [n,nblocks], vamp [n,nblocks])."""
    sizes = np.asarray(sizes, np.int32).reshape(-1, 2)
    li = np.asarray(local_iter, np.int32).reshape(-1)
    vin = np.asarray(vamp_in, np.int32).reshape(sizes.shape[0], nblocks)
    tree = np.zeros_like(vin)
    vout = np.zeros_like(vin)
    fn = lib().orc_choose_tree
    for c in range(sizes.shape[0]):
        for b in range(nblocks):
            v = C.c_int(int(vin[c, b]))
            tree[c, b] = fn(int(mode), int(li[c]), b, int(nblocks), int(sizes[c, 0]), int(sizes[c, 1]),
                            float(tree_ratio), C.byref(v))
            vout[c, b] = v.value
    return tree, vout


def radius_updates(radii, idx, op, alpha: float, r0: float, rmin: float) -> np.ndarray:
    """Apply the dynamic-domain updates op[i] (0 shrink, 1 grow) on radii[idx[i]]
    in order; returns the new float32 radii (FLT_MAX = unset)."""
    r = np.array(radii, np.float32, copy=True)
    L = lib()
    for i, o in zip(np.asarray(idx).reshape(-1), np.asarray(op).reshape(-1)):
        if int(o) == 0:
            L.orc_radius_shrink(_ptr(r), int(i), float(alpha), float(r0), float(rmin))
        else:
            L.orc_radius_grow(_ptr(r), int(i), float(alpha))
    return r


def edge_waypoints(base, end, granularity: int, resolution: float = 0.0) -> np.ndarray:
    b = np.ascontiguousarray(base, dtype=np.float32)
    e = np.ascontiguousarray(end, dtype=np.float32)
    delta = (e - b).astype(np.float32)
    G = lib().orc_edge_waypoints(_ptr(delta), b.shape[0], int(granularity), float(resolution))
    out = np.zeros((G, b.shape[0]), dtype=np.float32)
    row = np.zeros(b.shape[0], dtype=np.float32)
    for k in range(G):
        lib().orc_waypoint(_ptr(b), _ptr(delta), b.shape[0], k, G, _ptr(row))
        out[k] = row
    return out


# --- planners ---

@dataclass
class PlanResult:
    solved: int
    tree_a: np.ndarray
    tree_b: np.ndarray
    parents_a: np.ndarray
    parents_b: np.ndarray
    tree_sizes: tuple
    completed: tuple
    iter_count: int
    connection: tuple
    edge_checks: int
    config_checks: int
    path: np.ndarray | None
    cost: float


def plan(scene: Scene, start, goals, lo, hi, *, max_iterations=10000, step_size=0.5,
         num_new_samples=128, balance_mode=1, tree_ratio=0.5, dynamic_domain=True,
         dd_alpha=1e-4, dd_radius=4.0, dd_min_radius=1.0, max_nodes=65536, granularity=16,
         collision_mode=0, collision_margin=0.02, edge_resolution=0.0) -> PlanResult:
    """Sequential pRRTC restatement (explorers advance in round-robin order)."""
    dim = scene.dim
    start = np.ascontiguousarray(start, dtype=np.float32).reshape(dim)
    goals = np.ascontiguousarray(goals, dtype=np.float32).reshape(-1, dim)
    lo = np.ascontiguousarray(lo, dtype=np.float32)
    hi = np.ascontiguousarray(hi, dtype=np.float32)
    p = OrcPlanParams(int(max_iterations), float(step_size), int(num_new_samples), int(balance_mode),
                      float(tree_ratio), int(bool(dynamic_domain)), float(dd_alpha), float(dd_radius),
                      float(dd_min_radius), dim, int(max_nodes), int(granularity), int(collision_mode),
                      float(collision_margin), float(edge_resolution))
    ta = np.zeros((dim, max_nodes), dtype=np.float32)
    tb = np.zeros((dim, max_nodes), dtype=np.float32)
    pa = np.zeros(max_nodes, dtype=np.int32)
    pb = np.zeros(max_nodes, dtype=np.int32)
    out = OrcPlanOut()
    out.tree_a, out.tree_b, out.parents_a, out.parents_b = _ptr(ta), _ptr(tb), _ptr(pa), _ptr(pb)
    rc = lib().orc_prrtc_plan(scene.ref, _ptr(start), _ptr(goals), goals.shape[0], _ptr(lo), _ptr(hi),
                              C.byref(p), C.byref(out))
    if rc == -2:
        raise ValueError("invalid planner arguments")
    path, cost = None, float("inf")
    conn = (out.connection[0], out.connection[1], out.connection[2])
    if out.solved == 1:
        path, cost = trace_path(ta, tb, pa, pb, conn)
    return PlanResult(out.solved, ta, tb, pa, pb, (out.tree_sizes[0], out.tree_sizes[1]),
                      (out.completed[0], out.completed[1]), out.iter_count, conn,
                      out.edge_checks, out.config_checks, path, cost)


def trace_path(ta, tb, pa, pb, conn, max_len: int = 1 << 16):
    dim, N = ta.shape
    path = np.zeros((max_len, dim), dtype=np.float32)
    c3 = (C.c_int * 3)(*conn)
    L = lib().orc_trace_path(_ptr(np.ascontiguousarray(ta)), _ptr(np.ascontiguousarray(tb)),
                             _ptr(np.ascontiguousarray(pa)), _ptr(np.ascontiguousarray(pb)), N, dim, c3,
                             _ptr(path), max_len)
    if L < 0:
        raise RuntimeError("path longer than max_len")
    path = path[:L].copy()
    return path, float(lib().orc_path_cost(_ptr(path), L, dim))


@dataclass
class HostPlanResult:
    solved: bool
    iterations: int
    size_a: int
    size_b: int
    path: np.ndarray | None
    cost: float
    config_checks: int


def rrtc_host_plan(scene: Scene, start, goal, lo, hi, *, max_iterations=5000, step_size=0.5,
                   num_new_samples=128, granularity=16, max_nodes=65536, connect_max_steps=32,
                   seed=0, collision_mode=0, collision_margin=0.02, n_threads=1,
                   max_path=4096) -> HostPlanResult:
    """Host-driven batched RRT-Connect, the reference's CPU path (prrtc_robogpu.py:103-298)."""
    dim = scene.dim
    s = np.ascontiguousarray(start, dtype=np.float32).reshape(dim)
    g = np.ascontiguousarray(goal, dtype=np.float32).reshape(-1, dim)[0].copy()
    lo = np.ascontiguousarray(lo, dtype=np.float32)
    hi = np.ascontiguousarray(hi, dtype=np.float32)
    path = np.zeros((max_path, dim), dtype=np.float32)
    out = OrcHostOut()
    lib().orc_rrtc_host_plan(scene.ref, _ptr(s), _ptr(g), _ptr(lo), _ptr(hi), int(max_iterations),
                             float(step_size), int(num_new_samples), int(granularity), int(max_nodes),
                             int(connect_max_steps), int(seed), int(collision_mode), float(collision_margin),
                             int(n_threads), _ptr(path), int(max_path), C.byref(out))
    p = path[: out.path_len].copy() if out.solved else None
    return HostPlanResult(bool(out.solved), out.iterations, out.size_a, out.size_b, p,
                          float(out.cost), int(out.config_checks))


def cpu_count() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1
