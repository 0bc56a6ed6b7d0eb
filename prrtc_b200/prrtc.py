"""pRRTC planning API -- drop-in mirror of P-RRAX's ``cuda-rrtc/jax/prrtc.py``.

Same function names, keyword arguments, defaults, validation and error
behaviour as the reference (prrtc.py:255-585 ``prrtc_plan``, 882-1434
``prrtc_plan_batch``, 1437-1508 ``prrtc_nearest_neighbor`` / ``prrtc_extend``),
with torch tensors in place of jax arrays.  All computation runs in
libprrtc_b200.so on the GPU; there is no CPU fallback.

Differences from the reference, all deliberate:
  * the host never blocks inside the planner call; scalars of the result are
    read once at the end;
  * the path is extracted by a device kernel (one read-back) instead of a
    per-node device->host walk (prrtc.py:603-631);
  * unused tree slots are NaN (the planner's "unwritten" sentinel), not 0;
    consumers slice by tree size exactly as the reference's results do;
  * extra keyword-only arguments: ``edge_resolution`` (raise the waypoints of an
    edge to ceil(len/res)), ``threads_per_explorer``, ``waypoint_chunk``;
    ``prrtc_plan_batch`` also takes ``goal_counts``, ``problem_order``,
    ``launch`` ("persistent" -- one persistent launch; "per_problem" -- one
    planner launch per problem over a pool of streams, the reference's form),
    ``tail_explorers`` (persistent launch: idle CTAs join problems that are
    still running once every explorer slot is taken; False keeps exactly
    ``num_new_samples`` explorers per problem, as the reference), and
    ``point_cloud`` / ``r_env`` (an environment point cloud checked inside the
    kernel, shared by the batch; a collision_context's ``point_cloud`` entry
    does the same), and ``ctas_per_sm`` (persistent launch: at most that many
    CTAs per SM with a shared-memory carve-out that just holds them, leaving
    the rest of the SM's memory to L1).
"""
from __future__ import annotations

import ctypes as C
from typing import NamedTuple, Optional, Sequence

import numpy as np
import torch

from . import _lib
from .device import REQUIRED_KEYS, DeviceContext, Stager, as_tensor, cuda_device, ptr, stream_handle, workspace

_COLLISION_MODES = {"binary": 0, "differentiable": 1, "binary_coarse": 2, "binary_coarse_coop": 3}
PATH_MAX_LEN = 16384
_SIDE_STREAMS: dict = {}


def _side_stream(device: torch.device) -> torch.cuda.Stream:
    """A stream of this module's own per device, for read-backs that must wait
    for one call only and not for later work queued on the caller's stream."""
    key = device.index if device.index is not None else torch.cuda.current_device()
    if key not in _SIDE_STREAMS:
        _SIDE_STREAMS[key] = torch.cuda.Stream(device=device)
    return _SIDE_STREAMS[key]


class PRRTCResult(NamedTuple):
    """Result of pRRTC planning (prrtc.py:31-45)."""

    solved: bool
    path: Optional[torch.Tensor]
    tree_a_size: int
    tree_b_size: int
    iterations: int
    cost: float
    kernel_time_ms: Optional[float] = None
    tree_a_configs: Optional[torch.Tensor] = None
    tree_b_configs: Optional[torch.Tensor] = None
    tree_a_parents: Optional[torch.Tensor] = None
    tree_b_parents: Optional[torch.Tensor] = None


def _resolve_collision_mode(collision_checker: str) -> int:
    """prrtc.py:57-73."""
    try:
        return _COLLISION_MODES[collision_checker]
    except KeyError:
        if collision_checker == "robogpu":
            raise ValueError(
                "collision_checker='robogpu' is not available in the in-kernel planner: the point-cloud "
                "checker runs host-driven. Use a host-driven planner loop with an external edge checker."
            ) from None
        raise ValueError(
            f"collision_checker must be one of {sorted(_COLLISION_MODES)}, got {collision_checker!r}"
        ) from None


def _validate(step_size, granularity):
    step_size = float(step_size)
    if step_size <= 0.0:
        raise ValueError("step_size must be > 0")
    granularity = int(granularity)
    if granularity < 1 or (granularity & (granularity - 1)) != 0:
        raise ValueError(f"granularity must be a power of 2, got {granularity}")
    if granularity > 64:
        raise ValueError(f"granularity must be <= 64 (PRRTC_BLOCK_THREADS_MAX), got {granularity}")
    return step_size, granularity


def _check_context(collision_context, allow_unsafe_no_collision):
    if collision_context is None and not allow_unsafe_no_collision:
        raise ValueError(
            "Collision-aware planning is the default. Provide collision_context "
            "with required keys or set allow_unsafe_no_collision=True to opt out. "
            f"Required keys: {REQUIRED_KEYS}"
        )
    if collision_context is not None:
        missing = [k for k in REQUIRED_KEYS if k not in collision_context]
        if missing:
            raise ValueError(f"collision_context missing required keys: {missing}")


def _attrs(max_iterations, step_size, num_new_samples, balance_mode, tree_ratio, dynamic_domain, dd_alpha,
           dd_radius, dd_min_radius, dim, max_nodes, granularity, collision_mode, collision_margin) -> _lib.Attrs:
    a = _lib.Attrs()
    a.max_iterations = int(min(max_iterations, 2**31 - 1))
    a.step_size = float(step_size)
    a.num_new_samples = int(num_new_samples)
    a.balance_mode = int(balance_mode)
    a.tree_ratio = float(tree_ratio)
    a.dynamic_domain = 1 if dynamic_domain else 0
    a.dd_alpha = float(dd_alpha)
    a.dd_radius = float(dd_radius)
    a.dd_min_radius = float(dd_min_radius)
    a.dim = int(dim)
    a.max_nodes = int(max_nodes)
    a.granularity = int(granularity)
    a.collision_mode = int(collision_mode)
    a.collision_margin = float(collision_margin)
    return a


def _tuning(edge_resolution=0.0, threads_per_explorer=0, waypoint_chunk=0, resident_ctas=0,
            tail_explorers=True, ctas_per_sm=0) -> _lib.Tuning:
    t = _lib.Tuning()
    t.ctas_per_sm = int(ctas_per_sm or 0)
    t.tail_explorers = 0 if tail_explorers else -1
    t.edge_resolution = float(edge_resolution or 0.0)
    t.threads_per_explorer = int(threads_per_explorer or 0)
    t.waypoint_chunk = int(waypoint_chunk or 0)
    t.resident_ctas = int(resident_ctas or 0)
    return t


def _outputs_struct(ta, tb, pa, pb, sizes, completed, iters, conn, solved, ktime) -> _lib.Outputs:
    o = _lib.Outputs()
    o.tree_a_configs, o.tree_b_configs = ta.data_ptr(), tb.data_ptr()
    o.tree_a_parents, o.tree_b_parents = pa.data_ptr(), pb.data_ptr()
    o.tree_sizes, o.completed, o.iter_count = sizes.data_ptr(), completed.data_ptr(), iters.data_ptr()
    o.connection_info, o.solved_flag, o.kernel_time_ms = conn.data_ptr(), solved.data_ptr(), ktime.data_ptr()
    return o


class _Results:
    """Raw planner outputs of B problems plus device-extracted paths."""

    def __init__(self, B: int, dim: int, N: int, device: torch.device, lead: tuple):
        self.B, self.dim, self.N = B, dim, N
        self.caps = None  # per-problem tree capacities, when they differ from N
        self.ta = torch.empty(lead + (dim, N), dtype=torch.float32, device=device)
        self.tb = torch.empty(lead + (dim, N), dtype=torch.float32, device=device)
        self.pa = torch.empty(lead + (N,), dtype=torch.int32, device=device)
        self.pb = torch.empty(lead + (N,), dtype=torch.int32, device=device)
        # scalars packed into one int32 block [B, 16] -> a single device->host copy
        self.block = torch.zeros((B, 16), dtype=torch.int32, device=device)
        self.sizes = torch.empty((B, 2), dtype=torch.int32, device=device)
        self.completed = torch.empty((B, 2), dtype=torch.int32, device=device)
        self.iters = torch.empty((B, 1), dtype=torch.int32, device=device)
        self.conn = torch.empty((B, 3), dtype=torch.int32, device=device)
        self.solved = torch.empty((B, 1), dtype=torch.int32, device=device)
        self.ktime = torch.empty((B,), dtype=torch.float32, device=device)
        self.max_len = int(min(PATH_MAX_LEN, 2 * N + 2))
        self.paths = torch.empty((B, self.max_len, dim), dtype=torch.float32, device=device)
        self.lengths = torch.empty((B,), dtype=torch.int32, device=device)
        self.costs = torch.empty((B,), dtype=torch.float32, device=device)
        self.packed = self.packed_h = self.block_h = self.ready = None
        self.d2h_bytes = 0  # device->host bytes of the read-back

    def outputs(self) -> _lib.Outputs:
        return _outputs_struct(self.ta, self.tb, self.pa, self.pb, self.sizes, self.completed, self.iters,
                               self.conn, self.solved, self.ktime)

    def extract(self, stream_ptr: int, pack_paths: bool = False) -> None:
        """Queue path extraction and the result block; with ``pack_paths`` the
        solved paths are also copied back to back into ``self.packed`` (the
        block's column 12 holds each path's first row there)."""
        lib = _lib.load()
        _lib.check(lib.prrtc_b200_extract_paths(self.B, self.dim, self.N, ptr(self.ta), ptr(self.tb), ptr(self.pa),
                                                ptr(self.pb), ptr(self.conn), ptr(self.solved), self.max_len,
                                                ptr(self.paths), ptr(self.lengths), ptr(self.costs), stream_ptr),
                   "prrtc_b200_extract_paths")
        # room for an average of 128 waypoints per path (at least 65536 in all);
        # a path past it is read from the path buffer on its own
        rows = min(self.B * self.max_len, max(128 * self.B, 65536))
        self.packed = (torch.empty((rows, self.dim), dtype=torch.float32, device=self.paths.device)
                       if pack_paths else None)
        _lib.check(lib.prrtc_b200_result_block(
            self.B, self.dim, self.max_len, ptr(self.sizes), ptr(self.completed), ptr(self.iters), ptr(self.conn),
            ptr(self.solved), ptr(self.ktime), ptr(self.lengths), ptr(self.costs), ptr(self.paths), ptr(self.block),
            ptr(self.packed), 0 if self.packed is None else self.packed.shape[0], stream_ptr),
            "prrtc_b200_result_block")

    def prefetch_host(self, path_rows: int = 0) -> None:
        """Queue, on the current stream right behind the planner's kernels, the
        device->host copies that ``to_results`` needs: the result block and the
        first ``path_rows`` rows of the packed paths, into pinned memory, then an
        event.  Copies issued this way run on the copy engine as soon as this
        call's kernels are done; a copy issued later, when the stream or the
        GPU already holds the next call's persistent planner, would wait for it."""
        self.block_h = torch.empty((self.B, 16), dtype=torch.int32, pin_memory=True)
        self.block_h.copy_(self.block, non_blocking=True)
        self.d2h_bytes = self.block.numel() * 4
        self.packed_h = None
        if self.packed is not None and path_rows > 0:
            n = min(int(path_rows), self.packed.shape[0])
            self.packed_h = torch.empty((n, self.dim), dtype=torch.float32, pin_memory=True)
            self.packed_h.copy_(self.packed[:n], non_blocking=True)
            self.d2h_bytes += self.packed_h.numel() * 4
        self.ready = torch.cuda.Event()
        self.ready.record()

    def _host_paths(self, host: np.ndarray) -> Optional[np.ndarray]:
        """Every solved path on the host: rows of the packed paths (prefetched,
        plus the rest copied now on a side stream that waits only for this
        call), or the [B, longest] slice of the path buffer."""
        if self.packed is None:
            lmax = int(max(0, host[:, 10].max())) if self.B else 0
            return self.paths[:, :lmax].cpu().numpy() if lmax > 0 else None
        ok = host[:, 12] >= 0
        total = int((host[ok, 12] + host[ok, 10]).max()) if ok.any() else 0
        if self.ready is None:  # nothing prefetched: read on the caller's stream
            return self.packed[:total].cpu().numpy() if total else None
        have = 0 if self.packed_h is None else self.packed_h.shape[0]
        parts = [self.packed_h.numpy()[:min(have, total)]] if have else []
        if total > have:
            side = _side_stream(self.packed.device)
            side.wait_event(self.ready)
            with torch.cuda.stream(side):
                rest = torch.empty((total - have, self.dim), dtype=torch.float32, pin_memory=True)
                rest.copy_(self.packed[have:total], non_blocking=True)
            self.d2h_bytes += rest.numel() * 4
            side.synchronize()
            parts.append(rest.numpy())
        # a private copy: the pinned blocks go back to the allocator's cache now
        return np.concatenate(parts, 0) if len(parts) > 1 else (parts[0].copy() if parts else None)

    def to_results(self, trees: bool = True, paths_on_host: bool = False,
                   timeout_s: Optional[float] = None) -> list[PRRTCResult]:
        """One read-back of the [B,16] scalar block (plus, with paths_on_host, one
        bulk copy of every path) and the per-problem PRRTCResults.  With
        ``timeout_s``, the wait for the call's kernels polls and raises
        PrrtcTimeout after that many seconds."""
        if self.ready is not None:
            _lib.wait_event(self.ready, timeout_s, "planner results")
            host = self.block_h.numpy().copy()
        else:
            if timeout_s is not None:
                done = torch.cuda.Event()
                done.record()
                _lib.wait_event(done, timeout_s, "planner results")
            host = self.block.cpu().numpy()
        if (host[:, 8] == -2).any():
            raise _lib.PrrtcError("a device-side wait ran out (scene staging): the planner stopped and these "
                                  "results are incomplete")
        hpaths = self._host_paths(host) if paths_on_host else None
        packed = self.packed is not None and paths_on_host
        out = []
        # plain Python scalars for the per-problem loop (numpy scalar access is slow)
        rows = host.tolist()
        kts = host[:, 9].copy().view(np.float32).tolist()
        costs = host[:, 11].copy().view(np.float32).tolist()
        inf = float("inf")
        make = tuple.__new__  # positional construction: the loop runs once per problem
        from_numpy = torch.from_numpy
        for i in range(self.B):
            row = rows[i]
            solved = row[8] == 1
            size_a, size_b = row[0], row[1]
            length = row[10]
            cost = costs[i] if solved else inf
            path = None
            if solved:
                if length > 0 and packed:
                    path = (from_numpy(hpaths[row[12]:row[12] + length]) if row[12] >= 0
                            else self._path_row(i, length))  # past the packed capacity
                elif length > 0:
                    path = from_numpy(hpaths[i, :length]) if hpaths is not None else self.paths[i, :length]
                else:  # longer than the device path buffer: walk on the host
                    path = self._host_trace(i)
                    cost = float(torch.linalg.norm(torch.diff(path, dim=0), dim=1).sum())
                    if paths_on_host:
                        path = path.cpu()
            tac = tbc = tap = tbp = None
            if trees:  # per-problem views only when asked for (each is a tensor op)
                cap = self.N if self.caps is None else min(int(self.caps[i]), self.N)
                na, nb = min(size_a, cap), min(size_b, cap)
                batched = self.ta.dim() == 3
                tac = (self.ta[i] if batched else self.ta)[:, :na]
                tbc = (self.tb[i] if batched else self.tb)[:, :nb]
                tap = (self.pa[i] if batched else self.pa)[:na]
                tbp = (self.pb[i] if batched else self.pb)[:nb]
            # field order of PRRTCResult
            out.append(make(PRRTCResult, (solved, path, size_a, size_b, row[4], cost, kts[i], tac, tbc, tap, tbp)))
        return out

    def _path_row(self, i: int, length: int) -> torch.Tensor:
        """Path i from the path buffer to the host, on the side stream (waits for
        this call only)."""
        if self.ready is None:
            return self.paths[i, :length].cpu()
        side = _side_stream(self.paths.device)
        side.wait_event(self.ready)
        with torch.cuda.stream(side):
            out = self.paths[i, :length].to("cpu", non_blocking=True)
        side.synchronize()
        self.d2h_bytes += out.numel() * 4
        return out

    def _host_trace(self, i: int) -> torch.Tensor:
        ta = (self.ta[i] if self.ta.dim() == 3 else self.ta).cpu()
        tb = (self.tb[i] if self.tb.dim() == 3 else self.tb).cpu()
        pa = (self.pa[i] if self.pa.dim() == 2 else self.pa).cpu().numpy()
        pb = (self.pb[i] if self.pb.dim() == 2 else self.pb).cpu().numpy()
        a, b = (int(x) for x in self.conn[i, :2].cpu())
        nodes, curr = [], a
        for _ in range(self.N):
            nodes.append(ta[:, curr])
            if pa[curr] == curr:
                break
            curr = int(pa[curr])
        nodes.reverse()
        curr = b
        for _ in range(self.N):
            nodes.append(tb[:, curr])
            if pb[curr] == curr:
                break
            curr = int(pb[curr])
        return torch.stack(nodes, 0).to(self.paths.device)


def prrtc_plan(
    start_config,
    goal_configs,
    max_iterations: int = 1_000_000,
    step_size: float = 0.5,
    num_new_samples: int = 128,
    granularity: int = 16,
    max_nodes: int = 1_000_000,
    balance_mode: int = 1,
    tree_ratio: float = 0.5,
    dynamic_domain: bool = True,
    dd_alpha: float = 1e-4,
    dd_radius: float = 4.0,
    dd_min_radius: float = 1.0,
    min_vals=None,
    max_vals=None,
    collision_context: Optional[dict] = None,
    allow_unsafe_no_collision: bool = False,
    jit_trace: bool = False,
    collision_checker: str = "binary",
    collision_margin: float = 0.02,
    *,
    edge_resolution: float = 0.0,
    threads_per_explorer: int = 0,
    waypoint_chunk: int = 0,
    device=None,
    timeout_s: Optional[float] = None,
) -> PRRTCResult:
    """Plan one problem with the parallel bidirectional RRT-Connect planner (prrtc.py:255-585).

    ``jit_trace`` is accepted for signature compatibility; the call is already a
    single asynchronous C-ABI dispatch.  ``timeout_s`` bounds the host's wait
    for the result (PrrtcTimeout after that many seconds; None waits for good).
    """
    collision_mode = _resolve_collision_mode(collision_checker)
    lib = _lib.load()
    collision_margin = float(collision_margin)
    start_shape = tuple(start_config.shape) if hasattr(start_config, "shape") else np.shape(start_config)
    start_rows = 1 if len(start_shape) <= 1 else int(np.prod(start_shape[:-1]))
    if start_rows != 1:
        raise ValueError(
            "prrtc_plan currently accepts a single start configuration per call. "
            "For batches, call prrtc_plan_batch."
        )
    step_size, granularity = _validate(step_size, granularity)
    _check_context(collision_context, allow_unsafe_no_collision)
    dev = cuda_device(device)
    # every host input of the call (start, goals, limits, robot and world
    # tables) goes to the device in one pinned copy, not one blocking pageable
    # copy per table; tensors already on the device pass through
    stage = Stager(dev)
    if isinstance(start_config, torch.Tensor):
        dim = int(start_config.numel())
    else:
        dim = int(np.asarray(start_config).size)
    k_start = stage.add(start_config, torch.float32, (dim,))
    k_goals = stage.add(goal_configs, torch.float32, (-1, dim))
    k_lo = stage.add(np.full(dim, -np.pi, np.float32) if min_vals is None else min_vals, torch.float32, (dim,))
    k_hi = stage.add(np.full(dim, np.pi, np.float32) if max_vals is None else max_vals, torch.float32, (dim,))
    ctx = DeviceContext(collision_context, dev, stager=stage)
    stage.commit()
    ctx.finish()
    start, goals, lo, hi = (stage.get(k) for k in (k_start, k_goals, k_lo, k_hi))

    inp = _lib.Inputs()
    inp.start_config, inp.goal_configs, inp.num_goals = start.data_ptr(), goals.data_ptr(), goals.shape[0]
    inp.min_vals, inp.max_vals = lo.data_ptr(), hi.data_ptr()
    inp.robot, inp.world = ctx.robot(), ctx.world()
    attrs = _attrs(max_iterations, step_size, num_new_samples, balance_mode, tree_ratio, dynamic_domain, dd_alpha,
                   dd_radius, dd_min_radius, dim, max_nodes, granularity, collision_mode, collision_margin)
    tun = _tuning(edge_resolution, threads_per_explorer, waypoint_chunk)
    from .pointcloud import cloud_from_context

    cloud = cloud_from_context(collision_context, dev)  # optional "point_cloud" [M,3] + "r_env"
    if cloud is not None:
        tun.point_cloud = cloud.address()
    res = _Results(1, dim, int(max_nodes), dev, ())
    ws = workspace(lib.prrtc_b200_plan_workspace_size(C.byref(inp), C.byref(attrs), C.byref(tun)), dev)
    sp = stream_handle()
    outs = res.outputs()
    _lib.check(lib.prrtc_b200_plan(C.byref(inp), C.byref(outs), C.byref(attrs), C.byref(tun), ws.data_ptr(),
                                   ws.numel(), sp), "prrtc_b200_plan")
    res.extract(sp)
    return res.to_results(timeout_s=timeout_s)[0]


_TABLES = (("world_spheres", 4, np.float32), ("world_capsules", 7, np.float32), ("world_boxes", 15, np.float32),
           ("world_halfspaces", 6, np.float32), ("self_pairs", 2, np.int32))
_FEAT = {k: f for k, f, _ in _TABLES}


def _tables(contexts: Sequence[Optional[dict]], key: str, feat: int, dt) -> list:
    """Table `key` of every context as a 2-D array (absent = zero rows)."""
    out = []
    empty = np.zeros((0, feat), dtype=dt)
    for i, c in enumerate(contexts):
        x = None if c is None else c.get(key)
        if x is None:
            out.append(empty)
            continue
        a = x if (isinstance(x, np.ndarray) and x.dtype == dt) else np.asarray(x, dtype=dt)
        if a.ndim != 2 or a.shape[1] != feat:
            raise ValueError(f"collision_context[{i}]['{key}'] must have shape (N, {feat}), got {a.shape}")
        out.append(a)
    return out


def _pack_worlds(contexts: Sequence[Optional[dict]], B: int, skip=()):
    """Padded [B, max_n, feat] world/self tensors + counts (prrtc.py:1009-1067);
    keys in `skip` are left out."""
    packed, counts = {}, {}
    for key, feat, dt in _TABLES:
        if key in skip:
            continue
        arrs = _tables(contexts, key, feat, dt)
        n = np.fromiter((a.shape[0] for a in arrs), dtype=np.int32, count=len(arrs))
        m = int(n.max()) if B else 0
        p = np.zeros((B, m, feat), dtype=dt)
        total = int(n.sum())
        if total:
            # one scatter: row r of the concatenation goes to (problem, row within problem)
            flat = np.concatenate(arrs, axis=0)
            prob = np.repeat(np.arange(B), n)
            within = np.arange(total) - np.repeat(np.cumsum(n) - n, n)
            p[prob, within] = flat
        packed[key], counts[key] = p, n
    return packed, counts


def _shared_table(contexts: Sequence[Optional[dict]], key: str):
    """The table `key` when every context holds the same one (same object or
    equal contents), else None."""
    first = contexts[0].get(key) if contexts and contexts[0] is not None else None
    if first is None:
        return None
    a0 = np.asarray(first)
    b0 = None
    for c in contexts[1:]:
        if c is None:
            return None
        x = c.get(key)
        if x is first:
            continue
        if x is None:
            return None
        x = np.asarray(x)
        if x.shape != a0.shape:
            return None
        if x.size == 0:
            continue
        if b0 is None:
            b0 = a0.tobytes()
        if x.tobytes() != b0:
            return None
    return np.ascontiguousarray(a0, dtype=np.int32 if key == "self_pairs" else np.float32).reshape(-1, _FEAT[key])


_PACK_SPECS = tuple((k, f, "i" if dt == np.int32 else "f") for k, f, dt in _TABLES)


def _native_pack(contexts: Sequence[Optional[dict]], stage: Stager):
    """The world / self tables of every context packed by the native host
    packer straight into the call's pinned staging buffer: padded
    [B, max_n, feat] tables + int32 counts, or one copy of a table every
    context shares (same layout as _pack_worlds / _shared_table; rows past a
    problem's count are left unwritten, the planner never reads them).  Returns
    ({key: (table key, counts key or None, width)}, {key: counts}), or None
    when some table is not a C-contiguous float32 / int32 numpy array (the
    Python packer then handles the call)."""
    hp = _lib.hostpack()
    try:
        info = hp.scan(contexts, _PACK_SPECS)
    except TypeError:
        return None
    B = len(contexts)
    world_keys, counts, layout = {}, {}, []
    for (key, feat, kind), (shared, width, cbytes) in zip(_PACK_SPECS, info):
        dt = torch.int32 if kind == "i" else torch.float32
        if shared:
            rows = int(np.frombuffer(cbytes, np.int32)[0])
            k_tab = stage.reserve(dt, (rows, feat))
            world_keys[key] = (k_tab, None, rows)
            layout.append((True, rows, k_tab, None))
        else:
            counts[key] = np.frombuffer(cbytes, np.int32)
            k_tab, k_cnt = stage.reserve(dt, (B, width, feat)), stage.reserve(torch.int32, (B,))
            world_keys[key] = (k_tab, k_cnt, width)
            layout.append((False, width, k_tab, k_cnt))

    def fill(hv, offset_of):
        hp.fill(contexts, _PACK_SPECS,
                [(s, w, offset_of(kt), offset_of(kc) if kc is not None else -1) for s, w, kt, kc in layout], hv)

    stage.on_fill(fill)
    return world_keys, counts


_LPT_WEIGHTS = (("world_spheres", 1.0), ("world_capsules", 2.0), ("world_boxes", 3.0), ("world_halfspaces", 1.0))


def _lpt_from_counts(counts: dict, B: int) -> np.ndarray:
    """lpt_order from the per-problem row counts of the packed tables (a table
    shared by every problem adds the same cost to each and is left out)."""
    cost = np.zeros(B, dtype=np.float64)
    for k, w in _LPT_WEIGHTS:
        if k in counts:
            cost += w * counts[k]
    return np.argsort(-cost, kind="stable").astype(np.int32)


def lpt_order(contexts: Sequence[Optional[dict]], goal_counts=None) -> np.ndarray:
    """Longest-processing-time order: problems with the most collision work first."""
    cost = np.zeros(len(contexts), dtype=np.float64)
    for k, w in _LPT_WEIGHTS:
        cost += w * np.fromiter(((0 if c is None or c.get(k) is None else len(c[k])) for c in contexts),
                                dtype=np.float64, count=len(contexts))
    return np.argsort(-cost, kind="stable").astype(np.int32)


def prrtc_plan_batch_async(
    start_configs,
    goal_configs,
    max_iterations: int = 1_000_000,
    step_size: float = 0.5,
    num_new_samples: int = 128,
    granularity: int = 16,
    max_nodes: int = 1_000_000,
    balance_mode: int = 1,
    tree_ratio: float = 0.5,
    dynamic_domain: bool = True,
    dd_alpha: float = 1e-4,
    dd_radius: float = 4.0,
    dd_min_radius: float = 1.0,
    min_vals=None,
    max_vals=None,
    collision_context=None,
    allow_unsafe_no_collision: bool = False,
    jit_trace: bool = False,
    collision_checker: str = "binary",
    collision_margin: float = 0.02,
    *,
    goal_counts=None,
    problem_order="auto",
    launch: str = "persistent",
    edge_resolution: float = 0.0,
    threads_per_explorer: int = 0,
    waypoint_chunk: int = 0,
    resident_ctas: int = 0,
    return_trees: bool = True,
    paths_on_host: bool = False,
    point_cloud=None,
    r_env: float = 0.02,
    tail_explorers: bool = True,
    ctas_per_sm: int = 0,
    device=None,
) -> "PendingBatch":
    """Plan B independent problems (prrtc.py:882-1434), without waiting: the
    work is queued on the current stream and ``.results()`` of the returned
    handle reads it back.  Several batches can be in flight at once; queue
    back-to-back batches on ONE stream.  The persistent planner holds every SM
    until its batch is done, so a planner launch queued on a second stream
    takes the SMs that the first batch's tail frees, and the first batch's
    closing kernels (finalize, path extraction) then wait for the whole second
    batch.  Each call queues its device->host read-back right behind its own
    kernels, so ``.results()`` of an earlier call waits for that call only,
    not for later calls on the same stream.

    ``collision_context`` is one dict shared by every problem, or a list/tuple of
    per-problem dicts (robot tables from the first non-None entry; worlds and
    self pairs packed into padded tensors with counts).  ``paths_on_host``
    returns every path as a CPU tensor, copied with one bulk device->host copy.
    ``max_nodes`` may also be a per-problem sequence of tree capacities: the
    problems then share one launch (row stride = the largest capacity) and
    each tree overflows at its own capacity.
    """
    caps = None
    if isinstance(max_nodes, (list, tuple, np.ndarray, torch.Tensor)):
        caps = np.asarray(max_nodes.cpu() if isinstance(max_nodes, torch.Tensor) else max_nodes,
                          dtype=np.int64).reshape(-1)
        if caps.size == 0 or (caps < 1).any():
            raise ValueError("per-problem max_nodes must be >= 1")
        max_nodes = int(caps.max())
    lib = _lib.load()
    collision_mode = _resolve_collision_mode(collision_checker)
    step_size, granularity = _validate(step_size, granularity)
    if collision_context is None:
        _check_context(None, allow_unsafe_no_collision)
    dev = cuda_device(device)
    # every host input of the call (configs, limits, counts, order, capacities,
    # robot tables, packed worlds) goes to the device in one pinned copy
    stage = Stager(dev)
    starts_np = starts_dev = None
    if isinstance(start_configs, torch.Tensor) and start_configs.device == dev:
        starts_dev = start_configs.to(torch.float32)
        shape = tuple(starts_dev.shape)
    else:
        starts_np = np.asarray(start_configs.cpu() if isinstance(start_configs, torch.Tensor) else start_configs,
                               dtype=np.float32)
        shape = starts_np.shape
    if len(shape) == 1:
        shape = (1,) + shape
    B, dim = int(shape[0]), int(shape[1])
    k_starts = stage.add(starts_dev if starts_dev is not None else starts_np, torch.float32, (B, dim))
    gshape = tuple(goal_configs.shape) if isinstance(goal_configs, torch.Tensor) else np.shape(goal_configs)
    if len(gshape) == 2:
        gshape = (gshape[0], 1, gshape[1])
    if len(gshape) != 3 or gshape[0] != B:
        raise ValueError(f"goal_configs must have shape (batch, num_goals, dim), got {tuple(gshape)} "
                         f"with batch_size={B}")
    G = int(gshape[1])
    k_goals = stage.add(goal_configs, torch.float32, gshape)
    k_lo = stage.add(np.full(dim, -np.pi, np.float32) if min_vals is None else min_vals, torch.float32, (dim,))
    k_hi = stage.add(np.full(dim, np.pi, np.float32) if max_vals is None else max_vals, torch.float32, (dim,))
    k_gc = stage.add(goal_counts, torch.int32, (B,)) if goal_counts is not None else None

    per_problem = isinstance(collision_context, (list, tuple))
    if per_problem:
        if len(collision_context) != B:
            raise ValueError("When collision_context is a list/tuple, it must have length "
                             f"equal to batch_size ({B}), got {len(collision_context)}")
        contexts = list(collision_context)
        first = next((c for c in contexts if c is not None), None)
        if first is None:
            _check_context(None, allow_unsafe_no_collision)
        else:
            for i, c in enumerate(contexts):
                if c is not None:
                    missing = [k for k in REQUIRED_KEYS if k not in c]
                    if missing:
                        raise ValueError(f"collision_context[{i}] missing required keys: {missing}")
    else:
        _check_context(collision_context, allow_unsafe_no_collision)
        contexts = [collision_context] * B
        first = collision_context

    robot_ctx = DeviceContext(first, dev, world_keys=not per_problem, stager=stage)
    keys = ("world_spheres", "world_capsules", "world_boxes", "world_halfspaces", "self_pairs")
    world_keys, counts = {}, None
    native = _native_pack(contexts, stage) if per_problem and first is not None else None
    if native is not None:
        world_keys, counts = native
    elif per_problem and first is not None:
        # a table every problem shares (typically the robot's self pairs) goes
        # once, unbatched, with no count pointer
        shared = {k: _shared_table(contexts, k) for k in keys}
        packed, counts = _pack_worlds(contexts, B, skip={k for k in keys if shared[k] is not None})
        for key in keys:
            if shared[key] is not None:
                world_keys[key] = (stage.add(shared[key], torch.int32 if key == "self_pairs" else torch.float32),
                                   None, int(shared[key].shape[0]))
            else:
                world_keys[key] = (stage.add(packed[key], torch.int32 if key == "self_pairs" else torch.float32),
                                   stage.add(counts[key], torch.int32), int(packed[key].shape[1]))
    order = None
    if isinstance(problem_order, str):
        if problem_order == "auto" and per_problem:
            # longest-processing-time order from the packed counts (same order as lpt_order)
            order = _lpt_from_counts(counts, B) if counts is not None else lpt_order(contexts)
    elif problem_order is not None:
        order = np.asarray(problem_order, dtype=np.int32).reshape(B)
    k_order = stage.add(order, torch.int32) if order is not None else None
    k_caps = None
    if caps is not None:
        if caps.size != B:
            raise ValueError(f"per-problem max_nodes must have batch_size ({B}) entries, got {caps.size}")
        k_caps = stage.add(caps, torch.int32)
    stage.commit()
    robot_ctx.finish()

    starts, goals, lo, hi = stage.get(k_starts), stage.get(k_goals), stage.get(k_lo), stage.get(k_hi)
    bi = _lib.BatchInputs()
    bi.batch = B
    bi.start_configs, bi.goal_configs, bi.num_goals = starts.data_ptr(), goals.data_ptr(), G
    keep = [stage]
    if k_gc is not None:
        bi.goal_counts = stage.get(k_gc).data_ptr()
    bi.min_vals, bi.max_vals = lo.data_ptr(), hi.data_ptr()
    bi.robot = robot_ctx.robot()
    if world_keys:
        for key, (k_tab, k_cnt, width) in world_keys.items():
            setattr(bi, key, ptr(stage.get(k_tab)))
            setattr(bi, "max_" + key, width)
            setattr(bi, key + "_count", ptr(stage.get(k_cnt)) if k_cnt is not None else None)
    elif first is not None:
        w = robot_ctx.world()
        bi.world_spheres, bi.max_world_spheres = w.world_spheres, w.n_world_spheres
        bi.world_capsules, bi.max_world_capsules = w.world_capsules, w.n_world_capsules
        bi.world_boxes, bi.max_world_boxes = w.world_boxes, w.n_world_boxes
        bi.world_halfspaces, bi.max_world_halfspaces = w.world_halfspaces, w.n_world_halfspaces
        bi.self_pairs, bi.max_self_pairs = w.self_pairs, w.n_self_pairs
    if k_order is not None:
        bi.problem_order = stage.get(k_order).data_ptr()
    if k_caps is not None:
        bi.problem_capacity = stage.get(k_caps).data_ptr()
    attrs = _attrs(max_iterations, step_size, num_new_samples, balance_mode, tree_ratio, dynamic_domain, dd_alpha,
                   dd_radius, dd_min_radius, dim, max_nodes, granularity, collision_mode, collision_margin)
    tun = _tuning(edge_resolution, threads_per_explorer, waypoint_chunk, resident_ctas, tail_explorers, ctas_per_sm)
    from .pointcloud import PointCloud, cloud_from_context

    # one environment point cloud for the whole batch: a PointCloud, or the
    # "point_cloud" entry of the first collision_context that has one
    cloud = point_cloud if isinstance(point_cloud, PointCloud) else None
    if cloud is None:
        src = {"point_cloud": point_cloud, "r_env": r_env} if point_cloud is not None else next(
            (c for c in contexts if c is not None and c.get("point_cloud") is not None), None)
        cloud = cloud_from_context(src, dev)
    if cloud is not None:
        tun.point_cloud = cloud.address()
        keep.append(cloud)
    res = _Results(B, dim, int(max_nodes), dev, (B,))
    res.caps = caps
    sp = stream_handle()
    if launch == "persistent":
        ws = workspace(lib.prrtc_b200_plan_batch_workspace_size(C.byref(bi), C.byref(attrs), C.byref(tun)), dev)
        outs = res.outputs()
        _lib.check(lib.prrtc_b200_plan_batch(C.byref(bi), C.byref(outs), C.byref(attrs), C.byref(tun),
                                             ws.data_ptr(), ws.numel(), sp), "prrtc_b200_plan_batch")
    elif launch == "per_problem":
        if caps is not None:
            raise ValueError("per-problem max_nodes needs launch='persistent'")
        _plan_per_problem(lib, bi, res, attrs, tun, contexts, robot_ctx, starts, goals, goal_counts, lo, hi, dev)
    else:
        raise ValueError(f"launch must be 'persistent' or 'per_problem', got {launch!r}")
    res.extract(sp, pack_paths=paths_on_host)
    # the read-back is queued now, behind this call's kernels (about 24 waypoints
    # per path prefetched; longer paths cost one more copy in results())
    res.prefetch_host(24 * B if paths_on_host else 0)
    # everything the queued kernels read stays referenced until results()
    keep += [robot_ctx] + ([ws] if launch == "persistent" else [])
    return PendingBatch(res, keep, torch.cuda.current_stream(dev), return_trees, paths_on_host)


class PendingBatch:
    """A queued batch: its outputs plus every input it still reads."""

    def __init__(self, res: "_Results", keep: list, stream, trees: bool, paths_on_host: bool):
        self.res, self.keep, self.stream = res, keep, stream
        self.trees, self.paths_on_host = trees, paths_on_host

    def results(self, timeout_s: Optional[float] = None) -> list[PRRTCResult]:
        """The batch's results, waiting for its kernels: blocking, or with
        ``timeout_s`` polling and raising PrrtcTimeout after that many seconds
        (the batch then stays pending and ``results`` can be called again)."""
        with torch.cuda.stream(self.stream):
            out = self.res.to_results(trees=self.trees, paths_on_host=self.paths_on_host, timeout_s=timeout_s)
        self.keep = []
        return out

    @property
    def d2h_bytes(self) -> int:
        """Bytes read back to the host by the prefetch and ``results()``."""
        return self.res.d2h_bytes


def prrtc_plan_batch(start_configs, goal_configs, *args, timeout_s: Optional[float] = None,
                     **kwargs) -> list[PRRTCResult]:
    """Plan B independent problems (prrtc.py:882-1434): the arguments of
    ``prrtc_plan_batch_async``, waiting for the results (``timeout_s``: see
    ``PendingBatch.results``)."""
    return prrtc_plan_batch_async(start_configs, goal_configs, *args, **kwargs).results(timeout_s=timeout_s)


def _plan_per_problem(lib, bi, res, attrs, tun, contexts, robot_ctx, starts, goals, goal_counts, lo, hi, dev,
                      n_streams: int = 8):
    """One plain planner launch per problem over a pool of streams (the reference's
    batch handlers launch each problem on its own child stream, prrtc_planner.cu:1785-1900)."""
    B, dim, G = int(starts.shape[0]), int(starts.shape[1]), int(goals.shape[1])
    main = torch.cuda.current_stream()
    streams = [torch.cuda.Stream(device=dev) for _ in range(min(n_streams, B))]
    ev = torch.cuda.Event()
    ev.record(main)
    gcs = None if goal_counts is None else np.asarray(goal_counts).reshape(B)
    keep = []
    for i in range(B):
        s = streams[i % len(streams)]
        s.wait_event(ev)
        ctx = DeviceContext(contexts[i], dev) if contexts[i] is not None else DeviceContext(None, dev)
        keep.append(ctx)
        inp = _lib.Inputs()
        inp.start_config = starts[i].data_ptr()
        ng = G if gcs is None else max(1, min(int(gcs[i]), G))
        inp.goal_configs, inp.num_goals = goals[i].data_ptr(), ng
        inp.min_vals, inp.max_vals = lo.data_ptr(), hi.data_ptr()
        inp.robot, inp.world = ctx.robot(), ctx.world()
        outs = _outputs_struct(res.ta[i], res.tb[i], res.pa[i], res.pb[i], res.sizes[i], res.completed[i],
                               res.iters[i], res.conn[i], res.solved[i], res.ktime[i:i + 1])
        ws = workspace(lib.prrtc_b200_plan_workspace_size(C.byref(inp), C.byref(attrs), C.byref(tun)), dev)
        ws.record_stream(s)
        keep.append(ws)
        _lib.check(lib.prrtc_b200_plan(C.byref(inp), C.byref(outs), C.byref(attrs), C.byref(tun), ws.data_ptr(),
                                       ws.numel(), s.cuda_stream), "prrtc_b200_plan")
    for s in streams:
        main.wait_stream(s)
    torch.cuda.current_stream().synchronize()


def prrtc_nearest_neighbor(tree_configs, query_configs, tree_size):
    """Nearest tree node of each query (prrtc.py:1437-1469).  Returns (distances, indices)."""
    lib = _lib.load()
    dev = cuda_device(tree_configs.device if isinstance(tree_configs, torch.Tensor) else None)
    tree = as_tensor(tree_configs, torch.float32, dev)
    q = as_tensor(query_configs, torch.float32, dev)
    dim, N = int(tree.shape[0]), int(tree.shape[1])
    q = q.reshape(-1, dim)
    B = int(q.shape[0])
    ts = as_tensor(np.array([int(tree_size)], dtype=np.int32), torch.int32, dev)
    idx = torch.empty((B,), dtype=torch.int32, device=dev)
    dist = torch.empty((B,), dtype=torch.float32, device=dev)
    ws = workspace(lib.prrtc_b200_nearest_neighbor_workspace_size(B), dev)
    _lib.check(lib.prrtc_b200_nearest_neighbor(ptr(tree), dim, N, ptr(ts), ptr(q), B, ptr(idx), ptr(dist),
                                               ws.data_ptr(), ws.numel(), stream_handle()),
               "prrtc_b200_nearest_neighbor")
    return dist, idx


def prrtc_extend(tree_configs, nearest_indices, samples, step_size):
    """Step-limited extend (prrtc.py:1472-1508).  Returns (new_configs, parent_indices, valid_flags)."""
    lib = _lib.load()
    dev = cuda_device(tree_configs.device if isinstance(tree_configs, torch.Tensor) else None)
    tree = as_tensor(tree_configs, torch.float32, dev)
    dim, N = int(tree.shape[0]), int(tree.shape[1])
    ni = as_tensor(nearest_indices, torch.int32, dev).reshape(-1)
    s = as_tensor(samples, torch.float32, dev).reshape(-1, dim)
    B = int(s.shape[0])
    st = as_tensor(np.array([step_size], dtype=np.float32), torch.float32, dev)
    out = torch.empty((B, dim), dtype=torch.float32, device=dev)
    par = torch.empty((B,), dtype=torch.int32, device=dev)
    valid = torch.empty((B,), dtype=torch.int32, device=dev)
    _lib.check(lib.prrtc_b200_extend(ptr(tree), dim, N, ptr(ni), ptr(s), B, ptr(st), ptr(out), ptr(par),
                                     ptr(valid), stream_handle()), "prrtc_b200_extend")
    return out, par, valid


def prrtc_iteration(tree_a_configs: torch.Tensor, tree_b_configs: torch.Tensor, tree_a_parents: torch.Tensor,
                    tree_b_parents: torch.Tensor, samples, tree_sizes: torch.Tensor, completed: torch.Tensor,
                    step_size):
    """Legacy single iteration (the "prrtc_iteration" target, prrtc_iteration.cu:180-277).

    Updates the four tree tensors, ``tree_sizes`` and ``completed`` in place (CUDA
    int32/float32 tensors, as the reference's kernel writes its input buffers)
    and returns (new_configs as int32 float bits [batch, dim], new_parents,
    valid_flags, solved_flag)."""
    lib = _lib.load()
    for name, t, dt in (("tree_a_configs", tree_a_configs, torch.float32), ("tree_b_configs", tree_b_configs,
                        torch.float32), ("tree_a_parents", tree_a_parents, torch.int32),
                        ("tree_b_parents", tree_b_parents, torch.int32), ("tree_sizes", tree_sizes, torch.int32),
                        ("completed", completed, torch.int32)):
        if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != dt or not t.is_contiguous():
            raise ValueError(f"{name} must be a contiguous CUDA {dt} tensor (updated in place)")
    dev = tree_a_configs.device
    dim, N = int(tree_a_configs.shape[0]), int(tree_a_configs.shape[1])
    s = as_tensor(samples, torch.float32, dev).reshape(-1, dim)
    B = int(s.shape[0])
    st = as_tensor(np.array([step_size], dtype=np.float32).reshape(-1)[:1], torch.float32, dev)
    new_cfg = torch.empty((B, dim), dtype=torch.int32, device=dev)
    par = torch.empty((B,), dtype=torch.int32, device=dev)
    valid = torch.empty((B,), dtype=torch.int32, device=dev)
    solved = torch.empty((1,), dtype=torch.int32, device=dev)
    _lib.check(lib.prrtc_b200_iteration(ptr(tree_a_configs), ptr(tree_b_configs), ptr(tree_a_parents),
                                        ptr(tree_b_parents), dim, N, ptr(s), B, ptr(tree_sizes), ptr(completed),
                                        ptr(st), ptr(new_cfg), ptr(par), ptr(valid), ptr(solved), stream_handle()),
               "prrtc_b200_iteration")
    return new_cfg, par, valid, solved
