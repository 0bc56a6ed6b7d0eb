"""The allocation-free collision check, through the C-ABI.

prrtc_b200_check_configs_noalloc serves callers that cannot allocate device
memory or pass a workspace (work issued during another library's stream
capture, real-time loops that forbid allocation, plug-in hosts without an
allocator).  It must return exactly the verdicts of the workspace entry point,
prrtc_b200_check_configs, and of the oracle away from contact, and keep doing
so across consecutive calls that reuse its file-scope scene buffer with
different scenes -- including a scene too large to stage in shared memory
(read from the buffer in global memory) -- and reject a scene beyond the buffer
without touching its outputs.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from conftest import make_problem

pytestmark = pytest.mark.gpu

CHECKERS = ["binary", "differentiable", "binary_coarse", "binary_coarse_coop"]
ETOOLARGE = -5
NOALLOC_SCENE_MAX = 256 * 1024


def _entry(lib):
    fn = lib.prrtc_b200_check_configs_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_int32, C.c_float, C.c_int32,
                   C.c_void_p, C.c_void_p]
    return fn


def _noalloc(fn, chk, dim, q, mode, full):
    got = torch.full((q.shape[0],), -7, dtype=torch.int32, device=q.device)
    rc = fn(C.byref(chk._robot), C.byref(chk._world), dim, q.data_ptr(), q.shape[0], mode, 0.02, full,
            got.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == 0, rc
    torch.cuda.synchronize()
    return got.cpu().numpy()


def _assert_matches_oracle(orc, ctx, dim, q, mode, got):
    sc = orc.Scene(ctx, dim)
    qn = q.cpu().numpy()
    want = sc.check_configs(qn, mode, 0.02)
    thr = 0.02 if mode == 1 else 0.0
    far = np.abs(sc.min_distances(qn) - thr) > 1e-4
    assert far.mean() > 0.95
    assert np.array_equal(got[far], want[far]), f"{(got[far] != want[far]).sum()} verdicts differ from the oracle"


def test_noalloc_matches_workspace_entry_point_and_oracle_on_consecutive_calls(cuda, orc):
    from prrtc_b200 import _lib
    from prrtc_b200.collision import CollisionChecker

    fn = _entry(_lib.load())
    rng = np.random.default_rng(23)
    # consecutive calls with different scenes and every checker, then the first scene again
    for kind, seed, mode in (("tabletop", 7, 3), ("uneven", 8, 0), ("tabletop", 9, 2), ("spheres16", 3, 1),
                             ("tabletop", 7, 3)):
        pr = make_problem(kind, seed)
        chk = CollisionChecker(pr.context, pr.dim, CHECKERS[mode], 0.02, device=cuda)
        q = torch.from_numpy(rng.uniform(pr.lower, pr.upper, (4099, pr.dim)).astype(np.float32)).to(cuda)
        for full in (0, 1):
            want = chk.check(q, full_sweep=bool(full)).cpu().numpy()
            got = _noalloc(fn, chk, pr.dim, q, mode, full)
            assert np.array_equal(got, want), f"{kind} mode {mode} full_sweep {full}"
        _assert_matches_oracle(orc, pr.context, pr.dim, q, mode, got)
        assert 0.02 < got.mean() < 0.999


def test_noalloc_scene_read_from_global_memory(cuda, orc):
    """A scene of about 215 KiB packed fits the 256 KiB buffer but not the
    checker's shared-memory staging, so every CTA reads it from the buffer in
    global memory: same verdicts as the workspace entry point (which takes the
    same path) and the oracle, on two calls in a row."""
    from prrtc_b200 import _lib
    from prrtc_b200.collision import CollisionChecker

    lib = _lib.load()
    fn = _entry(lib)
    pr = make_problem("spheres16", 5)
    rng = np.random.default_rng(31)
    ctx = dict(pr.context)
    n = 6400
    c = rng.uniform((-5.0, -5.0, 0.0), (5.0, 5.0, 4.0), (n, 3))
    c = c[np.hypot(c[:, 0], c[:, 1]) > 0.35]
    ctx["world_spheres"] = np.concatenate([c, rng.uniform(0.005, 0.02, (c.shape[0], 1))], 1).astype(np.float32)
    chk = CollisionChecker(ctx, pr.dim, "binary", 0.02, device=cuda)
    stride = lib.prrtc_b200_check_configs_workspace_size(C.byref(chk._robot), C.byref(chk._world))
    assert 190 * 1024 < stride <= NOALLOC_SCENE_MAX, stride
    q = torch.from_numpy(rng.uniform(pr.lower, pr.upper, (1031, pr.dim)).astype(np.float32)).to(cuda)
    want = chk.check(q).cpu().numpy()
    for _ in range(2):
        got = _noalloc(fn, chk, pr.dim, q, 0, 0)
        assert np.array_equal(got, want)
    _assert_matches_oracle(orc, ctx, pr.dim, q, 0, got)
    assert 0.02 < got.mean() < 0.999


def test_noalloc_rejects_scene_beyond_buffer(cuda):
    from prrtc_b200 import _lib
    from prrtc_b200.collision import CollisionChecker

    fn = _entry(_lib.load())
    pr = make_problem("spheres16", 0)
    ctx = dict(pr.context)
    ctx["world_spheres"] = np.tile(ctx["world_spheres"], (1300, 1))  # 20800 spheres: > 256 KiB packed
    chk = CollisionChecker(ctx, pr.dim, device=cuda)
    q = torch.zeros((4, pr.dim), dtype=torch.float32, device=cuda)
    out = torch.full((4,), 1234, dtype=torch.int32, device=cuda)
    rc = fn(C.byref(chk._robot), C.byref(chk._world), pr.dim, q.data_ptr(), 4, 0, 0.0, 0, out.data_ptr(),
            torch.cuda.current_stream().cuda_stream)
    assert rc == ETOOLARGE
    assert "no-allocation" in _lib.load().prrtc_b200_error_string(rc).decode()
    torch.cuda.synchronize()
    assert (out.cpu().numpy() == 1234).all(), "a rejected call wrote its outputs"
