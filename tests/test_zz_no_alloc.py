"""The allocation-free collision check, through the C-ABI.

prrtc_b200_check_configs_noalloc serves callers that cannot allocate device
memory or pass a workspace (work issued during another library's stream
capture, real-time loops that forbid allocation, plug-in hosts without an
allocator).  It must return exactly the verdicts of the workspace entry point,
prrtc_b200_check_configs, and keep doing so across consecutive calls that reuse
its file-scope scene buffer with different scenes.
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


def _entry(lib):
    fn = lib.prrtc_b200_check_configs_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_int32, C.c_float, C.c_int32,
                   C.c_void_p, C.c_void_p]
    return fn


def test_noalloc_matches_workspace_entry_point_on_consecutive_calls(cuda):
    from prrtc_b200 import _lib
    from prrtc_b200.collision import CollisionChecker

    fn = _entry(_lib.load())
    rng = np.random.default_rng(23)
    # two calls in a row with different scenes, then the first scene again
    for kind, seed, mode in (("tabletop", 7, 3), ("uneven", 8, 0), ("tabletop", 7, 1)):
        pr = make_problem(kind, seed)
        chk = CollisionChecker(pr.context, pr.dim, CHECKERS[mode], 0.02, device=cuda)
        q = torch.from_numpy(rng.uniform(pr.lower, pr.upper, (4099, pr.dim)).astype(np.float32)).to(cuda)
        for full in (0, 1):
            want = chk.check(q, full_sweep=bool(full)).cpu().numpy()
            got = torch.full((q.shape[0],), -7, dtype=torch.int32, device=cuda)
            rc = fn(C.byref(chk._robot), C.byref(chk._world), pr.dim, q.data_ptr(), q.shape[0], mode, 0.02, full,
                    got.data_ptr(), torch.cuda.current_stream().cuda_stream)
            assert rc == 0, rc
            torch.cuda.synchronize()
            assert np.array_equal(got.cpu().numpy(), want), f"{kind} mode {mode} full_sweep {full}"


def test_noalloc_rejects_scene_beyond_buffer(cuda):
    from prrtc_b200 import _lib
    from prrtc_b200.collision import CollisionChecker

    fn = _entry(_lib.load())
    pr = make_problem("spheres16", 0)
    ctx = dict(pr.context)
    ctx["world_spheres"] = np.tile(ctx["world_spheres"], (1300, 1))  # 20800 spheres: > 256 KiB packed
    chk = CollisionChecker(ctx, pr.dim, device=cuda)
    q = torch.zeros((4, pr.dim), dtype=torch.float32, device=cuda)
    out = torch.zeros(4, dtype=torch.int32, device=cuda)
    rc = fn(C.byref(chk._robot), C.byref(chk._world), pr.dim, q.data_ptr(), 4, 0, 0.0, 0, out.data_ptr(),
            torch.cuda.current_stream().cuda_stream)
    assert rc == ETOOLARGE
    assert "no-allocation" in _lib.load().prrtc_b200_error_string(rc).decode()
