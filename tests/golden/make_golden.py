"""Generate golden vectors from the REFERENCE's own device code (run on a GPU box).

Uses oracle/_ref/libprrtc_ref.so, built by oracle/ref/build_ref.py from the
reference's sources (Halton sampler, prime shuffle, tree-side balance, planner
NN / extend / waypoint / connect arithmetic, dynamic-domain radius updates).  Inputs are regenerated from seeds by
tests/test_golden.py, so only seeds and the reference's outputs are stored.

Usage: python tests/golden/make_golden.py OUT.npz
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]
REF = ROOT / "oracle" / "_ref" / "libprrtc_ref.so"

HALTON_EXPLORERS = [0, 1, 2, 3, 7, 31, 63, 64, 127, 128, 255]
HALTON_N = 64
STEP_TRIALS = 48
CONNECT_TRIALS = 48
BALANCE_TRIALS = 32
RADIUS_TRIALS = 16
CONTENTION_TRIALS = 8
FLT_MAX = float(np.finfo(np.float32).max)


def halton_bounds(dim):
    """Sampling bounds of the Halton vectors (float32, made on the host so the
    generator and the test use the same bits)."""
    return np.full(dim, -2.8, np.float32), np.linspace(1.0, 3.0, dim).astype(np.float32)


def step_inputs(k):
    rng = np.random.default_rng(1000 + k)
    dim = 7 if k % 3 else 14
    N = 1024
    n = int(rng.integers(1, N))
    tree = np.full((dim, N), np.nan, np.float32)
    tree[:, :n] = rng.uniform(-2.8, 2.8, (dim, n)).astype(np.float32)
    sample = rng.uniform(-2.8, 2.8, dim).astype(np.float32)
    step = [0.1, 0.5, 3.0, 20.0][k % 4]
    block = [16, 32, 64][k % 3]
    return dim, N, n, tree, sample, step, block


def connect_inputs(k):
    rng = np.random.default_rng(2000 + k)
    dim = 7 if k % 2 else 14
    N = 256
    tree = rng.uniform(-2.8, 2.8, (dim, N)).astype(np.float32)
    cand = rng.uniform(-2.8, 2.8, dim).astype(np.float32)
    step = [0.1, 0.5, 1.0, 0.05][k % 4]
    return dim, N, tree, cand, step


def balance_inputs(k):
    """Tree-side cases for one (mode, explorer count, tree_ratio): sizes [n,2],
    iteration counts [n], mode-2 sides [n, nblocks]."""
    rng = np.random.default_rng(3000 + k)
    mode = k % 4
    nblocks = [1, 2, 3, 7, 16, 32, 128, 129][(k // 4) % 8]
    ratio = float(np.float32([0.5, 0.3, 0.9, 0.0, 1.0, 0.45][k % 6]))
    n = 96
    sizes = rng.integers(1, 4000, (n, 2)).astype(np.int32)
    sizes[:8] = rng.integers(0, 3, (8, 2))                         # empty and tiny trees
    sizes[8:16, 1] = sizes[8:16, 0]                                # equal sizes
    edge = int(1.5 * nblocks)
    sizes[16:32, 1] = sizes[16:32, 0] + edge + rng.integers(-2, 3, 16)  # around the 1.5 nblocks switch
    sizes[32:40, 0] = sizes[32:40, 1] + edge + rng.integers(-2, 3, 8)
    sizes = np.maximum(sizes, 0).astype(np.int32)
    local_iter = rng.integers(2, 5000, n).astype(np.int32)
    local_iter[rng.random(n) < 0.15] = 1
    vamp = rng.integers(0, 2, (n, nblocks)).astype(np.int32)
    return mode, nblocks, ratio, sizes, local_iter, vamp


def radius_inputs(k):
    """Dynamic-domain update sequence on 8 nodes, applied in order."""
    rng = np.random.default_rng(4000 + k)
    alpha = float(np.float32([1e-4, 0.01, 0.3, 0.05][k % 4]))
    r0 = float(np.float32([4.0, 1.5][k % 2]))
    rmin = float(np.float32([1.0, 0.1, 2.0][k % 3]))
    radii = rng.uniform(0.05, 8.0, 8).astype(np.float32)
    radii[rng.random(8) < 0.4] = FLT_MAX
    radii[0] = FLT_MAX
    radii[1] = np.float32(rmin)
    if k % 4 == 3:
        radii[2] = np.inf
    idx = rng.integers(0, 8, 256).astype(np.int32)
    op = (rng.random(256) < [0.8, 0.5, 0.2, 0.5][k % 4]).astype(np.int32)  # 1 = grow
    return alpha, r0, rmin, radii, idx, op


def contention_inputs(k):
    """Many concurrent updates of 4 nodes, one kind per node (the final radii
    then do not depend on the order the CAS loops serialise in)."""
    rng = np.random.default_rng(5000 + k)
    alpha, r0, rmin = float(np.float32(0.01)), 4.0, float(np.float32(0.5))
    radii = np.array([FLT_MAX, 3.0, FLT_MAX, 1.25], np.float32)
    kinds = np.array([0, 0, 1, 1], np.int32) if k % 2 == 0 else np.array([1, 0, 0, 1], np.int32)
    idx = rng.integers(0, 4, 1024).astype(np.int32)
    return alpha, r0, rmin, radii, idx, kinds[idx]


def main(out):
    lib = C.CDLL(str(REF))
    P, I, F = C.c_void_p, C.c_int, C.c_float
    lib.ref_halton_samples.argtypes = [I, I, I, P, P, P, P]
    lib.ref_prime_order.argtypes = [I, P, P]
    lib.ref_step.argtypes = [P, I, I, I, P, P, I, F, I, P, P, P, P, P, P]
    lib.ref_connect.argtypes = [P, I, I, P, F, I, F, P, P, P]
    lib.ref_balance.argtypes = [P, P, P, I, I, I, F, P, P, P]
    lib.ref_radius.argtypes = [P, P, P, I, F, F, F, I, P]
    dev = torch.device("cuda", 0)
    s = torch.cuda.current_stream().cuda_stream
    res = {}
    po = torch.empty(16, dtype=torch.int32, device=dev)
    orders = []
    for e in range(256):
        assert lib.ref_prime_order(e, po.data_ptr(), s) == 0
        orders.append(po.cpu().numpy().copy())
    res["prime_orders"] = np.stack(orders)
    for dim in (7, 14):
        lo_h, hi_h = halton_bounds(dim)
        res[f"halton_lo_dim{dim}"], res[f"halton_hi_dim{dim}"] = lo_h, hi_h
        lo, hi = torch.from_numpy(lo_h).to(dev), torch.from_numpy(hi_h).to(dev)
        outs = []
        for e in HALTON_EXPLORERS:
            o = torch.empty((HALTON_N, dim), device=dev)
            assert lib.ref_halton_samples(e, HALTON_N, dim, lo.data_ptr(), hi.data_ptr(), o.data_ptr(), s) == 0
            outs.append(o.cpu().numpy())
        res[f"halton_dim{dim}"] = np.stack(outs)
    # planner step: NN + extend + waypoints
    for k in range(STEP_TRIALS):
        dim, N, n, tree, sample, step, block = step_inputs(k)
        tt, ts = torch.from_numpy(tree).to(dev), torch.from_numpy(sample).to(dev)
        tr = torch.full((N,), np.finfo(np.float32).max, device=dev)
        od, oi, osk = torch.empty(1, device=dev), torch.empty(1, dtype=torch.int32, device=dev), torch.empty(
            1, dtype=torch.int32, device=dev)
        oc, ow = torch.empty(dim, device=dev), torch.empty((block, dim), device=dev)
        assert lib.ref_step(tt.data_ptr(), N, dim, n, ts.data_ptr(), tr.data_ptr(), 1, step, block, od.data_ptr(),
                            oi.data_ptr(), osk.data_ptr(), oc.data_ptr(), ow.data_ptr(), s) == 0
        res[f"step{k}_dsq"] = od.cpu().numpy()
        res[f"step{k}_idx"] = oi.cpu().numpy()
        res[f"step{k}_cand"] = oc.cpu().numpy()
        res[f"step{k}_wp"] = ow.cpu().numpy()
    for k in range(CONNECT_TRIALS):
        dim, N, tree, cand, step = connect_inputs(k)
        # the nearest node comes from the reference step harness itself
        tt, tc = torch.from_numpy(tree).to(dev), torch.from_numpy(cand).to(dev)
        tr = torch.full((N,), np.finfo(np.float32).max, device=dev)
        od, oi, osk = torch.empty(1, device=dev), torch.empty(1, dtype=torch.int32, device=dev), torch.empty(
            1, dtype=torch.int32, device=dev)
        oc, ow = torch.empty(dim, device=dev), torch.empty((32, dim), device=dev)
        assert lib.ref_step(tt.data_ptr(), N, dim, N, tc.data_ptr(), tr.data_ptr(), 0, 1e9, 32, od.data_ptr(),
                            oi.data_ptr(), osk.data_ptr(), oc.data_ptr(), ow.data_ptr(), s) == 0
        cdsq, cidx = float(od.item()), int(oi.item())
        ne, vec = torch.empty(1, dtype=torch.int32, device=dev), torch.empty(dim, device=dev)
        assert lib.ref_connect(tt.data_ptr(), N, dim, tc.data_ptr(), cdsq, cidx, step, ne.data_ptr(), vec.data_ptr(),
                               s) == 0
        res[f"conn{k}_idx"] = np.array([cidx], np.int32)
        res[f"conn{k}_dsq"] = np.array([cdsq], np.float32)
        res[f"conn{k}_next"] = ne.cpu().numpy()
        res[f"conn{k}_vec"] = vec.cpu().numpy()
    for k in range(BALANCE_TRIALS):
        mode, nb, ratio, sizes, li, vamp = balance_inputs(k)
        t_s, t_l, t_v = (torch.from_numpy(x).to(dev) for x in (sizes, li, vamp))
        t_out, v_out = torch.empty_like(t_v), torch.empty_like(t_v)
        assert lib.ref_balance(t_s.data_ptr(), t_l.data_ptr(), t_v.data_ptr(), sizes.shape[0], nb, mode, ratio,
                               t_out.data_ptr(), v_out.data_ptr(), s) == 0
        res[f"bal{k}_tree"] = t_out.cpu().numpy()
        res[f"bal{k}_vamp"] = v_out.cpu().numpy()
    for k in range(RADIUS_TRIALS):
        alpha, r0, rmin, radii, idx, op = radius_inputs(k)
        tr, ti, to = (torch.from_numpy(x).to(dev) for x in (radii, idx, op))
        assert lib.ref_radius(tr.data_ptr(), ti.data_ptr(), to.data_ptr(), idx.shape[0], alpha, r0, rmin, 1, s) == 0
        res[f"rad{k}"] = tr.cpu().numpy()
    for k in range(CONTENTION_TRIALS):
        alpha, r0, rmin, radii, idx, op = contention_inputs(k)
        tr, ti, to = (torch.from_numpy(x).to(dev) for x in (radii, idx, op))
        assert lib.ref_radius(tr.data_ptr(), ti.data_ptr(), to.data_ptr(), idx.shape[0], alpha, r0, rmin, 0, s) == 0
        res[f"radc{k}"] = tr.cpu().numpy()
    np.savez_compressed(out, **res)
    print(out, len(res), "arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else str(ROOT / "tests" / "golden" / "ref_pins.npz"))
