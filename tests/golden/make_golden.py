"""Generate golden vectors from the REFERENCE's own device code (run on a GPU box).

Uses oracle/_ref/libprrtc_ref.so, built by oracle/ref/build_ref.py from the
reference's sources (Halton sampler, prime shuffle, planner NN / extend /
waypoint / connect arithmetic).  Inputs are regenerated from seeds by
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


def main(out):
    lib = C.CDLL(str(REF))
    P, I, F = C.c_void_p, C.c_int, C.c_float
    lib.ref_halton_samples.argtypes = [I, I, I, P, P, P, P]
    lib.ref_prime_order.argtypes = [I, P, P]
    lib.ref_step.argtypes = [P, I, I, I, P, P, I, F, I, P, P, P, P, P, P]
    lib.ref_connect.argtypes = [P, I, I, P, F, I, F, P, P, P]
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
    np.savez_compressed(out, **res)
    print(out, len(res), "arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else str(ROOT / "tests" / "golden" / "ref_pins.npz"))
