"""CPU pinning of the oracle against golden vectors produced by the reference's
own device code (tests/golden/ref_pins.npz, made by tests/golden/make_golden.py
from the reference-fragment harness on a B200).  Bit-exact."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import sys

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
from make_golden import (CONNECT_TRIALS, HALTON_EXPLORERS, HALTON_N, STEP_TRIALS,  # noqa: E402
                         connect_inputs, step_inputs)

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_pins.npz"


@pytest.fixture(scope="module")
def gold():
    if not GOLDEN.exists():
        pytest.skip("golden vectors not generated")
    return np.load(GOLDEN)


def bits(a):
    return np.ascontiguousarray(np.asarray(a, np.float32)).view(np.uint32)


def test_prime_orders(orc, gold):
    for e in range(256):
        assert np.array_equal(orc.prime_order(e), gold["prime_orders"][e])


@pytest.mark.parametrize("dim", [7, 14])
def test_halton_samples(orc, gold, dim):
    lo, hi = gold[f"halton_lo_dim{dim}"], gold[f"halton_hi_dim{dim}"]
    for i, e in enumerate(HALTON_EXPLORERS):
        assert np.array_equal(bits(orc.halton_samples(e, HALTON_N, lo, hi)), bits(gold[f"halton_dim{dim}"][i])), e


def test_planner_step_nn_extend_waypoints(orc, gold):
    for k in range(STEP_TRIALS):
        dim, N, n, tree, sample, step, block = step_inputs(k)
        idx, dsq = orc.nearest(tree, n, sample)
        assert idx == int(gold[f"step{k}_idx"][0]), k
        assert bits([dsq])[0] == bits(gold[f"step{k}_dsq"])[0], k
        cand = orc.extend(tree[:, idx], sample, float(np.sqrt(np.float32(dsq))), step)
        assert np.array_equal(bits(cand), bits(gold[f"step{k}_cand"])), k
        wp = orc.edge_waypoints(tree[:, idx], cand, block)
        assert np.array_equal(bits(wp), bits(gold[f"step{k}_wp"])), k


def test_connect_vectors(orc, gold):
    for k in range(CONNECT_TRIALS):
        dim, N, tree, cand, step = connect_inputs(k)
        idx, dsq = orc.nearest(tree, N, cand)
        assert idx == int(gold[f"conn{k}_idx"][0]) and bits([dsq])[0] == bits(gold[f"conn{k}_dsq"])[0]
        cd = np.sqrt(np.float32(dsq), dtype=np.float32)
        ne = int(np.ceil(np.float32(cd) / np.float32(step))) if cd > 1e-8 else 0
        assert ne == int(gold[f"conn{k}_next"][0])
        vec = ((tree[:, idx] - cand) / np.float32(ne)).astype(np.float32) if ne else np.zeros(dim, np.float32)
        assert np.array_equal(bits(vec), bits(gold[f"conn{k}_vec"]))


def _need(gold, key):
    if key not in gold.files:
        pytest.fail(f"{GOLDEN.name} lacks {key}: regenerate it with tests/golden/make_golden.py on a GPU")


def test_tree_balance(orc, gold):
    """Tree-side balance, all four modes, against the reference's own lines
    (prrtc_planner.cu:790-824) run on a B200."""
    from make_golden import BALANCE_TRIALS, balance_inputs

    _need(gold, "bal0_tree")
    for k in range(BALANCE_TRIALS):
        mode, nb, ratio, sizes, li, vamp = balance_inputs(k)
        tree, v = orc.choose_tree(mode, sizes, li, vamp, nb, ratio)
        assert np.array_equal(tree, gold[f"bal{k}_tree"]), k
        assert np.array_equal(v, gold[f"bal{k}_vamp"]), k


def test_dynamic_domain_radii(orc, gold):
    """Shrink / grow sequences and contended updates against the reference's
    own CAS loops (prrtc_planner.cu:46-83) run on a B200."""
    from make_golden import CONTENTION_TRIALS, RADIUS_TRIALS, contention_inputs, radius_inputs

    _need(gold, "rad0")
    for k in range(RADIUS_TRIALS):
        alpha, r0, rmin, radii, idx, op = radius_inputs(k)
        assert np.array_equal(bits(orc.radius_updates(radii, idx, op, alpha, r0, rmin)), bits(gold[f"rad{k}"])), k
    for k in range(CONTENTION_TRIALS):
        alpha, r0, rmin, radii, idx, op = contention_inputs(k)
        assert np.array_equal(bits(orc.radius_updates(radii, idx, op, alpha, r0, rmin)), bits(gold[f"radc{k}"])), k
