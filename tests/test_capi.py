"""C-ABI surface: the library loads, exports every function include/prrtc_b200.h
declares, and rejects malformed arguments before any CUDA call (no GPU needed)."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared():
    text = (ROOT / "include" / "prrtc_b200.h").read_text()
    return sorted(set(re.findall(r"\b(prrtc_b200_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared()
    for must in ("prrtc_b200_plan", "prrtc_b200_plan_batch", "prrtc_b200_nearest_neighbor", "prrtc_b200_extend",
                 "prrtc_b200_check_configs", "prrtc_b200_extract_paths", "prrtc_b200_smooth_cost_grad"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from prrtc_b200 import _lib

    lib = _lib.load()
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.EXPORTS) <= set(declared())


def test_invalid_arguments_rejected_without_gpu():
    from prrtc_b200 import _lib

    lib = _lib.load()
    a = _lib.Attrs()
    a.dim, a.max_nodes, a.step_size, a.num_new_samples, a.granularity = 7, 1024, 0.5, 8, 16
    inp, out = _lib.Inputs(), _lib.Outputs()
    # null outputs / inputs
    assert lib.prrtc_b200_plan(C.byref(inp), C.byref(out), C.byref(a), None, None, 0, None) == _lib.EARG
    bad = _lib.Attrs.from_buffer_copy(a)
    bad.granularity = 12
    assert lib.prrtc_b200_plan(C.byref(inp), C.byref(out), C.byref(bad), None, None, 0, None) == _lib.EARG
    bad = _lib.Attrs.from_buffer_copy(a)
    bad.step_size = 0.0
    assert lib.prrtc_b200_plan(C.byref(inp), C.byref(out), C.byref(bad), None, None, 0, None) == _lib.EARG
    bad = _lib.Attrs.from_buffer_copy(a)
    bad.dim = 17
    assert lib.prrtc_b200_plan(C.byref(inp), C.byref(out), C.byref(bad), None, None, 0, None) == _lib.EUNSUPPORTED
    assert lib.prrtc_b200_nearest_neighbor(None, 7, 10, None, None, 4, None, None, None, 0, None) == _lib.EARG
    assert lib.prrtc_b200_error_string(_lib.EWORKSPACE).decode().startswith("workspace")


def test_workspace_sizes_are_host_arithmetic():
    from prrtc_b200 import _lib

    lib = _lib.load()
    a = _lib.Attrs()
    a.dim, a.max_nodes = 7, 65536
    inp = _lib.Inputs()
    inp.robot.n_joints, inp.robot.n_spheres = 7, 56
    inp.world.n_world_spheres, inp.world.n_self_pairs = 16, 960
    n1 = lib.prrtc_b200_plan_workspace_size(C.byref(inp), C.byref(a), None)
    a.max_nodes = 4096
    n2 = lib.prrtc_b200_plan_workspace_size(C.byref(inp), C.byref(a), None)
    # radii for two trees dominate: 2 * max_nodes floats
    assert n1 - n2 == 2 * (65536 - 4096) * 4
    assert lib.prrtc_b200_nearest_neighbor_workspace_size(100) >= 800


def test_api_validation_matches_reference_errors():
    import numpy as np

    import prrtc_b200 as P

    start, goal = np.zeros(7, np.float32), np.ones((1, 7), np.float32)
    with pytest.raises(ValueError, match="step_size"):
        P.prrtc_plan(start, goal, step_size=0.0, allow_unsafe_no_collision=True)
    with pytest.raises(ValueError, match="power of 2"):
        P.prrtc_plan(start, goal, granularity=12, allow_unsafe_no_collision=True)
    with pytest.raises(ValueError, match="<= 64"):
        P.prrtc_plan(start, goal, granularity=128, allow_unsafe_no_collision=True)
    with pytest.raises(ValueError, match="robogpu"):
        P.prrtc_plan(start, goal, collision_checker="robogpu")
    with pytest.raises(ValueError, match="collision_checker must be one of"):
        P.prrtc_plan(start, goal, collision_checker="sdf")
    with pytest.raises(ValueError, match="Collision-aware planning is the default"):
        P.prrtc_plan(start, goal)
    with pytest.raises(ValueError, match="missing required keys"):
        P.prrtc_plan(start, goal, collision_context={"fk_twists": np.zeros((1, 6))})
    with pytest.raises(ValueError, match="single start configuration"):
        P.prrtc_plan(np.zeros((2, 7)), goal, allow_unsafe_no_collision=True)


def test_batch_table_sharing_host_logic():
    """prrtc_plan_batch sends a table once, unbatched, when every problem holds
    the same one (empty tables included) and pads it per problem otherwise."""
    from prrtc_b200.prrtc import _pack_worlds, _shared_table

    sp = np.array([[0, 5], [1, 6]], np.int32)
    ctxs = [{"self_pairs": sp.copy(), "world_spheres": np.zeros((0, 4), np.float32),
             "world_boxes": np.full((i + 1, 15), i, np.float32)} for i in range(3)]
    assert np.array_equal(_shared_table(ctxs, "self_pairs"), sp)
    assert _shared_table(ctxs, "world_spheres").shape == (0, 4)
    assert _shared_table(ctxs, "world_boxes") is None
    assert _shared_table(ctxs, "world_capsules") is None  # absent key
    ctxs[2]["self_pairs"] = sp[:1]
    assert _shared_table(ctxs, "self_pairs") is None
    packed, counts = _pack_worlds(ctxs, 3, skip={"world_spheres"})
    assert "world_spheres" not in packed
    assert packed["world_boxes"].shape == (3, 3, 15) and counts["world_boxes"].tolist() == [1, 2, 3]
    assert counts["self_pairs"].tolist() == [2, 2, 1]


def _native_layout(info, specs, B):
    """Byte layout of the native packer's output for `info` (scan result)."""
    layout, off = [], 0
    for (key, feat, kind), (shared, width, cbytes) in zip(specs, info):
        if shared:
            rows = int(np.frombuffer(cbytes, np.int32)[0])
            layout.append((True, rows, off, -1))
            off += rows * feat * 4
        else:
            layout.append((False, width, off, off + B * width * feat * 4))
            off += B * width * feat * 4 + B * 4
    return layout, off


def test_native_host_packer_matches_python():
    """The native packer (scan + fill into a staging buffer) writes exactly the
    counted rows, the counts and the shared tables of the Python packer (rows
    past a problem's count are not read by the planner and not written)."""
    from prrtc_b200 import _lib
    from prrtc_b200.prrtc import _PACK_SPECS, _pack_worlds, _shared_table

    hp = _lib.hostpack()
    rng = np.random.default_rng(3)
    sp = rng.integers(0, 50, (40, 2)).astype(np.int32)
    half = np.array([[0, 0, 1, 0, 0, 0]], np.float32)
    ctxs = []
    for i in range(37):
        c = {"self_pairs": sp if i % 2 else sp.copy(), "world_halfspaces": half.copy(),
             "world_spheres": rng.normal(size=(int(rng.integers(0, 9)), 4)).astype(np.float32),
             "world_boxes": rng.normal(size=(int(rng.integers(0, 4)), 15)).astype(np.float32)}
        if i % 5 == 0:
            c["world_capsules"] = rng.normal(size=(int(rng.integers(1, 3)), 7)).astype(np.float32)
        if i == 7:
            c["world_boxes"] = None
        ctxs.append(c)
    ctxs[11] = None
    B = len(ctxs)
    for trial in range(2):
        if trial == 1:  # every context present: self pairs and the halfspace become shared
            ctxs[11] = dict(ctxs[10])
        info = hp.scan(ctxs, _PACK_SPECS)
        layout, total = _native_layout(info, _PACK_SPECS, B)
        buf = np.full(total + 64, 0x7F, np.uint8)
        hp.fill(ctxs, _PACK_SPECS, layout, buf)
        shared = {k: _shared_table(ctxs, k) for k, _, _ in _PACK_SPECS}
        packed, counts = _pack_worlds(ctxs, B, skip={k for k in shared if shared[k] is not None})
        for (key, feat, kind), (is_sh, width, cbytes), (_, w2, off, coff) in zip(_PACK_SPECS, info, layout):
            dt = np.int32 if kind == "i" else np.float32
            assert is_sh == (shared[key] is not None), key
            if is_sh:
                got = buf[off:off + shared[key].nbytes].view(dt).reshape(shared[key].shape)
                assert np.array_equal(got, shared[key])
            else:
                ref = packed[key]
                assert width == ref.shape[1]
                got = buf[off:off + ref.nbytes].view(dt).reshape(ref.shape)
                for i in range(B):
                    n = int(counts[key][i])
                    assert np.array_equal(got[i, :n], ref[i, :n]), (key, i)
                assert np.array_equal(buf[coff:coff + 4 * B].view(np.int32), counts[key])
                assert np.array_equal(np.frombuffer(cbytes, np.int32), counts[key])
        assert (buf[total:] == 0x7F).all()  # nothing written past the layout
    assert shared["self_pairs"] is not None and shared["world_halfspaces"] is not None


def test_native_host_packer_declines_other_types():
    """Tables that are not C-contiguous float32 / int32 arrays raise TypeError
    (the batch call then packs in Python); a short staging buffer is refused."""
    from prrtc_b200 import _lib
    from prrtc_b200.prrtc import _PACK_SPECS

    hp = _lib.hostpack()
    good = {"world_spheres": np.zeros((2, 4), np.float32)}
    for bad in (np.zeros((2, 4), np.float64), [[0.0] * 4] * 2, np.zeros((4, 2), np.float32).T,
                np.zeros((2, 5), np.float32), np.zeros(8, np.float32)):
        with pytest.raises(TypeError):
            hp.scan([good, {"world_spheres": bad}], _PACK_SPECS)
    with pytest.raises(TypeError):
        hp.scan([good, {"self_pairs": np.zeros((2, 2), np.int64)}], _PACK_SPECS)
    info = hp.scan([good, good], _PACK_SPECS)
    layout, total = _native_layout(info, _PACK_SPECS, 2)
    with pytest.raises(ValueError):
        hp.fill([good, good], _PACK_SPECS, layout, np.zeros(max(total - 1, 0), np.uint8))


def test_native_host_packer_reads_non_numpy_buffers():
    """A table that is not a numpy array but exports a C-contiguous float32
    buffer (a memoryview here) is read through the buffer protocol: same scan
    and same bytes as the numpy array."""
    from prrtc_b200 import _lib
    from prrtc_b200.prrtc import _PACK_SPECS

    hp = _lib.hostpack()
    a = np.arange(12, dtype=np.float32).reshape(3, 4)
    ctxs_np = [{"world_spheres": a}, {"world_spheres": a[:1].copy()}]
    ctxs_mv = [{"world_spheres": memoryview(a)}, {"world_spheres": memoryview(a[:1].copy())}]
    info_np, info_mv = hp.scan(ctxs_np, _PACK_SPECS), hp.scan(ctxs_mv, _PACK_SPECS)
    assert info_np == info_mv
    layout, total = _native_layout(info_np, _PACK_SPECS, 2)
    b1, b2 = np.zeros(total, np.uint8), np.zeros(total, np.uint8)
    hp.fill(ctxs_np, _PACK_SPECS, layout, b1)
    hp.fill(ctxs_mv, _PACK_SPECS, layout, b2)
    assert np.array_equal(b1, b2) and b1.any()


def test_autotuner_second_round_decides(monkeypatch):
    """Host logic of the autotuner: every candidate gets three timed launches,
    the three best by median six more each, and the best median over all of a
    finalist's launches wins -- so a candidate that was lucky in the first
    round loses to a steadily faster one.  Fake planners, no GPU."""
    import torch

    from prrtc_b200 import autotune, batch

    class FakePlanner:
        def __init__(self, problems, N, s, dev):
            self.key = (s.num_new_samples, s.threads_per_explorer, s.waypoint_chunk, s.ctas_per_sm)

        def launch(self):
            pass

    cands = ((1, 128, 32, 0), (2, 128, 32, 0), (4, 128, 32, 0), (2, 256, 32, 2))
    # first three timed launches, then the second-round launches
    script = {
        (1, 128, 32, 0): [100, 100, 100] + [100] * 6,
        (2, 128, 32, 0): [300, 300, 300] + [110] * 6,    # lucky first round, slower after
        (4, 128, 32, 0): [90, 90, 90] + [90] * 6,
        (2, 256, 32, 2): [150, 150, 150] + [200] * 6,    # steadily the fastest
    }
    calls = []

    def fake_rate(pl, flush=None):  # the script runs on per candidate, across planner objects
        r = script[pl.key][calls.count(pl.key)]
        calls.append(pl.key)
        return float(r)

    monkeypatch.setattr(batch, "BatchPlanner", FakePlanner)
    monkeypatch.setattr(autotune, "_rate", fake_rate)
    monkeypatch.setattr(autotune, "_key", lambda *a: "fake")
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    best = autotune.choose([object()], 4096, batch.PlanSettings(), torch.device("cpu"), candidates=cands,
                           use_cache=False)
    assert best == {"num_new_samples": 2, "threads_per_explorer": 256, "waypoint_chunk": 32, "ctas_per_sm": 2}
    assert calls.count((4, 128, 32, 0)) == 3          # not a finalist
    assert calls.count((2, 256, 32, 2)) == 9          # finalist: 3 + 6


def test_native_host_packer_random_contexts():
    """Seeded random batches (ragged tables, absent keys, None contexts, shared
    and equal-content tables): the native packer's counted rows, counts and
    shared tables equal the Python packer's."""
    from prrtc_b200 import _lib
    from prrtc_b200.prrtc import _PACK_SPECS, _pack_worlds, _shared_table

    hp = _lib.hostpack()
    feats = {k: f for k, f, _ in _PACK_SPECS}
    for seed in range(25):
        rng = np.random.default_rng(1000 + seed)
        B = int(rng.integers(1, 40))
        shared = {k: rng.normal(size=(int(rng.integers(0, 5)), f)).astype(np.int32 if k == "self_pairs" else np.float32)
                  for k, f in feats.items()}
        ctxs = []
        for i in range(B):
            if rng.random() < 0.05:
                ctxs.append(None)
                continue
            c = {}
            for k, f in feats.items():
                u = rng.random()
                dt = np.int32 if k == "self_pairs" else np.float32
                if u < 0.15:
                    continue                                     # absent
                if u < 0.45:
                    c[k] = shared[k] if rng.random() < 0.5 else shared[k].copy()   # same object / same content
                else:
                    c[k] = (rng.normal(size=(int(rng.integers(0, 9)), f)) * 10).astype(dt)
            ctxs.append(c)
        info = hp.scan(ctxs, _PACK_SPECS)
        layout, total = _native_layout(info, _PACK_SPECS, B)
        buf = np.full(total + 32, 0x5A, np.uint8)
        hp.fill(ctxs, _PACK_SPECS, layout, buf)
        sh = {k: _shared_table(ctxs, k) for k in feats}
        packed, counts = _pack_worlds(ctxs, B, skip={k for k in sh if sh[k] is not None})
        for (key, feat, kind), (is_sh, width, cbytes), (_, _, off, coff) in zip(_PACK_SPECS, info, layout):
            dt = np.int32 if kind == "i" else np.float32
            assert is_sh == (sh[key] is not None), (seed, key)
            if is_sh:
                assert np.array_equal(buf[off:off + sh[key].nbytes].view(dt).reshape(sh[key].shape), sh[key])
            else:
                ref = packed[key]
                got = buf[off:off + ref.nbytes].view(dt).reshape(ref.shape)
                n = counts[key]
                assert np.array_equal(buf[coff:coff + 4 * B].view(np.int32), n), (seed, key)
                for i in range(B):
                    assert np.array_equal(got[i, :n[i]], ref[i, :n[i]]), (seed, key, i)
        assert (buf[total:] == 0x5A).all()


def test_lpt_order_from_packed_counts_equals_lpt_order():
    """The batch call orders problems by the row counts the packer already has
    (_lpt_from_counts); that order equals lpt_order over the contexts, shared
    tables (same cost for every problem) left out."""
    from prrtc_b200.prrtc import _PACK_SPECS, _lpt_from_counts, _pack_worlds, _shared_table, lpt_order

    rng = np.random.default_rng(9)
    for trial in range(10):
        B = int(rng.integers(1, 60))
        ctxs = []
        shared_half = np.zeros((1, 6), np.float32)
        for i in range(B):
            c = {"world_spheres": np.zeros((int(rng.integers(0, 5)), 4), np.float32),
                 "world_boxes": np.zeros((int(rng.integers(0, 4)), 15), np.float32),
                 "world_halfspaces": shared_half}
            if rng.random() < 0.3:
                c["world_capsules"] = np.zeros((int(rng.integers(0, 3)), 7), np.float32)
            ctxs.append(c if rng.random() > 0.05 else None)
        keys = [k for k, _, _ in _PACK_SPECS]
        sh = {k: _shared_table(ctxs, k) for k in keys}
        _, counts = _pack_worlds(ctxs, B, skip={k for k in keys if sh[k] is not None})
        assert np.array_equal(_lpt_from_counts(counts, B), lpt_order(ctxs))
