"""GPU parity: the CUDA path (through the C-ABI) against the oracle and against
the reference's own device code compiled from its sources (oracle/_ref)."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import pytest
import torch

from conftest import make_problem

pytestmark = pytest.mark.gpu

REF_LIB = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libprrtc_ref.so"


def _ref():
    if not REF_LIB.exists():
        pytest.skip("reference harness oracle/_ref/libprrtc_ref.so not built (needs the reference sources)")
    lib = C.CDLL(str(REF_LIB))
    P, I, F = C.c_void_p, C.c_int, C.c_float
    lib.ref_halton_samples.argtypes = [I, I, I, P, P, P, P]
    lib.ref_prime_order.argtypes = [I, P, P]
    lib.ref_step.argtypes = [P, I, I, I, P, P, I, F, I, P, P, P, P, P, P]
    lib.ref_connect.argtypes = [P, I, I, P, F, I, F, P, P, P]
    lib.ref_nn.argtypes = [P, I, I, I, P, I, P, P, P]
    lib.ref_extend.argtypes = [P, P, P, F, I, I, I, P, P, P, P]
    return lib


def _bits(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32)).view(np.uint32)


def _s():
    return torch.cuda.current_stream().cuda_stream


@pytest.mark.parametrize("dim", [7, 14])
def test_halton_bit_exact(cuda, orc, dim):
    from prrtc_b200.collision import halton_samples

    lo = np.full(dim, -2.8, np.float32)
    hi = np.full(dim, 2.8, np.float32)
    for e in (0, 1, 5, 63, 127, 255):
        mine = halton_samples(e, 300, lo, hi).cpu().numpy()
        ora = orc.halton_samples(e, 300, lo, hi)
        assert np.array_equal(_bits(mine), _bits(ora)), f"explorer {e}"


def test_reference_sampler_pins_oracle(cuda, orc):
    ref = _ref()
    for dim in (7, 14):
        lo = torch.full((dim,), -2.8, device=cuda)
        hi = torch.linspace(1.0, 3.0, dim, device=cuda)
        for e in (0, 1, 2, 17, 127, 255):
            out = torch.empty((257, dim), device=cuda)
            assert ref.ref_halton_samples(e, 257, dim, lo.data_ptr(), hi.data_ptr(), out.data_ptr(), _s()) == 0
            po = torch.empty(16, dtype=torch.int32, device=cuda)
            assert ref.ref_prime_order(e, po.data_ptr(), _s()) == 0
            ora = orc.halton_samples(e, 257, lo.cpu().numpy(), hi.cpu().numpy())
            assert np.array_equal(po.cpu().numpy(), orc.prime_order(e))
            assert np.array_equal(_bits(out.cpu().numpy()), _bits(ora)), f"explorer {e} dim {dim}"


def _random_tree(rng, dim, N, n):
    t = np.full((dim, N), np.nan, np.float32)
    t[:, :n] = rng.uniform(-2.8, 2.8, (dim, n)).astype(np.float32)
    return t


@pytest.mark.parametrize("block", [16, 64])
def test_reference_step_pins_oracle(cuda, orc, block):
    """NN + extend + waypoints of the reference planner (842-904) vs the oracle."""
    ref = _ref()
    rng = np.random.default_rng(3)
    dim, N = 7, 4096
    for trial in range(20):
        n = int(rng.integers(1, N))
        tree = _random_tree(rng, dim, N, n)
        sample = rng.uniform(-2.8, 2.8, dim).astype(np.float32)
        radii = np.full(N, np.finfo(np.float32).max, np.float32)
        tt = torch.from_numpy(tree).to(cuda)
        out_d = torch.empty(1, device=cuda)
        out_i = torch.empty(1, dtype=torch.int32, device=cuda)
        out_s = torch.empty(1, dtype=torch.int32, device=cuda)
        out_c = torch.empty(dim, device=cuda)
        out_w = torch.empty((block, dim), device=cuda)
        step = 0.5 if trial % 2 else 10.0
        ts, tr = torch.from_numpy(sample).to(cuda), torch.from_numpy(radii).to(cuda)
        rc = ref.ref_step(tt.data_ptr(), N, dim, n, ts.data_ptr(), tr.data_ptr(), 1, step, block, out_d.data_ptr(),
                          out_i.data_ptr(), out_s.data_ptr(), out_c.data_ptr(), out_w.data_ptr(), _s())
        assert rc == 0
        idx, dsq = orc.nearest(tree, n, sample)
        assert int(out_i.item()) == idx
        assert _bits(out_d.cpu().numpy())[0] == _bits([dsq])[0]
        assert out_s.item() == 0
        cand = orc.extend(tree[:, idx], sample, float(np.sqrt(np.float32(dsq))), step)
        assert np.array_equal(_bits(out_c.cpu().numpy()), _bits(cand))
        wps = orc.edge_waypoints(tree[:, idx], cand, block)
        assert np.array_equal(_bits(out_w.cpu().numpy()), _bits(wps))


def test_reference_connect_pins_oracle(cuda, orc):
    ref = _ref()
    rng = np.random.default_rng(5)
    dim, N = 7, 256
    for _ in range(50):
        tree = _random_tree(rng, dim, N, N)
        cand = rng.uniform(-2.8, 2.8, dim).astype(np.float32)
        cidx, cdsq = orc.nearest(tree, N, cand)
        step = float(rng.choice([0.1, 0.5, 1.0]))
        n_ext = torch.empty(1, dtype=torch.int32, device=cuda)
        vec = torch.empty(dim, device=cuda)
        tt, tc = torch.from_numpy(tree).to(cuda), torch.from_numpy(cand).to(cuda)
        assert ref.ref_connect(tt.data_ptr(), N, dim, tc.data_ptr(), cdsq, cidx, step,
                               n_ext.data_ptr(), vec.data_ptr(), _s()) == 0
        cd = np.sqrt(np.float32(cdsq), dtype=np.float32)
        ne = int(np.ceil(np.float32(cd) / np.float32(step))) if cd > 1e-8 else 0
        assert n_ext.item() == ne
        want = ((tree[:, cidx] - cand) / np.float32(ne)).astype(np.float32) if ne else np.zeros(dim, np.float32)
        assert np.array_equal(_bits(vec.cpu().numpy()), _bits(want))


@pytest.mark.parametrize("batch", [1, 5, 13, 64])
def test_nearest_neighbor_matches_oracle_and_reference(cuda, orc, batch):
    """batch >= 4 with a tree row length divisible by 4 takes the query-tiled
    kernel (8 queries per tile, ragged last tile); the rest the per-query one."""
    from prrtc_b200 import prrtc_nearest_neighbor

    rng = np.random.default_rng(7 + batch)
    for dim, N, n in ((7, 65536, 50000), (14, 8192, 8192), (3, 4099, 4000), (16, 4096, 4093)):
        tree = _random_tree(rng, dim, N, n)
        q = rng.uniform(-2.8, 2.8, (batch, dim)).astype(np.float32)
        tt, tq = torch.from_numpy(tree).to(cuda), torch.from_numpy(q).to(cuda)
        dist, idx = prrtc_nearest_neighbor(tt, tq, n)
        oi, od = orc.nearest_batch(tree, n, q)
        assert np.array_equal(idx.cpu().numpy(), oi)
        assert np.array_equal(_bits(dist.cpu().numpy()), _bits(np.sqrt(od.astype(np.float32))))
        if REF_LIB.exists():
            ref = _ref()
            ri = torch.empty(batch, dtype=torch.int32, device=cuda)
            rd = torch.empty(batch, device=cuda)
            assert ref.ref_nn(tt.data_ptr(), dim, N, n, tq.data_ptr(), batch, ri.data_ptr(),
                              rd.data_ptr(), _s()) == 0
            assert np.array_equal(ri.cpu().numpy(), oi)  # random floats: no ties
            assert np.array_equal(_bits(rd.cpu().numpy()), _bits(dist.cpu().numpy()))


def test_nearest_neighbor_ties_lowest_index(cuda, orc):
    from prrtc_b200 import prrtc_nearest_neighbor

    dim, N = 7, 8192
    rng = np.random.default_rng(11)
    base = rng.uniform(-1, 1, (dim, 37)).astype(np.float32)
    tree = np.tile(base, (1, N // 37 + 1))[:, :N].copy()
    cols = [3, 5, 36, 0, 1, 2, 4, 6, 7, 8, 30]  # 11 queries: the query-tiled kernel
    for sel in (cols[:3], cols):
        q = base[:, sel].T.copy()
        dist, idx = prrtc_nearest_neighbor(torch.from_numpy(tree).to(cuda), torch.from_numpy(q).to(cuda), N)
        assert idx.cpu().tolist() == sel
        assert np.all(dist.cpu().numpy() == 0.0)
        oi, _ = orc.nearest_batch(tree, N, q)
        assert oi.tolist() == sel


def test_extend_matches_reference(cuda, orc):
    from prrtc_b200 import prrtc_extend

    rng = np.random.default_rng(13)
    dim, N = 7, 1024
    tree = _random_tree(rng, dim, N, N)
    ni = rng.integers(0, N, 100).astype(np.int32)
    s = rng.uniform(-2.8, 2.8, (100, dim)).astype(np.float32)
    tt, tn, tsm = torch.from_numpy(tree).to(cuda), torch.from_numpy(ni).to(cuda), torch.from_numpy(s).to(cuda)
    out, par, valid = prrtc_extend(tt, tn, tsm, 0.5)
    assert np.array_equal(par.cpu().numpy(), ni) and np.all(valid.cpu().numpy() == 1)
    if REF_LIB.exists():
        ref = _ref()
        ro = torch.empty((100, dim), device=cuda)
        rp = torch.empty(100, dtype=torch.int32, device=cuda)
        rv = torch.empty(100, dtype=torch.int32, device=cuda)
        assert ref.ref_extend(tt.data_ptr(), tn.data_ptr(), tsm.data_ptr(), 0.5, dim, N, 100, ro.data_ptr(), rp.data_ptr(),
                              rv.data_ptr(), _s()) == 0
        assert np.array_equal(_bits(ro.cpu().numpy()), _bits(out.cpu().numpy()))


def _rot_angle(Ra, Rb):
    """Rotation angle between two rotation matrices, well conditioned near 0:
    |Ra - Rb|_F = 2 sqrt(2) sin(theta / 2)."""
    s = np.linalg.norm(Ra - Rb) / (2.0 * np.sqrt(2.0))
    return float(2.0 * np.arcsin(min(1.0, s)))


@pytest.mark.parametrize("robot", ["arm", "dual"])
def test_fk_within_1e5_of_f64(cuda, orc, robot, arm, dual):
    from prrtc_b200.collision import forward_kinematics
    from prrtc_b200.context import build_collision_context

    rob = arm if robot == "arm" else dual
    ctx = build_collision_context(rob, None)
    rng = np.random.default_rng(17)
    q = rng.uniform(rob.lower, rob.upper, (500, rob.dim)).astype(np.float32)
    F = forward_kinematics(q, ctx).cpu().numpy()
    sc = orc.Scene(ctx, rob.dim)
    worst_t = worst_r = 0.0
    for i in range(q.shape[0]):
        ref = sc.fk(q[i].astype(np.float64))
        for k in range(ref.shape[0]):
            worst_t = max(worst_t, float(np.abs(F[i, k, 9:] - ref[k, 9:]).max()))
            worst_r = max(worst_r, _rot_angle(F[i, k, :9].reshape(3, 3).astype(np.float64), ref[k, :9].reshape(3, 3)))
    assert worst_t < 1e-5, worst_t
    assert worst_r < 1e-5, worst_r


WORLDS = ["spheres16", "tabletop", "uneven", "large"]


@pytest.mark.parametrize("kind", WORLDS)
@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_collision_verdicts_match_oracle(cuda, orc, kind, mode):
    from prrtc_b200.collision import CollisionChecker

    pr = make_problem(kind, 1)
    ctx = pr.context
    rng = np.random.default_rng(19)
    q = rng.uniform(pr.lower, pr.upper, (3000, pr.dim)).astype(np.float32)
    names = ["binary", "differentiable", "binary_coarse", "binary_coarse_coop"]
    chk = CollisionChecker(ctx, pr.dim, names[mode], 0.02)
    mine = chk.check(q).cpu().numpy()
    sweep = chk.check(q, full_sweep=True).cpu().numpy()
    assert np.array_equal(mine, sweep)
    sc = orc.Scene(ctx, pr.dim)
    ora = sc.check_configs(q, mode, 0.02)
    md = sc.min_distances(q)
    thr = 0.02 if mode == 1 else 0.0
    far = np.abs(md - thr) > 1e-4
    assert far.mean() > 0.95
    assert np.array_equal(mine[far], ora[far]), f"{(mine[far] != ora[far]).sum()} verdicts differ"
    assert 0.02 < mine.mean() < 0.999


def _check_tree_sound(sc, tree, parents, size, dim, sample=200):
    n = min(size, tree.shape[1])
    idx = np.linspace(0, n - 1, min(n, sample)).astype(int)
    nodes = tree[:, idx].T
    assert not np.isnan(nodes).any()
    d = sc.min_distances(nodes)
    assert (d > -2e-3).all(), d.min()
    assert (parents[:n] >= 0).all() and (parents[:n] < n).all()


@pytest.mark.parametrize("kind,seed,checker", [("spheres16", 0, "binary"), ("spheres16", 1, "binary_coarse_coop"),
                                               ("tabletop", 2, "binary_coarse"), ("tabletop", 3, "differentiable"),
                                               ("uneven", 4, "binary_coarse_coop")])
def test_plan_solves_and_revalidates(cuda, orc, kind, seed, checker):
    from prrtc_b200 import prrtc_plan

    pr = make_problem(kind, seed)
    r = prrtc_plan(pr.start, pr.goals, max_iterations=5000, num_new_samples=64, max_nodes=65536,
                   min_vals=pr.lower, max_vals=pr.upper, collision_context=pr.context, collision_checker=checker,
                   edge_resolution=0.01)
    assert r.solved
    path = r.path.cpu().numpy()
    assert np.array_equal(path[0], pr.start)
    assert any(np.array_equal(path[-1], g) for g in pr.goals)
    sc = orc.Scene(pr.context, pr.dim)
    ok, md = sc.validate_planned_path(path)
    assert ok, md
    assert abs(r.cost - float(np.linalg.norm(np.diff(path, axis=0), axis=1).sum())) < 1e-3
    assert r.kernel_time_ms > 0.0
    _check_tree_sound(sc, r.tree_a_configs.cpu().numpy(), r.tree_a_parents.cpu().numpy(), r.tree_a_size, pr.dim)
    _check_tree_sound(sc, r.tree_b_configs.cpu().numpy(), r.tree_b_parents.cpu().numpy(), r.tree_b_size, pr.dim)


@pytest.mark.parametrize("launch,threads,ctas", [("persistent", 128, 0), ("persistent", 32, 0),
                                                 ("persistent", 128, 2), ("persistent", 32, 2),
                                                 ("persistent", 256, 2), ("persistent", 64, 0),
                                                 ("per_problem", 128, 0), ("per_problem", 32, 0),
                                                 ("per_problem", 256, 0)])
def test_batch_uneven_solves(cuda, orc, launch, threads, ctas):
    """threads=32 runs one-warp explorer CTAs; ctas=2 caps the persistent grid
    at two CTAs per SM with the smaller shared-memory carve-out."""
    from prrtc_b200 import prrtc_plan_batch

    probs = [make_problem("uneven", 100 + i) for i in range(12)]
    G = max(p.goals.shape[0] for p in probs)
    dim = probs[0].dim
    goals = np.zeros((len(probs), G, dim), np.float32)
    for i, p in enumerate(probs):
        goals[i, : p.goals.shape[0]] = p.goals
    res = prrtc_plan_batch(np.stack([p.start for p in probs]), goals, max_iterations=5000, num_new_samples=32,
                           max_nodes=16384, min_vals=probs[0].lower, max_vals=probs[0].upper,
                           collision_context=[p.context for p in probs], collision_checker="binary_coarse_coop",
                           goal_counts=[p.goals.shape[0] for p in probs], edge_resolution=0.01, launch=launch,
                           threads_per_explorer=threads, ctas_per_sm=ctas)
    assert len(res) == len(probs)
    assert sum(r.solved for r in res) >= len(probs) - 1
    for i, (p, r) in enumerate(zip(probs, res)):
        if not r.solved:
            continue
        path = r.path.cpu().numpy()
        assert np.array_equal(path[0], p.start)
        assert any(np.array_equal(path[-1], g) for g in p.goals)
        sc = orc.Scene(p.context, dim)
        ok, md = sc.validate_planned_path(path)
        assert ok, md
        if i < 3:
            _check_tree_sound(sc, r.tree_a_configs.cpu().numpy(), r.tree_a_parents.cpu().numpy(), r.tree_a_size, dim)
            _check_tree_sound(sc, r.tree_b_configs.cpu().numpy(), r.tree_b_parents.cpu().numpy(), r.tree_b_size, dim)


@pytest.mark.parametrize("threads,ctas", [(128, 0), (256, 2)])
def test_batch_dual_arm_large_world(cuda, orc, threads, ctas):
    """Dual-arm workload: 14 joints (18 with 4 mimic gripper joints), 120
    spheres, 256 spheres + 64 boxes + floor, 131072-node trees, 1-4 goals."""
    from prrtc_b200 import prrtc_plan_batch

    probs = [make_problem("large", 300 + i) for i in range(6)]
    G = max(p.goals.shape[0] for p in probs)
    dim = probs[0].dim
    assert dim == 14
    goals = np.zeros((len(probs), G, dim), np.float32)
    for i, p in enumerate(probs):
        goals[i, : p.goals.shape[0]] = p.goals
    res = prrtc_plan_batch(np.stack([p.start for p in probs]), goals, max_iterations=10000, num_new_samples=64,
                           max_nodes=131072, min_vals=probs[0].lower, max_vals=probs[0].upper,
                           collision_context=[p.context for p in probs], collision_checker="binary_coarse_coop",
                           goal_counts=[p.goals.shape[0] for p in probs], edge_resolution=0.01,
                           threads_per_explorer=threads, ctas_per_sm=ctas)
    assert sum(r.solved for r in res) >= len(probs) - 1
    for p, r in zip(probs, res):
        if not r.solved:
            continue
        path = r.path.cpu().numpy()
        assert np.array_equal(path[0], p.start)
        assert any(np.array_equal(path[-1], g) for g in p.goals)
        ok, md = orc.Scene(p.context, dim).validate_planned_path(path)
        assert ok, md


@pytest.mark.parametrize("N,batch", [(1024, 64), (4, 10)])
def test_legacy_iteration_matches_oracle(cuda, orc, N, batch):
    """prrtc_iteration: reset to one node per tree, then every sample extends
    tree (sample & 1) from its root into slot 1 + sample // 2 (bit-exact
    candidates; slots past max_nodes are invalid and not counted)."""
    from prrtc_b200 import prrtc_iteration

    rng = np.random.default_rng(N + batch)
    dim = 7
    ta = np.full((dim, N), np.nan, np.float32)
    tb = np.full((dim, N), np.nan, np.float32)
    ta[:, 0] = rng.uniform(-1, 1, dim)
    tb[:, 0] = rng.uniform(-1, 1, dim)
    samples = rng.uniform(-2.8, 2.8, (batch, dim)).astype(np.float32)
    step = 0.5
    tta, ttb = torch.from_numpy(ta).to(cuda), torch.from_numpy(tb).to(cuda)
    pa = torch.full((N,), -1, dtype=torch.int32, device=cuda)
    pb = torch.full((N,), -1, dtype=torch.int32, device=cuda)
    sizes = torch.tensor([7, 9], dtype=torch.int32, device=cuda)  # reset by the call
    comp = torch.tensor([7, 9], dtype=torch.int32, device=cuda)
    cfg, par, valid, solved = prrtc_iteration(tta, ttb, pa, pb, samples, sizes, comp, step)
    cfg = cfg.cpu().numpy()
    trees = [ta, tb]
    n_t = [(batch + 1) // 2, batch // 2]
    assert sizes.cpu().tolist() == [1 + min(n_t[0], N - 1), 1 + min(n_t[1], N - 1)]
    assert comp.cpu().tolist() == sizes.cpu().tolist() and solved.item() == 0
    out = [tta.cpu().numpy(), ttb.cpu().numpy()]
    outp = [pa.cpu().numpy(), pb.cpu().numpy()]
    for b in range(batch):
        t = b & 1
        idx, dsq = orc.nearest(trees[t], 1, samples[b])
        assert idx == 0
        cand = orc.extend(trees[t][:, 0], samples[b], float(np.sqrt(np.float32(dsq), dtype=np.float32)), step)
        assert np.array_equal(cfg[b], np.ascontiguousarray(cand, np.float32).view(np.int32))
        slot = 1 + b // 2
        assert valid[b].item() == int(slot < N) and par[b].item() == 0
        if slot < N:
            assert np.array_equal(out[t][:, slot].view(np.int32), cfg[b]) and outp[t][slot] == 0


@pytest.mark.parametrize("mode", [0, 3])
def test_absent_spheres_and_downward_halfspace(cuda, orc, mode):
    """A sphere on a link that does not exist and chunk padding (57 spheres) must
    never collide, even with a halfspace whose normal points down (a ceiling):
    the padding must not sit at a finite far-away point."""
    from prrtc_b200.collision import CollisionChecker

    pr = make_problem("tabletop", 6)
    ctx = dict(pr.context)
    ctx["world_halfspaces"] = np.concatenate(
        [ctx["world_halfspaces"], np.array([[0, 0, -1, 0, 0, 2.5]], np.float32)])
    J = ctx["fk_parent_idx"].shape[0]
    ctx["sphere_link_idx"] = np.concatenate([ctx["sphere_link_idx"], np.array([J + 5], np.int32)])
    ctx["sphere_local"] = np.concatenate([ctx["sphere_local"], np.zeros((1, 3), np.float32)])
    ctx["sphere_radius"] = np.concatenate([ctx["sphere_radius"], np.array([0.05], np.float32)])
    rng = np.random.default_rng(23)
    q = rng.uniform(pr.lower, pr.upper, (2000, pr.dim)).astype(np.float32)
    names = ["binary", "differentiable", "binary_coarse", "binary_coarse_coop"]
    mine = CollisionChecker(ctx, pr.dim, names[mode], 0.02).check(q).cpu().numpy()
    sc = orc.Scene(ctx, pr.dim)
    ora = sc.check_configs(q, mode, 0.02)
    far = np.abs(sc.min_distances(q)) > 1e-4
    assert np.array_equal(mine[far], ora[far])
    assert 0.02 < mine.mean() < 0.98


def test_async_batches_on_two_streams(cuda, orc):
    """Two batches of different tree capacity queued on two streams before
    either is read back; both read back solved, re-validating paths."""
    from prrtc_b200 import prrtc_plan_batch_async

    groups = {4096: [make_problem("uneven", 400 + i) for i in range(4)],
              16384: [make_problem("uneven", 410 + i) for i in range(4)]}
    streams = {N: torch.cuda.Stream(device=cuda) for N in groups}
    pending = {}
    for N, probs in groups.items():
        G = max(p.goals.shape[0] for p in probs)
        goals = np.zeros((len(probs), G, probs[0].dim), np.float32)
        for i, p in enumerate(probs):
            goals[i, : p.goals.shape[0]] = p.goals
        with torch.cuda.stream(streams[N]):
            pending[N] = prrtc_plan_batch_async(
                np.stack([p.start for p in probs]), goals, max_iterations=5000, num_new_samples=8, max_nodes=N,
                min_vals=probs[0].lower, max_vals=probs[0].upper, collision_context=[p.context for p in probs],
                collision_checker="binary_coarse_coop", goal_counts=[p.goals.shape[0] for p in probs],
                edge_resolution=0.01, return_trees=False, paths_on_host=True)
    for N, probs in groups.items():
        res = pending[N].results()
        assert sum(r.solved for r in res) >= len(probs) - 1
        for p, r in zip(probs, res):
            if r.solved:
                ok, md = orc.Scene(p.context, p.dim).validate_planned_path(r.path.numpy())
                assert ok, md


def test_async_batches_pipelined_on_one_stream(cuda, orc):
    """Three calls queued on one stream before the first is read back (the
    bench's end-to-end form): every call's results, read in order, match its own
    problems, and every packed path re-validates."""
    from prrtc_b200 import prrtc_plan_batch_async

    batches = [[make_problem("uneven", 420 + 10 * k + i) for i in range(5)] for k in range(3)]
    st = torch.cuda.Stream(device=cuda)
    pending = []
    with torch.cuda.stream(st):
        for probs in batches:
            G = max(p.goals.shape[0] for p in probs)
            goals = np.zeros((len(probs), G, probs[0].dim), np.float32)
            for i, p in enumerate(probs):
                goals[i, : p.goals.shape[0]] = p.goals
            pending.append(prrtc_plan_batch_async(
                np.stack([p.start for p in probs]), goals, max_iterations=5000, num_new_samples=4,
                max_nodes=[p.max_nodes for p in probs], min_vals=probs[0].lower, max_vals=probs[0].upper,
                collision_context=[p.context for p in probs], collision_checker="binary_coarse_coop",
                goal_counts=[p.goals.shape[0] for p in probs], edge_resolution=0.01, return_trees=False,
                paths_on_host=True))
    for probs, pend in zip(batches, pending):
        res = pend.results()
        assert pend.d2h_bytes >= len(probs) * 64
        assert sum(r.solved for r in res) >= len(probs) - 1
        for p, r in zip(probs, res):
            if r.solved:
                path = r.path.numpy()
                assert path.shape[1] == p.dim and r.path.device.type == "cpu"
                assert np.array_equal(path[0], p.start.astype(np.float32))
                assert any(np.array_equal(path[-1], g.astype(np.float32)) for g in p.goals)
                ok, md = orc.Scene(p.context, p.dim).validate_planned_path(path)
                assert ok, md
                assert abs(r.cost - np.linalg.norm(np.diff(path, axis=0), axis=1).sum()) < 1e-3 * max(1.0, r.cost)


def test_explore_events_time_the_planner_kernel(cuda):
    """tuning.explore_events: the library records the pair right around the
    planner kernel, eagerly and as external event nodes of a captured graph, so
    the span is positive and shorter than the whole planner call."""
    from prrtc_b200.batch import BatchPlanner, PlanSettings

    probs = [make_problem("uneven", 600 + i) for i in range(6)]
    pl = BatchPlanner(probs, [p.max_nodes for p in probs], PlanSettings(num_new_samples=2), cuda)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    ev1.record()
    pl.tun.explore_events[0], pl.tun.explore_events[1] = ev0.cuda_event, ev1.cuda_event
    for graph in (False, True):
        if graph:
            pl.capture()
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record()
        pl.run()
        c1.record()
        c1.synchronize()
        k_ms, call_ms = ev0.elapsed_time(ev1), c0.elapsed_time(c1)
        assert 0.0 < k_ms <= call_ms, (graph, k_ms, call_ms)
        assert (pl.summary_block()[:, 8] == 1).sum().item() >= len(probs) - 1
    pl.graph = None


def test_result_block_and_packed_paths(cuda):
    """prrtc_b200_result_block through the C-ABI against a numpy restatement:
    1500 problems (two chunks of the one-CTA scan), unsolved, failed, empty and
    too-long (-1) paths, and a packed capacity that the last paths overflow."""
    from prrtc_b200 import _lib

    lib = _lib.load()
    rng = np.random.default_rng(5)
    B, dim, L = 1500, 7, 40
    solved = rng.choice([1, 1, 1, 0, -1], B).astype(np.int32)
    lengths = rng.integers(1, L + 1, B).astype(np.int32)
    lengths[rng.random(B) < 0.05] = -1
    lengths[solved != 1] = 0
    sizes = rng.integers(1, 1 << 20, (B, 2)).astype(np.int32)
    completed = rng.integers(0, 2, (B, 2)).astype(np.int32)
    iters = rng.integers(0, 10000, B).astype(np.int32)
    conn = rng.integers(-1, 1000, (B, 3)).astype(np.int32)
    kms = rng.random(B).astype(np.float32)
    costs = rng.random(B).astype(np.float32)
    paths = rng.standard_normal((B, L, dim)).astype(np.float32)
    live = (solved == 1) & (lengths > 0)
    cap = int(lengths[live].sum()) - 500  # the last few paths do not fit
    t = {k: torch.from_numpy(v).to(cuda) for k, v in dict(sizes=sizes, completed=completed, iters=iters, conn=conn,
                                                          solved=solved, kms=kms, lengths=lengths, costs=costs,
                                                          paths=paths).items()}
    block = torch.full((B, 16), 77, dtype=torch.int32, device=cuda)
    packed = torch.full((cap, dim), np.nan, dtype=torch.float32, device=cuda)
    rc = lib.prrtc_b200_result_block(B, dim, L, *(t[k].data_ptr() for k in ("sizes", "completed", "iters", "conn",
                                                                         "solved", "kms", "lengths", "costs",
                                                                         "paths")),
                                     block.data_ptr(), packed.data_ptr(), cap, torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    got = block.cpu().numpy()
    off = np.concatenate([[0], np.cumsum(np.where(live, lengths, 0))[:-1]])
    want_off = np.where(live & (off + np.where(live, lengths, 0) <= cap), off, -1)
    want = np.zeros((B, 16), np.int32)
    want[:, 0:2], want[:, 2:4], want[:, 4], want[:, 5:8] = sizes, completed, iters, conn
    want[:, 8], want[:, 9], want[:, 10], want[:, 11], want[:, 12] = solved, kms.view(np.int32), lengths, \
        costs.view(np.int32), want_off
    assert np.array_equal(got, want)
    assert (want_off == -1).sum() > (~live).sum()  # some live paths overflowed
    pk = packed.cpu().numpy()
    for b in np.flatnonzero(want_off >= 0):
        assert np.array_equal(pk[want_off[b]:want_off[b] + lengths[b]], paths[b, :lengths[b]])
    used = int((want_off + lengths)[want_off >= 0].max())
    assert np.isnan(pk[used:]).all()  # nothing written past the last packed path


def test_staging_wait_that_runs_out_reports_minus_two(cuda):
    """Failure path of the bounded scene-staging wait, without a fault: with no
    polls allowed every CTA's wait gives up at once (its copy still lands
    before the CTA leaves), the open problems come back as solved_flag -2 and
    the Python layer raises; the same planner then runs normally."""
    from prrtc_b200._lib import PrrtcError
    from prrtc_b200.batch import BatchPlanner, PlanSettings

    probs = [make_problem("uneven", 500 + i) for i in range(3)]
    pl = BatchPlanner(probs, 16384, PlanSettings(num_new_samples=2), cuda)
    pl.tun.staging_wait_polls = -1
    pl.launch()
    blk = pl.summary_block().cpu().numpy()
    assert (blk[:, 8] == -2).all()
    with pytest.raises(PrrtcError):
        pl.results()
    pl.tun.staging_wait_polls = 0
    pl.launch()
    res = pl.results()
    assert sum(r.solved for r in res) >= len(probs) - 1


@pytest.mark.parametrize("batch", [1, 3])
def test_nearest_neighbor_large_tree(cuda, orc, batch):
    """1-3 queries over a 117 MB tree (larger than L2): a ragged tree size, NaN
    slots and a duplicated node (ties go to the lowest index) match the oracle."""
    from prrtc_b200 import prrtc_nearest_neighbor

    rng = np.random.default_rng(31 + batch)
    dim, N, n = 7, 1 << 22, (1 << 22) - 12345
    tree = np.full((dim, N), np.nan, np.float32)
    tree[:, :n] = rng.uniform(-2.8, 2.8, (dim, n)).astype(np.float32)
    q = rng.uniform(-2.8, 2.8, (batch, dim)).astype(np.float32)
    tree[:, n - 7] = q[0]          # an exact hit near the end ...
    tree[:, 1000] = q[0]           # ... and the same node earlier: index 1000 wins
    dist, idx = prrtc_nearest_neighbor(torch.from_numpy(tree).to(cuda), torch.from_numpy(q).to(cuda), n)
    oi, od = orc.nearest_batch(tree, n, q)
    assert idx.cpu().numpy().tolist() == oi.tolist()
    assert idx[0].item() == 1000 and dist[0].item() == 0.0
    assert np.array_equal(dist.cpu().numpy().view(np.uint32), np.sqrt(od.astype(np.float32)).view(np.uint32))


def test_batch_per_problem_capacity(cuda, orc):
    """Problems of different tree capacity in one launch: each tree stays within
    its own capacity; a capacity too small to solve overflows (solved_flag -1)
    without affecting the others."""
    from prrtc_b200 import prrtc_plan_batch

    probs = [make_problem("uneven", 600 + i) for i in range(6)]
    caps = [4096, 16384, 65536, 4096, 16384, 2]  # 2: any extend + connect overflows
    G = max(p.goals.shape[0] for p in probs)
    dim = probs[0].dim
    goals = np.zeros((len(probs), G, dim), np.float32)
    for i, p in enumerate(probs):
        goals[i, : p.goals.shape[0]] = p.goals
    res = prrtc_plan_batch(np.stack([p.start for p in probs]), goals, max_iterations=5000, num_new_samples=4,
                           max_nodes=caps, min_vals=probs[0].lower, max_vals=probs[0].upper,
                           collision_context=[p.context for p in probs], collision_checker="binary_coarse_coop",
                           goal_counts=[p.goals.shape[0] for p in probs], edge_resolution=0.01)
    for p, r, cap in zip(probs, res, caps):
        assert r.tree_a_configs.shape[1] <= cap and r.tree_b_configs.shape[1] <= cap
        if r.solved:
            ok, md = orc.Scene(p.context, dim).validate_planned_path(r.path.cpu().numpy())
            assert ok, md
    assert sum(r.solved for r in res[:5]) >= 4
    assert not res[5].solved and max(res[5].tree_a_size, res[5].tree_b_size) >= 2


@pytest.mark.parametrize("launch", ["persistent", "per_problem"])
def test_batch_mixed_full_and_trimmed_contexts(cuda, orc, launch):
    """The reference's batch scenario (test_prrtc.py:408-491): four problems
    whose contexts alternate between the full scene and one with the last
    world sphere and the last self pair removed, one goal each, step 0.6, 16
    samples, dynamic domain off.  Every solved path, and a sample of each
    solved problem's start tree, re-validates against that problem's own
    context (full or trimmed)."""
    from prrtc_b200 import prrtc_plan_batch

    base = make_problem("spheres16", 11)
    full = base.context
    trimmed = dict(full)
    trimmed["world_spheres"] = np.ascontiguousarray(full["world_spheres"][:-1])
    trimmed["self_pairs"] = np.ascontiguousarray(full["self_pairs"][:-1])
    ctxs = [full if i % 2 == 0 else trimmed for i in range(4)]
    rng = np.random.default_rng(11)
    starts, goals = [], []
    for i in range(4):
        sc = orc.Scene(ctxs[i], base.dim)
        pair = []
        while len(pair) < 2:
            q = rng.uniform(base.lower, base.upper).astype(np.float32)
            if not sc.in_collision(q) and sc.min_distance(q) > 1e-3:
                pair.append(q)
        starts.append(pair[0])
        goals.append(pair[1])
    res = prrtc_plan_batch(np.stack(starts), np.stack(goals)[:, None, :], max_iterations=1000, step_size=0.6,
                           num_new_samples=16, dynamic_domain=False, max_nodes=65536, min_vals=base.lower,
                           max_vals=base.upper, collision_context=ctxs, launch=launch)
    assert len(res) == 4
    assert sum(r.solved for r in res) >= 3
    for i, r in enumerate(res):
        if not r.solved:
            continue
        path = r.path.cpu().numpy()
        assert np.array_equal(path[0], starts[i]) and np.array_equal(path[-1], goals[i])
        ok, md = orc.Scene(ctxs[i], base.dim).validate_planned_path(path)
        assert ok, (i, md)
        _check_tree_sound(orc.Scene(ctxs[i], base.dim), r.tree_a_configs.cpu().numpy(),
                          r.tree_a_parents.cpu().numpy(), r.tree_a_size, base.dim)


def test_batch_inputs_as_device_tensors_and_tensor_contexts(cuda, orc):
    """The batch call with its configurations and limits already on the
    device (no copy) and per-problem contexts holding CPU torch tensors (no
    buffer protocol, so the Python packer runs instead of the native one)
    solves and re-validates like the same call with numpy inputs, which goes
    through the native packer."""
    from prrtc_b200 import prrtc_plan_batch

    probs = [make_problem("uneven", 500 + i) for i in range(6)]
    dim = probs[0].dim
    G = max(p.goals.shape[0] for p in probs)
    goals = np.zeros((len(probs), G, dim), np.float32)
    for i, p in enumerate(probs):
        goals[i, : p.goals.shape[0]] = p.goals
    starts = np.stack([p.start for p in probs])
    kw = dict(max_iterations=5000, num_new_samples=8, max_nodes=16384, collision_checker="binary_coarse_coop",
              goal_counts=[p.goals.shape[0] for p in probs], edge_resolution=0.01, return_trees=False)
    ref = prrtc_plan_batch(starts, goals, min_vals=probs[0].lower, max_vals=probs[0].upper,
                           collision_context=[p.context for p in probs], **kw)
    tctx = [{k: (torch.from_numpy(np.asarray(v)) if isinstance(v, np.ndarray) else v) for k, v in p.context.items()}
            for p in probs]
    res = prrtc_plan_batch(torch.from_numpy(starts).to(cuda), torch.from_numpy(goals).to(cuda),
                           min_vals=torch.from_numpy(np.asarray(probs[0].lower, np.float32)).to(cuda),
                           max_vals=torch.from_numpy(np.asarray(probs[0].upper, np.float32)).to(cuda),
                           collision_context=tctx, **kw)
    assert len(res) == len(ref) == len(probs)
    assert sum(r.solved for r in res) >= len(probs) - 1
    for p, r in zip(probs, res):
        if r.solved:
            ok, md = orc.Scene(p.context, dim).validate_planned_path(r.path.cpu().numpy())
            assert ok, md


@pytest.mark.parametrize("balance_mode,tree_ratio", [(0, 0.5), (2, 0.3), (3, 0.5)])
def test_plan_balance_modes(cuda, orc, balance_mode, tree_ratio):
    """Every tree-side rule of prrtc_planner.cu:790-824 (0: half the explorers
    per tree, 1: size ratio -- the default, tested throughout --, 2: the
    VAMP-style toggle, other: the smaller tree) plans and re-validates, in the
    single-plan and the batched launch."""
    from prrtc_b200 import prrtc_plan, prrtc_plan_batch

    pr = make_problem("tabletop", 21)
    sc = orc.Scene(pr.context, pr.dim)
    r = prrtc_plan(pr.start, pr.goals, max_iterations=4000, num_new_samples=32, max_nodes=65536,
                   balance_mode=balance_mode, tree_ratio=tree_ratio, min_vals=pr.lower, max_vals=pr.upper,
                   collision_context=pr.context, collision_checker="binary_coarse_coop", edge_resolution=0.01)
    assert r.solved
    ok, md = sc.validate_planned_path(r.path.cpu().numpy())
    assert ok, md
    probs = [make_problem("uneven", 600 + i) for i in range(4)]
    G = max(p.goals.shape[0] for p in probs)
    goals = np.zeros((len(probs), G, pr.dim), np.float32)
    for i, p in enumerate(probs):
        goals[i, : p.goals.shape[0]] = p.goals
    res = prrtc_plan_batch(np.stack([p.start for p in probs]), goals, max_iterations=4000, num_new_samples=4,
                           max_nodes=16384, balance_mode=balance_mode, tree_ratio=tree_ratio,
                           min_vals=probs[0].lower, max_vals=probs[0].upper,
                           collision_context=[p.context for p in probs], collision_checker="binary_coarse_coop",
                           goal_counts=[p.goals.shape[0] for p in probs], edge_resolution=0.01, return_trees=False)
    assert sum(x.solved for x in res) >= len(probs) - 1
    for p, x in zip(probs, res):
        if x.solved:
            ok, md = orc.Scene(p.context, pr.dim).validate_planned_path(x.path.cpu().numpy())
            assert ok, md


@pytest.mark.parametrize("launch", ["single", "persistent", "per_problem"])
def test_unsolvable_problem_ends_at_max_iterations(cuda, orc, launch):
    """A start configuration in collision makes the problem unsolvable (every
    connect toward the start tree ends on a colliding waypoint).  Each
    explorer then stops once its iteration count passes max_iterations
    (prrtc_planner.cu:770-780): not solved, no path, and the reported
    iteration count is max_iterations + 1, as in the oracle."""
    from prrtc_b200 import prrtc_plan, prrtc_plan_batch

    pr = make_problem("spheres16", 31)
    sc = orc.Scene(pr.context, pr.dim)
    rng = np.random.default_rng(31)
    while True:
        bad = rng.uniform(pr.lower, pr.upper).astype(np.float32)
        if sc.in_collision(bad) and sc.min_distance(bad) < -0.02:
            break
    max_it = 150
    ora = orc.plan(sc, bad, pr.goals[:1], pr.lower, pr.upper, max_iterations=max_it, num_new_samples=8,
                   max_nodes=65536)
    assert ora.solved != 1
    kw = dict(max_iterations=max_it, num_new_samples=8, max_nodes=65536, min_vals=pr.lower, max_vals=pr.upper)
    if launch == "single":
        r = prrtc_plan(bad, pr.goals[:1], collision_context=pr.context, **kw)
    else:
        r = prrtc_plan_batch(bad[None], pr.goals[:1][None], collision_context=[pr.context], launch=launch,
                             tail_explorers=False, **kw)[0]
    assert not r.solved and r.path is None
    assert r.iterations == ora.iter_count == max_it + 1


def _long_chain_robot():
    """A 12-dof arm in which every revolute joint is followed by two fixed
    joints (identity transforms): 36 joints, past the 32 that the in-register
    FK covers, so the checker takes its joint-parallel / chain-serial path."""
    from prrtc_b200 import scenes
    from prrtc_b200.context import RobotModel

    base = scenes.arm(0, 12)
    J0 = base.n_joints if hasattr(base, "n_joints") else base.twists.shape[0]
    twists, ptf, parent, act = [], [], [], []
    ident = np.array([1, 0, 0, 0, 0, 0, 0], np.float32)
    for j in range(J0):
        for k in range(3):
            twists.append(base.twists[j] if k == 0 else np.zeros(6, np.float32))
            ptf.append(base.parent_tf[j] if k == 0 else ident)
            parent.append(len(parent) - 1)
            act.append(int(base.act_idx[j]) if k == 0 else -1)
    J = len(parent)
    frame_map = {j: 3 * j + 2 for j in range(J0)}
    return RobotModel(
        twists=np.stack(twists).astype(np.float32), parent_tf=np.stack(ptf).astype(np.float32),
        parent_idx=np.asarray(parent, np.int32), act_idx=np.asarray(act, np.int32),
        mimic_mul=np.ones(J, np.float32), mimic_off=np.zeros(J, np.float32),
        mimic_act_idx=np.full(J, -1, np.int32), topo_inv=np.arange(J, dtype=np.int32),
        lower=base.lower, upper=base.upper,
        sphere_frame=np.asarray([frame_map[int(f)] for f in base.sphere_frame], np.int32),
        sphere_local=base.sphere_local, sphere_radius=base.sphere_radius,
        link_pairs=[(frame_map[i], frame_map[j]) for i, j in base.link_pairs])


def test_more_than_32_joints(cuda, orc):
    """Robots past 32 joints: FK within 1e-5 of float64, checker verdicts equal
    to the oracle's away from contact (flat and coarse checkers), and a plan
    that re-validates."""
    from prrtc_b200 import prrtc_plan, scenes
    from prrtc_b200.collision import CollisionChecker, forward_kinematics

    rob = _long_chain_robot()
    assert rob.twists.shape[0] == 36

    def checker(cfg, ctx):
        return orc.Scene(ctx, cfg.shape[1]).check_configs(cfg, 0)

    pr = scenes.make_problem("spheres16", 41, checker, robot=rob)
    sc = orc.Scene(pr.context, pr.dim)
    rng = np.random.default_rng(41)
    q = rng.uniform(pr.lower, pr.upper, (300, pr.dim)).astype(np.float32)
    F = forward_kinematics(q[:50], pr.context).cpu().numpy()
    for i in range(50):
        ref = sc.fk(q[i].astype(np.float64))
        assert np.abs(F[i, :, 9:] - ref[:, 9:]).max() < 1e-5
    far = np.abs(sc.min_distances(q)) > 1e-4
    for mode, name in ((0, "binary"), (2, "binary_coarse"), (3, "binary_coarse_coop")):
        v = CollisionChecker(pr.context, pr.dim, name, 0.02, cuda).check(q).cpu().numpy()
        assert np.array_equal(v[far], sc.check_configs(q, mode)[far]), name
    r = prrtc_plan(pr.start, pr.goals, max_iterations=5000, num_new_samples=32, max_nodes=65536,
                   min_vals=pr.lower, max_vals=pr.upper, collision_context=pr.context,
                   collision_checker="binary_coarse_coop", edge_resolution=0.02)
    assert r.solved
    ok, md = sc.validate_planned_path(r.path.cpu().numpy(), resolution=0.02)
    assert ok, md


# ----------------------------------------------------------------------------- tree balance, dynamic domain

def _golden_gen():
    import sys as _sys

    _sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
    import make_golden

    return make_golden


def test_choose_tree_matches_reference_and_oracle(cuda, orc):
    """Tree-side balance, all four modes (prrtc_planner.cu:790-824): the
    planner's device rule == the reference's own lines == the oracle, bit for
    bit, for explorer counts 1-129, sizes around every switch of the rule, first
    iterations and both mode-2 sides."""
    from prrtc_b200 import _lib

    lib, ref, g = _lib.load(), _ref(), _golden_gen()
    ref.ref_balance.argtypes = [C.c_void_p] * 3 + [C.c_int] * 3 + [C.c_float] + [C.c_void_p] * 3
    for k in range(g.BALANCE_TRIALS):
        mode, nb, ratio, sizes, li, vamp = g.balance_inputs(k)
        t_s, t_l, t_v = (torch.from_numpy(x).to(cuda) for x in (sizes, li, vamp))
        mine_t, mine_v = torch.empty_like(t_v), torch.empty_like(t_v)
        ref_t, ref_v = torch.empty_like(t_v), torch.empty_like(t_v)
        _lib.check(lib.prrtc_b200_choose_tree(mode, sizes.shape[0], t_s.data_ptr(), t_l.data_ptr(), t_v.data_ptr(), nb,
                                              ratio, mine_t.data_ptr(), mine_v.data_ptr(), _s()),
                   "prrtc_b200_choose_tree")
        assert ref.ref_balance(t_s.data_ptr(), t_l.data_ptr(), t_v.data_ptr(), sizes.shape[0], nb, mode, ratio,
                               ref_t.data_ptr(), ref_v.data_ptr(), _s()) == 0
        ora_t, ora_v = orc.choose_tree(mode, sizes, li, vamp, nb, ratio)
        assert np.array_equal(ref_t.cpu().numpy(), ora_t), f"reference vs oracle, case {k}"
        assert np.array_equal(ref_v.cpu().numpy(), ora_v), f"reference vs oracle mode-2 side, case {k}"
        assert np.array_equal(mine_t.cpu().numpy(), ora_t), f"planner rule vs oracle, case {k}"
        assert np.array_equal(mine_v.cpu().numpy(), ora_v), f"planner rule vs oracle mode-2 side, case {k}"


def test_radius_updates_match_reference_and_oracle(cuda, orc):
    """Dynamic-domain shrink / grow (prrtc_planner.cu:46-83): update sequences
    applied in order, and 1024 concurrent updates contending on four nodes (one
    kind per node, so the result does not depend on the CAS order): the
    planner's device loops == the reference's own loops == the oracle, bit for
    bit, from unset (FLT_MAX), clamped (rmin) and infinite radii."""
    from prrtc_b200 import _lib

    lib, ref, g = _lib.load(), _ref(), _golden_gen()
    ref.ref_radius.argtypes = [C.c_void_p] * 3 + [C.c_int, C.c_float, C.c_float, C.c_float, C.c_int, C.c_void_p]
    err = torch.zeros(1, dtype=torch.int32, device=cuda)
    cases = [(g.radius_inputs(k), 1) for k in range(g.RADIUS_TRIALS)] + \
            [(g.contention_inputs(k), 0) for k in range(g.CONTENTION_TRIALS)]
    for (alpha, r0, rmin, radii, idx, op), seq in cases:
        t_i, t_o = torch.from_numpy(idx).to(cuda), torch.from_numpy(op).to(cuda)
        mine, theirs = torch.from_numpy(radii).to(cuda), torch.from_numpy(radii).to(cuda)
        _lib.check(lib.prrtc_b200_radius_update(mine.data_ptr(), t_i.data_ptr(), t_o.data_ptr(), idx.shape[0], alpha,
                                                r0, rmin, seq, err.data_ptr(), _s()), "prrtc_b200_radius_update")
        assert ref.ref_radius(theirs.data_ptr(), t_i.data_ptr(), t_o.data_ptr(), idx.shape[0], alpha, r0, rmin, seq,
                              _s()) == 0
        want = orc.radius_updates(radii, idx, op, alpha, r0, rmin)
        assert np.array_equal(_bits(theirs.cpu().numpy()), _bits(want)), ("reference vs oracle", seq)
        assert np.array_equal(_bits(mine.cpu().numpy()), _bits(want)), ("planner loops vs oracle", seq)
    assert int(err.item()) == 0
