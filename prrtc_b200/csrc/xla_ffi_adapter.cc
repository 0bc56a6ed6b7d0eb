// xla_ffi_adapter.cc -- XLA FFI handlers exporting the reference's six symbols
// (PrrtcPlannerFfi, PrrtcPlannerBatchFfi, PrrtcPlannerBatchCtxFfi,
// PrrtcNearestNeighborFfi, PrrtcExtendFfi, PrrtcIterationFfi; registered by
// cuda-rrtc/jax/prrtc.py:141-146) on top of the C-ABI in include/prrtc_b200.h.
//
// Compiled only where jaxlib provides xla/ffi/api/ffi.h (prrtc_b200/build.py
// adds -DPRRTC_WITH_XLA_FFI and jaxlib's include directory).  The binding order,
// names and dtypes are the reference's interface contract
// (cuda-rrtc/CUDA/prrtc_planner.cu:1946-2117, prrtc_nearest_neighbor.cu:132-141,
// prrtc_extend.cu:129-140).  Unlike the reference handlers (cudaMalloc / cudaFree
// of their scratch and a blocking event sync per call) these never block the host
// and never call the CUDA allocator: each call's workspace, sized by the
// library's *_workspace_size query, comes from XLA's own scratch allocator
// (ffi::ScratchAllocator, bound as a context argument).  XLA releases that
// memory when the handler returns; its device allocator hands it out again only
// to work ordered after this call on the same compute stream, which is where the
// kernels run.
#if defined(PRRTC_WITH_XLA_FFI)

#include <cuda_runtime.h>

#include <optional>
#include <string>

#include "../../include/prrtc_b200.h"
#include "xla/ffi/api/ffi.h"

namespace ffi = xla::ffi;

namespace {

// 256-byte aligned workspace of `need` bytes from XLA's scratch allocator.
void* scratch_bytes(ffi::ScratchAllocator& scratch, size_t need) {
    std::optional<void*> p = scratch.Allocate(need > 0 ? need : 256, 256);
    return p.has_value() ? *p : nullptr;
}

ffi::Error no_scratch(size_t need) {
    return ffi::Error(ffi::ErrorCode::kResourceExhausted,
                      "prrtc_b200: XLA scratch allocation of " + std::to_string(need) + " bytes failed");
}

template <typename B>
int rows(const B& b) { return b.dimensions().size() == 0 ? 0 : static_cast<int>(b.dimensions()[0]); }

ffi::Error status(int rc) {
    if (rc == PRRTC_B200_OK) return ffi::Error::Success();
    const ffi::ErrorCode code = rc == PRRTC_B200_EARG ? ffi::ErrorCode::kInvalidArgument : ffi::ErrorCode::kInternal;
    return ffi::Error(code, prrtc_b200_error_string(rc));
}

using F32 = ffi::Buffer<ffi::DataType::F32>;
using S32 = ffi::Buffer<ffi::DataType::S32>;
using RF32 = ffi::Result<ffi::Buffer<ffi::DataType::F32>>;
using RS32 = ffi::Result<ffi::Buffer<ffi::DataType::S32>>;

prrtc_robot_t robot_of(F32 tw, F32 ptf, S32 par, S32 act, F32 mm, F32 mo, S32 mact, S32 topo, S32 sli, F32 sloc,
                       F32 srad, S32 cli, F32 cloc, F32 crad, S32 foff, S32 cpairs, S32 cranges) {
    prrtc_robot_t r{};
    r.fk_twists = tw.typed_data(); r.fk_parent_tf = ptf.typed_data(); r.fk_parent_idx = par.typed_data();
    r.fk_act_idx = act.typed_data(); r.fk_mimic_mul = mm.typed_data(); r.fk_mimic_off = mo.typed_data();
    r.fk_mimic_act_idx = mact.typed_data(); r.fk_topo_inv = topo.typed_data(); r.n_joints = rows(par);
    r.sphere_link_idx = sli.typed_data(); r.sphere_local = sloc.typed_data(); r.sphere_radius = srad.typed_data();
    r.n_spheres = rows(sli);
    const int k = rows(cli);
    r.coarse_sphere_link_idx = cli.typed_data(); r.coarse_sphere_local = cloc.typed_data();
    r.coarse_sphere_radius = crad.typed_data();
    r.fine_link_offsets = rows(foff) >= k + 1 ? foff.typed_data() : nullptr;
    r.n_coarse = r.fine_link_offsets ? k : 0;
    r.coarse_self_pairs = cpairs.typed_data(); r.self_pair_ranges = cranges.typed_data();
    r.n_coarse_self_pairs = r.n_coarse ? rows(cpairs) : 0;
    return r;
}

prrtc_attrs_t attrs_of(int max_iterations, float step_size, int num_new_samples, int balance_mode, float tree_ratio,
                       int dynamic_domain, float dd_alpha, float dd_radius, float dd_min_radius, int dim,
                       int max_nodes, int granularity, int collision_mode, float collision_margin) {
    prrtc_attrs_t a{};
    a.max_iterations = max_iterations; a.step_size = step_size; a.num_new_samples = num_new_samples;
    a.balance_mode = balance_mode; a.tree_ratio = tree_ratio; a.dynamic_domain = dynamic_domain;
    a.dd_alpha = dd_alpha; a.dd_radius = dd_radius; a.dd_min_radius = dd_min_radius; a.dim = dim;
    a.max_nodes = max_nodes; a.granularity = granularity; a.collision_mode = collision_mode;
    a.collision_margin = collision_margin;
    return a;
}

ffi::Error PlannerImpl(cudaStream_t stream, ffi::ScratchAllocator scratch, F32 start, F32 goals, F32 lo, F32 hi, F32 tw, F32 ptf, S32 par, S32 act,
                       F32 mm, F32 mo, S32 mact, S32 topo, S32 sli, F32 sloc, F32 srad, F32 ws, F32 wc, F32 wb, F32 wh,
                       S32 sp, S32 cli, F32 cloc, F32 crad, S32 foff, S32 cpairs, S32 cranges, RF32 ta, RF32 tb,
                       RS32 pa, RS32 pb, RS32 sizes, RS32 completed, RS32 iters, RS32 conn, RS32 solved, RF32 ktime,
                       int max_iterations, float step_size, int num_new_samples, int balance_mode, float tree_ratio,
                       int dynamic_domain, float dd_alpha, float dd_radius, float dd_min_radius, int dim,
                       int max_nodes, int granularity, int collision_mode, float collision_margin) {
    prrtc_inputs_t in{};
    in.start_config = start.typed_data();
    in.goal_configs = goals.typed_data();
    in.num_goals = rows(goals);
    in.min_vals = lo.typed_data();
    in.max_vals = hi.typed_data();
    in.robot = robot_of(tw, ptf, par, act, mm, mo, mact, topo, sli, sloc, srad, cli, cloc, crad, foff, cpairs, cranges);
    in.world.world_spheres = ws.typed_data(); in.world.n_world_spheres = rows(ws);
    in.world.world_capsules = wc.typed_data(); in.world.n_world_capsules = rows(wc);
    in.world.world_boxes = wb.typed_data(); in.world.n_world_boxes = rows(wb);
    in.world.world_halfspaces = wh.typed_data(); in.world.n_world_halfspaces = rows(wh);
    in.world.self_pairs = sp.typed_data(); in.world.n_self_pairs = rows(sp);
    prrtc_outputs_t out{ta->typed_data(), tb->typed_data(), pa->typed_data(), pb->typed_data(),
                        sizes->typed_data(), completed->typed_data(), iters->typed_data(), conn->typed_data(),
                        solved->typed_data(), ktime->typed_data()};
    const prrtc_attrs_t a = attrs_of(max_iterations, step_size, num_new_samples, balance_mode, tree_ratio,
                                     dynamic_domain, dd_alpha, dd_radius, dd_min_radius, dim, max_nodes, granularity,
                                     collision_mode, collision_margin);
    const size_t need = prrtc_b200_plan_workspace_size(&in, &a, nullptr);
    void* w = scratch_bytes(scratch, need);
    if (!w) return no_scratch(need);
    return status(prrtc_b200_plan(&in, &out, &a, nullptr, w, need, stream));
}

prrtc_outputs_t outputs_of(RF32 ta, RF32 tb, RS32 pa, RS32 pb, RS32 sizes, RS32 completed, RS32 iters, RS32 conn,
                           RS32 solved, RF32 ktime) {
    return prrtc_outputs_t{ta->typed_data(), tb->typed_data(), pa->typed_data(), pb->typed_data(),
                           sizes->typed_data(), completed->typed_data(), iters->typed_data(), conn->typed_data(),
                           solved->typed_data(), ktime->typed_data()};
}

// Batched planners (prrtc_planner.cu:1404-1944).  ctx: worlds are [B, max_n,
// feat] with per-problem counts ("prrtc_planner_batch_ctx"); otherwise one
// shared world ("prrtc_planner_batch", count pointers NULL).
ffi::Error run_batch(cudaStream_t stream, ffi::ScratchAllocator& scratch, F32 start, F32 goals, F32 lo, F32 hi, const prrtc_robot_t& robot,
                     F32 ws, F32 wc, F32 wb, F32 wh, S32 sp, const int32_t* cws, const int32_t* cwc,
                     const int32_t* cwb, const int32_t* cwh, const int32_t* csp, bool batched,
                     const prrtc_outputs_t& out, const prrtc_attrs_t& a) {
    prrtc_batch_inputs_t in{};
    in.batch = rows(start);
    if (in.batch == 0) return ffi::Error::Success();
    in.start_configs = start.typed_data();
    in.goal_configs = goals.typed_data();
    in.num_goals = goals.dimensions().size() >= 2 ? static_cast<int>(goals.dimensions()[1]) : 1;
    in.goal_counts = nullptr;
    in.min_vals = lo.typed_data();
    in.max_vals = hi.typed_data();
    in.robot = robot;
    auto max_n = [batched](const auto& b) {
        const auto d = b.dimensions();
        if (batched) return d.size() >= 2 ? static_cast<int>(d[1]) : 0;
        return d.size() >= 1 ? static_cast<int>(d[0]) : 0;
    };
    in.world_spheres = ws.typed_data(); in.max_world_spheres = max_n(ws); in.world_spheres_count = cws;
    in.world_capsules = wc.typed_data(); in.max_world_capsules = max_n(wc); in.world_capsules_count = cwc;
    in.world_boxes = wb.typed_data(); in.max_world_boxes = max_n(wb); in.world_boxes_count = cwb;
    in.world_halfspaces = wh.typed_data(); in.max_world_halfspaces = max_n(wh); in.world_halfspaces_count = cwh;
    in.self_pairs = sp.typed_data(); in.max_self_pairs = max_n(sp); in.self_pairs_count = csp;
    in.problem_order = nullptr;
    const size_t need = prrtc_b200_plan_batch_workspace_size(&in, &a, nullptr);
    void* w = scratch_bytes(scratch, need);
    if (!w) return no_scratch(need);
    return status(prrtc_b200_plan_batch(&in, &out, &a, nullptr, w, need, stream));
}

ffi::Error BatchCtxImpl(cudaStream_t stream, ffi::ScratchAllocator scratch, F32 start, F32 goals, F32 lo, F32 hi, F32 tw, F32 ptf, S32 par,
                        S32 act, F32 mm, F32 mo, S32 mact, S32 topo, S32 sli, F32 sloc, F32 srad, F32 ws, F32 wc,
                        F32 wb, F32 wh, S32 sp, S32 nws, S32 nwc, S32 nwb, S32 nwh, S32 nsp, S32 cli, F32 cloc,
                        F32 crad, S32 foff, S32 cpairs, S32 cranges, RF32 ta, RF32 tb, RS32 pa, RS32 pb,
                        RS32 sizes, RS32 completed, RS32 iters, RS32 conn, RS32 solved, RF32 ktime,
                        int max_iterations, float step_size, int num_new_samples, int balance_mode,
                        float tree_ratio, int dynamic_domain, float dd_alpha, float dd_radius, float dd_min_radius,
                        int dim, int max_nodes, int granularity, int collision_mode, float collision_margin) {
    const prrtc_robot_t robot =
        robot_of(tw, ptf, par, act, mm, mo, mact, topo, sli, sloc, srad, cli, cloc, crad, foff, cpairs, cranges);
    const prrtc_attrs_t a = attrs_of(max_iterations, step_size, num_new_samples, balance_mode, tree_ratio,
                                     dynamic_domain, dd_alpha, dd_radius, dd_min_radius, dim, max_nodes, granularity,
                                     collision_mode, collision_margin);
    return run_batch(stream, scratch, start, goals, lo, hi, robot, ws, wc, wb, wh, sp, nws.typed_data(), nwc.typed_data(),
                     nwb.typed_data(), nwh.typed_data(), nsp.typed_data(), true,
                     outputs_of(ta, tb, pa, pb, sizes, completed, iters, conn, solved, ktime), a);
}

ffi::Error BatchImpl(cudaStream_t stream, ffi::ScratchAllocator scratch, F32 start, F32 goals, F32 lo, F32 hi, F32 tw, F32 ptf, S32 par, S32 act,
                     F32 mm, F32 mo, S32 mact, S32 topo, S32 sli, F32 sloc, F32 srad, F32 ws, F32 wc, F32 wb,
                     F32 wh, S32 sp, S32 cli, F32 cloc, F32 crad, S32 foff, S32 cpairs, S32 cranges, RF32 ta,
                     RF32 tb, RS32 pa, RS32 pb, RS32 sizes, RS32 completed, RS32 iters, RS32 conn, RS32 solved,
                     RF32 ktime, int max_iterations, float step_size, int num_new_samples, int balance_mode,
                     float tree_ratio, int dynamic_domain, float dd_alpha, float dd_radius, float dd_min_radius,
                     int dim, int max_nodes, int granularity, int collision_mode, float collision_margin) {
    const prrtc_robot_t robot =
        robot_of(tw, ptf, par, act, mm, mo, mact, topo, sli, sloc, srad, cli, cloc, crad, foff, cpairs, cranges);
    const prrtc_attrs_t a = attrs_of(max_iterations, step_size, num_new_samples, balance_mode, tree_ratio,
                                     dynamic_domain, dd_alpha, dd_radius, dd_min_radius, dim, max_nodes, granularity,
                                     collision_mode, collision_margin);
    return run_batch(stream, scratch, start, goals, lo, hi, robot, ws, wc, wb, wh, sp, nullptr, nullptr, nullptr, nullptr,
                     nullptr, false, outputs_of(ta, tb, pa, pb, sizes, completed, iters, conn, solved, ktime), a);
}

// prrtc_nearest_neighbor.cu:80-141; the tree size is read on the device (no host sync).
ffi::Error NearestNeighborImpl(cudaStream_t stream, ffi::ScratchAllocator scratch, F32 tree, F32 queries, S32 tree_size, RS32 indices, RF32 dists) {
    const auto td = tree.dimensions();
    if (td.size() != 2) return ffi::Error(ffi::ErrorCode::kInvalidArgument, "tree_configs must be [dim, max_nodes]");
    const int dim = static_cast<int>(td[0]), max_nodes = static_cast<int>(td[1]);
    const int batch = rows(queries);
    if (batch == 0) return ffi::Error::Success();
    const size_t need = prrtc_b200_nearest_neighbor_workspace_size(batch);
    void* w = scratch_bytes(scratch, need);
    if (!w) return no_scratch(need);
    return status(prrtc_b200_nearest_neighbor(tree.typed_data(), dim, max_nodes, tree_size.typed_data(),
                                              queries.typed_data(), batch, indices->typed_data(),
                                              dists->typed_data(), w, need, stream));
}

// prrtc_extend.cu:76-140; the step size is read on the device (no host sync).
ffi::Error ExtendImpl(cudaStream_t stream, F32 tree, S32 nearest, F32 samples, F32 step, RF32 new_configs,
                      RS32 parents, RS32 valid) {
    const auto td = tree.dimensions();
    if (td.size() != 2) return ffi::Error(ffi::ErrorCode::kInvalidArgument, "tree_configs must be [dim, max_nodes]");
    const int batch = rows(nearest);
    if (batch == 0) return ffi::Error::Success();
    return status(prrtc_b200_extend(tree.typed_data(), static_cast<int>(td[0]), static_cast<int>(td[1]),
                                    nearest.typed_data(), samples.typed_data(), batch, step.typed_data(),
                                    new_configs->typed_data(), parents->typed_data(), valid->typed_data(), stream));
}

// prrtc_iteration.cu:180-277: like the reference, the tree buffers are
// updated in place although XLA passes them as inputs.
ffi::Error IterationImpl(cudaStream_t stream, F32 ta, F32 tb, S32 pa, S32 pb, F32 samples, S32 sizes, S32 completed,
                         F32 step, RS32 new_configs, RS32 new_parents, RS32 valid, RS32 solved) {
    const auto td = ta.dimensions();
    if (td.size() != 2) return ffi::Error(ffi::ErrorCode::kInvalidArgument, "tree_a_configs must be [dim, max_nodes]");
    const int batch = rows(samples);
    if (batch == 0) return ffi::Error::Success();
    return status(prrtc_b200_iteration(const_cast<float*>(ta.typed_data()), const_cast<float*>(tb.typed_data()),
                                       const_cast<int32_t*>(pa.typed_data()), const_cast<int32_t*>(pb.typed_data()),
                                       static_cast<int>(td[0]), static_cast<int>(td[1]), samples.typed_data(), batch,
                                       const_cast<int32_t*>(sizes.typed_data()),
                                       const_cast<int32_t*>(completed.typed_data()), step.typed_data(),
                                       new_configs->typed_data(), new_parents->typed_data(), valid->typed_data(),
                                       solved->typed_data(), stream));
}

}  // namespace

#define PRRTC_PLANNER_BINDING                                                                          \
    ffi::Ffi::Bind()                                                                                   \
        .Ctx<ffi::PlatformStream<cudaStream_t>>()                                                      \
        .Ctx<ffi::ScratchAllocator>()                                                                  \
        .Arg<F32>().Arg<F32>().Arg<F32>().Arg<F32>()                /* start, goals, min, max */       \
        .Arg<F32>().Arg<F32>().Arg<S32>().Arg<S32>()                /* twists, parent_tf, parent, act */ \
        .Arg<F32>().Arg<F32>().Arg<S32>().Arg<S32>()                /* mimic mul/off/act, topo_inv */  \
        .Arg<S32>().Arg<F32>().Arg<F32>()                           /* sphere link/local/radius */     \
        .Arg<F32>().Arg<F32>().Arg<F32>().Arg<F32>().Arg<S32>()     /* world x4, self_pairs */         \
        .Arg<S32>().Arg<F32>().Arg<F32>().Arg<S32>().Arg<S32>().Arg<S32>() /* coarse model */          \
        .Ret<F32>().Ret<F32>().Ret<S32>().Ret<S32>().Ret<S32>().Ret<S32>().Ret<S32>().Ret<S32>()       \
        .Ret<S32>().Ret<F32>()                                                                         \
        .Attr<int>("max_iterations").Attr<float>("step_size").Attr<int>("num_new_samples")            \
        .Attr<int>("balance_mode").Attr<float>("tree_ratio").Attr<int>("dynamic_domain")              \
        .Attr<float>("dd_alpha").Attr<float>("dd_radius").Attr<float>("dd_min_radius")                \
        .Attr<int>("dim").Attr<int>("max_nodes").Attr<int>("granularity").Attr<int>("collision_mode")  \
        .Attr<float>("collision_margin")

#define PRRTC_ROBOT_ARGS                                                                               \
    .Arg<F32>().Arg<F32>().Arg<S32>().Arg<S32>()                /* twists, parent_tf, parent, act */   \
        .Arg<F32>().Arg<F32>().Arg<S32>().Arg<S32>()            /* mimic mul/off/act, topo_inv */      \
        .Arg<S32>().Arg<F32>().Arg<F32>()                       /* sphere link/local/radius */

#define PRRTC_COARSE_ARGS .Arg<S32>().Arg<F32>().Arg<F32>().Arg<S32>().Arg<S32>().Arg<S32>()

#define PRRTC_RESULTS                                                                                  \
    .Ret<F32>().Ret<F32>().Ret<S32>().Ret<S32>().Ret<S32>().Ret<S32>().Ret<S32>().Ret<S32>()           \
        .Ret<S32>().Ret<F32>()

#define PRRTC_ATTRS                                                                                    \
    .Attr<int>("max_iterations").Attr<float>("step_size").Attr<int>("num_new_samples")                \
        .Attr<int>("balance_mode").Attr<float>("tree_ratio").Attr<int>("dynamic_domain")              \
        .Attr<float>("dd_alpha").Attr<float>("dd_radius").Attr<float>("dd_min_radius")                \
        .Attr<int>("dim").Attr<int>("max_nodes").Attr<int>("granularity").Attr<int>("collision_mode")  \
        .Attr<float>("collision_margin")

XLA_FFI_DEFINE_HANDLER_SYMBOL(PrrtcPlannerFfi, PlannerImpl, PRRTC_PLANNER_BINDING);

// prrtc_planner.cu:1946-2005
XLA_FFI_DEFINE_HANDLER_SYMBOL(PrrtcPlannerBatchCtxFfi, BatchCtxImpl,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Ctx<ffi::ScratchAllocator>()
                                  .Arg<F32>().Arg<F32>().Arg<F32>().Arg<F32>()  /* start, goals, min, max */
                                  PRRTC_ROBOT_ARGS
                                  .Arg<F32>().Arg<F32>().Arg<F32>().Arg<F32>().Arg<S32>()  /* batched worlds */
                                  .Arg<S32>().Arg<S32>().Arg<S32>().Arg<S32>().Arg<S32>()  /* counts */
                                  PRRTC_COARSE_ARGS PRRTC_RESULTS PRRTC_ATTRS);

// prrtc_planner.cu:2007-2061
XLA_FFI_DEFINE_HANDLER_SYMBOL(PrrtcPlannerBatchFfi, BatchImpl,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Ctx<ffi::ScratchAllocator>()
                                  .Arg<F32>().Arg<F32>().Arg<F32>().Arg<F32>()  /* start, goals, min, max */
                                  PRRTC_ROBOT_ARGS
                                  .Arg<F32>().Arg<F32>().Arg<F32>().Arg<F32>().Arg<S32>()  /* shared world */
                                  PRRTC_COARSE_ARGS PRRTC_RESULTS PRRTC_ATTRS);

// prrtc_nearest_neighbor.cu:132-141
XLA_FFI_DEFINE_HANDLER_SYMBOL(PrrtcNearestNeighborFfi, NearestNeighborImpl,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Ctx<ffi::ScratchAllocator>()
                                  .Arg<F32>().Arg<F32>().Arg<S32>()
                                  .Ret<S32>().Ret<F32>());

// prrtc_extend.cu:129-140
XLA_FFI_DEFINE_HANDLER_SYMBOL(PrrtcExtendFfi, ExtendImpl,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Arg<F32>().Arg<S32>().Arg<F32>().Arg<F32>()
                                  .Ret<F32>().Ret<S32>().Ret<S32>());

// prrtc_iteration.cu:261-277
XLA_FFI_DEFINE_HANDLER_SYMBOL(PrrtcIterationFfi, IterationImpl,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Arg<F32>().Arg<F32>().Arg<S32>().Arg<S32>().Arg<F32>().Arg<S32>().Arg<S32>()
                                  .Arg<F32>()
                                  .Ret<S32>().Ret<S32>().Ret<S32>().Ret<S32>());

#endif  // PRRTC_WITH_XLA_FFI
