// capi.cu -- the extern "C" entry points declared in include/prrtc_b200.h.
// Argument validation mirrors the reference's Python checks (cuda-rrtc/jax/
// prrtc.py:353-381: power-of-two granularity <= 64, step_size > 0) plus the
// compile-time limits of its kernels (CONFIG_DIM_MAX 16, PRRTC_MAX_JOINTS 64).
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <mutex>

#include "../../include/prrtc_b200.h"
#include "kernels.h"
#include "prrtc_device.cuh"

using namespace prrtc;

static thread_local int g_last_cuda = 0;

static int cuda_fail(cudaError_t e) {
    g_last_cuda = (int)e;
    return PRRTC_B200_ECUDA;
}

static bool aligned(const void* p, size_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0; }

static int check_attrs(const prrtc_attrs_t* a) {
    if (!a) return PRRTC_B200_EARG;
    if (a->dim < 1 || a->dim > PRRTC_B200_DIM_MAX) return PRRTC_B200_EUNSUPPORTED;
    if (a->max_nodes < 1) return PRRTC_B200_EARG;
    if (!(a->step_size > 0.0f)) return PRRTC_B200_EARG;
    if (a->num_new_samples < 1) return PRRTC_B200_EARG;
    const int g = a->granularity;
    if (g < 1 || (g & (g - 1)) != 0 || g > PRRTC_B200_GRANULARITY_MAX) return PRRTC_B200_EARG;
    if (a->collision_mode < 0 || a->collision_mode > 3) return PRRTC_B200_EARG;
    if (a->max_iterations < 0) return PRRTC_B200_EARG;
    return PRRTC_B200_OK;
}

static int check_robot(const prrtc_robot_t& r) {
    if (r.n_joints < 0 || r.n_spheres < 0 || r.n_coarse < 0 || r.n_coarse_self_pairs < 0) return PRRTC_B200_EARG;
    if (r.n_joints > 0 && (!r.fk_twists || !r.fk_parent_tf || !r.fk_parent_idx)) return PRRTC_B200_EARG;
    if (r.n_spheres > 0 && (!r.sphere_link_idx || !r.sphere_local || !r.sphere_radius)) return PRRTC_B200_EARG;
    if (r.n_coarse > 0 && (!r.coarse_sphere_link_idx || !r.coarse_sphere_local || !r.coarse_sphere_radius))
        return PRRTC_B200_EARG;
    if (r.n_coarse_self_pairs > 0 && (!r.coarse_self_pairs || !r.self_pair_ranges)) return PRRTC_B200_EARG;
    return PRRTC_B200_OK;
}

static void robot_to_pack(const prrtc_robot_t& r, PackSrc& s) {
    s.twists = r.fk_twists; s.ptf = r.fk_parent_tf; s.parent = r.fk_parent_idx; s.act = r.fk_act_idx;
    s.mmul = r.fk_mimic_mul; s.moff = r.fk_mimic_off; s.mact = r.fk_mimic_act_idx; s.topo_inv = r.fk_topo_inv;
    s.J = r.n_joints > 0 ? r.n_joints : 0;
    s.sli = r.sphere_link_idx; s.sloc = r.sphere_local; s.srad = r.sphere_radius; s.S = r.n_spheres;
    // the coarse model is usable only with its K+1 offsets
    const bool coarse = r.n_coarse > 0 && r.fine_link_offsets != nullptr;
    s.cli = r.coarse_sphere_link_idx; s.cloc = r.coarse_sphere_local; s.crad = r.coarse_sphere_radius;
    s.foff = coarse ? r.fine_link_offsets : nullptr;
    s.K = coarse ? r.n_coarse : 0;
    s.cpairs = r.coarse_self_pairs; s.cranges = r.self_pair_ranges;
    s.Q = coarse ? r.n_coarse_self_pairs : 0;
}

static void world_to_pack(const prrtc_world_t& w, PackSrc& s) {
    s.ws = w.world_spheres; s.ws_max = std::max(0, w.n_world_spheres); s.ws_cnt = nullptr;
    s.wc = w.world_capsules; s.wc_max = std::max(0, w.n_world_capsules); s.wc_cnt = nullptr;
    s.wb = w.world_boxes; s.wb_max = std::max(0, w.n_world_boxes); s.wb_cnt = nullptr;
    s.wh = w.world_halfspaces; s.wh_max = std::max(0, w.n_world_halfspaces); s.wh_cnt = nullptr;
    s.sp = w.self_pairs; s.sp_max = std::max(0, w.n_self_pairs); s.sp_cnt = nullptr;
}

static PackSrc make_pack(const prrtc_robot_t& r, const prrtc_world_t& w, int dim, int mode, float margin) {
    PackSrc s;
    memset(&s, 0, sizeof(s));
    robot_to_pack(r, s);
    world_to_pack(w, s);
    s.dim = dim;
    s.mode = mode;
    s.margin = margin;
    return s;
}

struct Tuned {
    float edge_res;
    int threads, cw, resident;
    unsigned long long* stats;
    const prrtc_point_cloud_t* cloud;
    int tail_join;
    int wait_polls;
    int ctas_per_sm;
    cudaEvent_t explore_events[2];
};

static PcView pc_view(const prrtc_point_cloud_t* c) {
    if (!c || c->n_points <= 0 || !c->points || !c->bucket_start) return PcView{nullptr, nullptr, 0, 0, 0.0f, 0.0f};
    return PcView{reinterpret_cast<const float4*>(c->points), c->bucket_start, c->n_points, c->n_buckets - 1,
                  1.0f / c->cell, c->r_env};
}

// A cloud descriptor is usable when its bucket count is a power of two and its
// cell and radius are sane (NULL or empty = no cloud).
static bool cloud_ok(const prrtc_point_cloud_t* c) {
    if (!c || c->n_points == 0) return true;
    const int H = c->n_buckets;
    return c->n_points > 0 && c->points && c->bucket_start && H > 0 && (H & (H - 1)) == 0 && H <= (1 << 24) &&
           c->cell >= 1e-3f && c->r_env >= 0.0f && aligned(c->points, 16);
}

static Tuned tuned(const prrtc_tuning_t* t) {
    Tuned o{0.0f, 128, 16, 0, nullptr, nullptr, 1, 0, 0, {nullptr, nullptr}};
    if (t) {
        if (t->edge_resolution > 0.0f) o.edge_res = t->edge_resolution;
        if (t->threads_per_explorer == 32 || t->threads_per_explorer == 64 || t->threads_per_explorer == 128 ||
            t->threads_per_explorer == 256)
            o.threads = t->threads_per_explorer;
        if (t->waypoint_chunk == 8 || t->waypoint_chunk == 16 || t->waypoint_chunk == 32 || t->waypoint_chunk == 64)
            o.cw = t->waypoint_chunk;
        if (t->resident_ctas > 0) o.resident = t->resident_ctas;
        o.stats = reinterpret_cast<unsigned long long*>(t->stats);
        o.cloud = t->point_cloud;
        o.tail_join = t->tail_explorers < 0 ? 0 : 1;
        o.wait_polls = t->staging_wait_polls > 0 ? t->staging_wait_polls : (t->staging_wait_polls < 0 ? -1 : 0);
        o.ctas_per_sm = t->ctas_per_sm > 0 ? t->ctas_per_sm : 0;
        o.explore_events[0] = static_cast<cudaEvent_t>(t->explore_events[0]);
        o.explore_events[1] = static_cast<cudaEvent_t>(t->explore_events[1]);
    }
    return o;
}

static void fill_launch(PlanLaunch& L, const prrtc_outputs_t* out, const prrtc_attrs_t* a, const Tuned& tu,
                        const PackSrc& s) {
    L.tree_a = out->tree_a_configs; L.tree_b = out->tree_b_configs;
    L.par_a = out->tree_a_parents; L.par_b = out->tree_b_parents;
    L.sizes = out->tree_sizes; L.completed = out->completed; L.iter_count = out->iter_count;
    L.connection = out->connection_info; L.solved = out->solved_flag; L.ktime = out->kernel_time_ms;
    L.E = a->num_new_samples; L.N = a->max_nodes; L.dim = a->dim;
    L.J = s.J; L.S = s.S; L.K = s.K; L.Q = s.Q;
    L.max_iter = a->max_iterations; L.balance_mode = a->balance_mode; L.dd = a->dynamic_domain ? 1 : 0;
    L.granularity = a->granularity; L.step = a->step_size; L.tree_ratio = a->tree_ratio;
    L.dd_alpha = a->dd_alpha; L.dd_radius = a->dd_radius; L.dd_min_radius = a->dd_min_radius;
    L.edge_res = tu.edge_res; L.threads = tu.threads; L.cw = tu.cw; L.resident = tu.resident;
    L.stats = tu.stats;
    L.pc = pc_view(tu.cloud);
    L.tail_join = tu.tail_join;
    L.wait_polls = tu.wait_polls;
    L.ctas_per_sm = tu.ctas_per_sm;
    L.explore_events[0] = tu.explore_events[0];
    L.explore_events[1] = tu.explore_events[1];
}

static bool outputs_ok(const prrtc_outputs_t* o) {
    return o && o->tree_a_configs && o->tree_b_configs && o->tree_a_parents && o->tree_b_parents &&
           o->tree_sizes && o->completed && o->iter_count && o->connection_info && o->solved_flag &&
           o->kernel_time_ms;
}

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

// A driver entry point looked up through the runtime (no link against libcuda).
static void* driver_entry(const char* name) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
        p = nullptr;
    return p;
}

// The current CUDA context's identity: cuCtxGetId, unique to each creation of a
// context (the primary context re-created after cudaDeviceReset gets a new id,
// while its handle may be the old one), else the handle itself; 0 = unknown.
unsigned long long prrtc::current_context_key() {
    static const auto get_ctx = reinterpret_cast<CtxGetCurrentFn>(driver_entry("cuCtxGetCurrent"));
    static const auto get_id = reinterpret_cast<CtxGetIdFn>(driver_entry("cuCtxGetId"));
    CUcontext ctx = nullptr;
    if (!get_ctx || get_ctx(&ctx) != CUDA_SUCCESS || !ctx) return 0ull;
    unsigned long long id = 0ull;
    if (get_id && get_id(ctx, &id) == CUDA_SUCCESS && id != 0ull) return id;
    return static_cast<unsigned long long>(reinterpret_cast<uintptr_t>(ctx));
}

extern "C" {

int prrtc_b200_version(void) { return 1; }

int prrtc_b200_last_cuda_error(void) { return g_last_cuda; }

const char* prrtc_b200_error_string(int code) {
    switch (code) {
        case PRRTC_B200_OK: return "ok";
        case PRRTC_B200_EARG: return "invalid argument";
        case PRRTC_B200_EWORKSPACE: return "workspace missing, too small or not 256-byte aligned";
        case PRRTC_B200_ECUDA: return cudaGetErrorString((cudaError_t)g_last_cuda);
        case PRRTC_B200_EUNSUPPORTED: return "shape outside the supported limits";
        case PRRTC_B200_ETOOLARGE:
            return "scene larger than the no-allocation scene buffer (PRRTC_B200_NOALLOC_SCENE_MAX bytes)";
        default: return "unknown error";
    }
}

size_t prrtc_b200_plan_workspace_size(const prrtc_inputs_t* in, const prrtc_attrs_t* a, const prrtc_tuning_t*) {
    if (!in || !a) return 0;
    const PackSrc s = make_pack(in->robot, in->world, a->dim, a->collision_mode, a->collision_margin);
    return plan_workspace_bytes(1, std::max(a->max_nodes, 1), blob_stride(s));
}

int prrtc_b200_plan(const prrtc_inputs_t* in, const prrtc_outputs_t* out, const prrtc_attrs_t* a,
                    const prrtc_tuning_t* tuning, void* ws, size_t ws_bytes, void* stream) {
    int rc = check_attrs(a);
    if (rc) return rc;
    if (!in || !outputs_ok(out) || !in->start_config || !in->goal_configs || !in->min_vals || !in->max_vals)
        return PRRTC_B200_EARG;
    if (in->num_goals < 1 || in->num_goals > a->max_nodes) return PRRTC_B200_EARG;
    if ((rc = check_robot(in->robot))) return rc;
    const Tuned tu = tuned(tuning);
    if (!cloud_ok(tu.cloud)) return PRRTC_B200_EARG;
    PackSrc s = make_pack(in->robot, in->world, a->dim, a->collision_mode, a->collision_margin);
    s.has_cloud = pc_view(tu.cloud).n > 0;
    const size_t stride = blob_stride(s);
    if (!ws || !aligned(ws, 256) || ws_bytes < plan_workspace_bytes(1, a->max_nodes, stride))
        return PRRTC_B200_EWORKSPACE;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    PlanLaunch L;
    memset(&L, 0, sizeof(L));
    L.B = 1;
    fill_launch(L, out, a, tu, s);
    plan_carve_workspace(L, ws, stride);
    L.blob_cap = (int)stride;
    L.starts = in->start_config; L.goals = in->goal_configs; L.num_goals = in->num_goals; L.goal_counts = nullptr;
    L.lo = in->min_vals; L.hi = in->max_vals;
    L.pairs = in->world.self_pairs; L.pairs_stride = 0;
    L.order = nullptr;
    L.persistent = 0;
    cudaError_t e = launch_pack(s, 1, L.blobs, stride, st);
    if (e != cudaSuccess) return cuda_fail(e);
    e = launch_plan(L, st);
    if (e != cudaSuccess) return cuda_fail(e);
    return PRRTC_B200_OK;
}

static PackSrc make_batch_pack(const prrtc_batch_inputs_t* in, int dim, int mode, float margin) {
    PackSrc s;
    memset(&s, 0, sizeof(s));
    robot_to_pack(in->robot, s);
    s.ws = in->world_spheres; s.ws_max = std::max(0, in->max_world_spheres); s.ws_cnt = in->world_spheres_count;
    s.wc = in->world_capsules; s.wc_max = std::max(0, in->max_world_capsules); s.wc_cnt = in->world_capsules_count;
    s.wb = in->world_boxes; s.wb_max = std::max(0, in->max_world_boxes); s.wb_cnt = in->world_boxes_count;
    s.wh = in->world_halfspaces; s.wh_max = std::max(0, in->max_world_halfspaces);
    s.wh_cnt = in->world_halfspaces_count;
    s.sp = in->self_pairs; s.sp_max = std::max(0, in->max_self_pairs); s.sp_cnt = in->self_pairs_count;
    s.dim = dim;
    s.mode = mode;
    s.margin = margin;
    return s;
}

size_t prrtc_b200_plan_batch_workspace_size(const prrtc_batch_inputs_t* in, const prrtc_attrs_t* a,
                                            const prrtc_tuning_t*) {
    if (!in || !a || in->batch < 1) return 0;
    const PackSrc s = make_batch_pack(in, a->dim, a->collision_mode, a->collision_margin);
    return plan_workspace_bytes(in->batch, std::max(a->max_nodes, 1), blob_stride(s));
}

int prrtc_b200_plan_batch(const prrtc_batch_inputs_t* in, const prrtc_outputs_t* out, const prrtc_attrs_t* a,
                          const prrtc_tuning_t* tuning, void* ws, size_t ws_bytes, void* stream) {
    int rc = check_attrs(a);
    if (rc) return rc;
    if (!in || !outputs_ok(out) || in->batch < 1 || !in->start_configs || !in->goal_configs || !in->min_vals ||
        !in->max_vals)
        return PRRTC_B200_EARG;
    if (in->num_goals < 1 || in->num_goals > a->max_nodes) return PRRTC_B200_EARG;
    if ((rc = check_robot(in->robot))) return rc;
    const Tuned tu = tuned(tuning);
    if (!cloud_ok(tu.cloud)) return PRRTC_B200_EARG;
    PackSrc s = make_batch_pack(in, a->dim, a->collision_mode, a->collision_margin);
    s.has_cloud = pc_view(tu.cloud).n > 0;
    const size_t stride = blob_stride(s);
    if (!ws || !aligned(ws, 256) || ws_bytes < plan_workspace_bytes(in->batch, a->max_nodes, stride))
        return PRRTC_B200_EWORKSPACE;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    PlanLaunch L;
    memset(&L, 0, sizeof(L));
    L.B = in->batch;
    fill_launch(L, out, a, tu, s);
    plan_carve_workspace(L, ws, stride);
    L.blob_cap = (int)stride;
    L.starts = in->start_configs; L.goals = in->goal_configs; L.num_goals = in->num_goals;
    L.goal_counts = in->goal_counts;
    L.lo = in->min_vals; L.hi = in->max_vals;
    L.pairs = in->self_pairs;
    L.pairs_stride = in->self_pairs_count ? (size_t)std::max(0, in->max_self_pairs) : 0;
    L.order = in->problem_order;
    L.caps = in->problem_capacity;
    L.persistent = 1;
    cudaError_t e = launch_pack(s, in->batch, L.blobs, stride, st);
    if (e != cudaSuccess) return cuda_fail(e);
    e = launch_plan(L, st);
    if (e != cudaSuccess) return cuda_fail(e);
    return PRRTC_B200_OK;
}

size_t prrtc_b200_nearest_neighbor_workspace_size(int32_t batch) {
    return (((size_t)std::max(batch, 1) * sizeof(unsigned long long)) + 255) & ~(size_t)255;
}

int prrtc_b200_nearest_neighbor(const float* tree, int32_t dim, int32_t max_nodes, const int32_t* tree_size,
                                const float* queries, int32_t batch, int32_t* indices, float* dists, void* ws,
                                size_t ws_bytes, void* stream) {
    if (batch == 0) return PRRTC_B200_OK;
    if (!tree || !queries || !indices || !dists || batch < 0 || max_nodes < 1) return PRRTC_B200_EARG;
    if (dim < 1 || dim > PRRTC_B200_DIM_MAX) return PRRTC_B200_EUNSUPPORTED;
    if (!ws || !aligned(ws, 256) || ws_bytes < prrtc_b200_nearest_neighbor_workspace_size(batch))
        return PRRTC_B200_EWORKSPACE;
    cudaError_t e = launch_nearest(tree, dim, max_nodes, tree_size, queries, batch, indices, dists,
                                   static_cast<unsigned long long*>(ws), static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? PRRTC_B200_OK : cuda_fail(e);
}

int prrtc_b200_extend(const float* tree, int32_t dim, int32_t max_nodes, const int32_t* nearest,
                      const float* samples, int32_t batch, const float* step, float* out, int32_t* parents,
                      int32_t* valid, void* stream) {
    if (batch == 0) return PRRTC_B200_OK;
    if (!tree || !nearest || !samples || !step || !out || !parents || !valid || batch < 0 || max_nodes < 1)
        return PRRTC_B200_EARG;
    if (dim < 1 || dim > PRRTC_B200_DIM_MAX) return PRRTC_B200_EUNSUPPORTED;
    cudaError_t e = launch_extend(tree, dim, max_nodes, nearest, samples, batch, step, out, parents, valid,
                                  static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? PRRTC_B200_OK : cuda_fail(e);
}

int prrtc_b200_iteration(float* ta, float* tb, int32_t* pa, int32_t* pb, int32_t dim, int32_t max_nodes,
                         const float* samples, int32_t batch, int32_t* sizes, int32_t* completed, const float* step,
                         int32_t* new_cfg, int32_t* new_par, int32_t* valid, int32_t* solved, void* stream) {
    if (batch == 0) return PRRTC_B200_OK;
    if (!ta || !tb || !pa || !pb || !samples || !sizes || !completed || !step || !new_cfg || !new_par || !valid ||
        !solved || batch < 0 || max_nodes < 1)
        return PRRTC_B200_EARG;
    if (dim < 1 || dim > PRRTC_B200_DIM_MAX) return PRRTC_B200_EUNSUPPORTED;
    if ((long long)batch * 32 > INT32_MAX) return PRRTC_B200_EUNSUPPORTED;
    cudaError_t e = launch_iteration(ta, tb, pa, pb, dim, max_nodes, samples, batch, sizes, completed, step, new_cfg,
                                     new_par, valid, solved, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? PRRTC_B200_OK : cuda_fail(e);
}

size_t prrtc_b200_check_configs_workspace_size(const prrtc_robot_t* robot, const prrtc_world_t* world) {
    if (!robot || !world) return 0;
    return blob_stride(make_pack(*robot, *world, 1, 0, 0.0f));
}

// The batched checker sweeps every obstacle for the flat checkers (binary,
// differentiable) even when early exit is allowed: the verdicts are the same,
// and the full sweep measured faster (471 vs 405 M checks/s on 2^20 random
// tabletop configurations, 79% in collision: most work items run before a
// configuration's first hit is known).  The coarse-gated checkers keep early
// exit (393 vs 385 M checks/s).
static int32_t batch_sweep(int32_t mode, int32_t full_sweep) { return (full_sweep || mode == 0 || mode == 1) ? 1 : 0; }

int prrtc_b200_check_configs(const prrtc_robot_t* robot, const prrtc_world_t* world, int32_t dim,
                             const float* configs, int32_t n, int32_t mode, float margin, int32_t full_sweep,
                             int32_t* verdicts, void* ws, size_t ws_bytes, void* stream) {
    if (n == 0) return PRRTC_B200_OK;
    if (!robot || !world || !configs || !verdicts || n < 0 || mode < 0 || mode > 3) return PRRTC_B200_EARG;
    if (dim < 1 || dim > PRRTC_B200_DIM_MAX) return PRRTC_B200_EUNSUPPORTED;
    int rc = check_robot(*robot);
    if (rc) return rc;
    const PackSrc s = make_pack(*robot, *world, dim, mode, margin);
    const size_t stride = blob_stride(s);
    if (!ws || !aligned(ws, 256) || ws_bytes < stride) return PRRTC_B200_EWORKSPACE;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char* blob = static_cast<unsigned char*>(ws);
    cudaError_t e = launch_pack(s, 1, blob, stride, st);
    if (e != cudaSuccess) return cuda_fail(e);
    e = launch_check(blob, (int)stride, world->self_pairs, s.J, s.S, s.K, s.Q, dim, configs, n,
                     batch_sweep(mode, full_sweep), verdicts,
                     st);
    return e == cudaSuccess ? PRRTC_B200_OK : cuda_fail(e);
}

static int pc_buckets(int32_t n_points, int32_t n_buckets) {
    if (n_buckets > 0) return n_buckets;
    int H = 1024;
    while (H < n_points && H < (1 << 24)) H <<= 1;
    return H;
}

size_t prrtc_b200_point_cloud_workspace_size(int32_t n_points, int32_t n_buckets) {
    if (n_points < 0) return 0;
    const int H = pc_buckets(n_points, n_buckets);
    return pc_workspace_bytes(n_points, H);
}

int prrtc_b200_point_cloud_build(const float* points, int32_t n_points, float cell, float r_env, int32_t n_buckets,
                                 void* ws, size_t ws_bytes, prrtc_point_cloud_t* cloud, void* stream) {
    if (!cloud || n_points < 0 || (n_points > 0 && !points) || n_buckets < 0) return PRRTC_B200_EARG;
    if (!(cell >= 1e-3f) || !(r_env >= 0.0f) || !(r_env < 1e3f)) return PRRTC_B200_EARG;
    const int H = pc_buckets(n_points, n_buckets);
    if ((H & (H - 1)) != 0 || H > (1 << 24)) return PRRTC_B200_EUNSUPPORTED;
    if (!ws || !aligned(ws, 256) || ws_bytes < pc_workspace_bytes(n_points, H)) return PRRTC_B200_EWORKSPACE;
    PcView v;
    cudaError_t e = launch_pc_build(points, n_points, cell, r_env, H, ws, &v, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e);
    cloud->points = reinterpret_cast<const float*>(v.pts);
    cloud->bucket_start = v.start;
    cloud->n_points = n_points;
    cloud->n_buckets = H;
    cloud->cell = cell;
    cloud->r_env = r_env;
    return PRRTC_B200_OK;
}

size_t prrtc_b200_check_edges_workspace_size(const prrtc_robot_t* robot, const prrtc_world_t* world,
                                             int32_t n_edges, int32_t granularity) {
    if (!robot || !world || n_edges < 0 || granularity < 0) return 0;
    const size_t blob = blob_stride(make_pack(*robot, *world, 1, 0, 0.0f));
    return blob + ((((size_t)n_edges * granularity * sizeof(int32_t)) + 255) & ~(size_t)255);
}

int prrtc_b200_check_edges(const prrtc_robot_t* robot, const prrtc_world_t* world, const prrtc_point_cloud_t* cloud,
                           int32_t dim, const float* edges, int32_t n_edges, int32_t G, int32_t mode, float margin,
                           int32_t* free_flags, void* ws, size_t ws_bytes, void* stream) {
    if (n_edges == 0) return PRRTC_B200_OK;
    if (!robot || !world || !edges || !free_flags || n_edges < 0 || G < 1 || mode < 0 || mode > 3)
        return PRRTC_B200_EARG;
    if (dim < 1 || dim > PRRTC_B200_DIM_MAX) return PRRTC_B200_EUNSUPPORTED;
    if ((long long)n_edges * G > INT32_MAX) return PRRTC_B200_EUNSUPPORTED;
    if (!cloud_ok(cloud)) return PRRTC_B200_EARG;
    int rc = check_robot(*robot);
    if (rc) return rc;
    PackSrc s = make_pack(*robot, *world, dim, mode, margin);
    const PcView pc = pc_view(cloud);
    s.has_cloud = pc.n > 0;
    const size_t stride = blob_stride(s);
    if (!ws || !aligned(ws, 256) || ws_bytes < prrtc_b200_check_edges_workspace_size(robot, world, n_edges, G))
        return PRRTC_B200_EWORKSPACE;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char* blob = static_cast<unsigned char*>(ws);
    int32_t* verdicts = reinterpret_cast<int32_t*>(blob + stride);
    cudaError_t e = launch_pack(s, 1, blob, stride, st);
    if (e != cudaSuccess) return cuda_fail(e);
    e = launch_check(blob, (int)stride, world->self_pairs, s.J, s.S, s.K, s.Q, dim, edges, n_edges * G,
                     batch_sweep(mode, 0), verdicts,
                     st, &pc);
    if (e != cudaSuccess) return cuda_fail(e);
    e = launch_edge_reduce(verdicts, n_edges, G, free_flags, st);
    return e == cudaSuccess ? PRRTC_B200_OK : cuda_fail(e);
}

int prrtc_b200_fk(const prrtc_robot_t* robot, int32_t dim, const float* configs, int32_t n, float* frames,
                  void* stream) {
    if (n == 0) return PRRTC_B200_OK;
    if (!robot || !configs || !frames || n < 0) return PRRTC_B200_EARG;
    if (dim < 1 || dim > PRRTC_B200_DIM_MAX) return PRRTC_B200_EUNSUPPORTED;
    if (robot->n_joints < 1 || robot->n_joints > PRRTC_B200_MAX_JOINTS) return PRRTC_B200_EUNSUPPORTED;
    FkTables t{robot->fk_twists, robot->fk_parent_tf, robot->fk_parent_idx, robot->fk_act_idx, robot->fk_mimic_mul,
               robot->fk_mimic_off, robot->fk_mimic_act_idx, robot->fk_topo_inv, robot->n_joints};
    cudaError_t e = launch_fk(t, dim, configs, n, frames, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? PRRTC_B200_OK : cuda_fail(e);
}

int prrtc_b200_halton(int32_t explorer, int32_t n, int32_t dim, const float* lo, const float* hi, float* samples,
                      void* stream) {
    if (n == 0) return PRRTC_B200_OK;
    if (!lo || !hi || !samples || n < 0 || explorer < 0) return PRRTC_B200_EARG;
    if (dim < 1 || dim > PRRTC_B200_DIM_MAX) return PRRTC_B200_EUNSUPPORTED;
    cudaError_t e = launch_halton(explorer, n, dim, lo, hi, samples, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? PRRTC_B200_OK : cuda_fail(e);
}

int prrtc_b200_choose_tree(int32_t mode, int32_t n, const int32_t* sizes, const int32_t* local_iter,
                           const int32_t* vamp_in, int32_t nblocks, float tree_ratio, int32_t* tree_out,
                           int32_t* vamp_out, void* stream) {
    if (n == 0) return PRRTC_B200_OK;
    if (n < 0 || mode < 0 || nblocks < 1 || nblocks > (1 << 24) || !sizes || !local_iter || !vamp_in || !tree_out ||
        !vamp_out)
        return PRRTC_B200_EARG;
    cudaError_t e = launch_choose_tree(mode, n, sizes, local_iter, vamp_in, nblocks, tree_ratio, tree_out, vamp_out,
                                       static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? PRRTC_B200_OK : cuda_fail(e);
}

int prrtc_b200_radius_update(float* radii, const int32_t* idx, const int32_t* op, int32_t n, float alpha, float r0,
                             float rmin, int32_t sequential, int32_t* err, void* stream) {
    if (n == 0) return PRRTC_B200_OK;
    if (n < 0 || !radii || !idx || !op) return PRRTC_B200_EARG;
    cudaError_t e = launch_radius_update(radii, idx, op, n, alpha, r0, rmin, sequential, err,
                                         static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? PRRTC_B200_OK : cuda_fail(e);
}

int prrtc_b200_extract_paths(int32_t batch, int32_t dim, int32_t max_nodes, const float* ta, const float* tb,
                             const int32_t* pa, const int32_t* pb, const int32_t* conn, const int32_t* solved,
                             int32_t max_len, float* paths, int32_t* lengths, float* costs, void* stream) {
    if (batch == 0) return PRRTC_B200_OK;
    if (batch < 0 || !ta || !tb || !pa || !pb || !conn || !solved || !paths || !lengths || !costs ||
        max_len < 1 || max_nodes < 1)
        return PRRTC_B200_EARG;
    if (dim < 1 || dim > PRRTC_B200_DIM_MAX) return PRRTC_B200_EUNSUPPORTED;
    if ((size_t)max_len * sizeof(int) > device_max_smem()) return PRRTC_B200_EUNSUPPORTED;
    cudaError_t e = launch_extract_paths(batch, dim, max_nodes, ta, tb, pa, pb, conn, solved, max_len, paths,
                                         lengths, costs, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? PRRTC_B200_OK : cuda_fail(e);
}

int prrtc_b200_result_block(int32_t batch, int32_t dim, int32_t max_len, const int32_t* sizes,
                            const int32_t* completed, const int32_t* iterations, const int32_t* connection_info,
                            const int32_t* solved_flag, const float* kernel_ms, const int32_t* lengths,
                            const float* costs, const float* paths, int32_t* block, float* packed_paths,
                            int64_t packed_capacity, void* stream) {
    if (batch == 0) return PRRTC_B200_OK;
    if (batch < 0 || !sizes || !completed || !iterations || !connection_info || !solved_flag || !kernel_ms ||
        !lengths || !costs || !block || packed_capacity < 0 || (packed_paths && (!paths || max_len < 1)))
        return PRRTC_B200_EARG;
    if (dim < 1 || dim > PRRTC_B200_DIM_MAX) return PRRTC_B200_EUNSUPPORTED;
    const ResultSrc R{sizes, completed, iterations, connection_info, solved_flag, kernel_ms, lengths, costs};
    cudaError_t e = launch_result_block(batch, dim, max_len, R, block, paths, packed_paths, packed_capacity,
                                        static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? PRRTC_B200_OK : cuda_fail(e);
}

size_t prrtc_b200_smooth_workspace_size(const prrtc_robot_t* robot, const prrtc_world_t* world) {
    if (!robot || !world) return 0;
    return blob_stride(make_pack(*robot, *world, 1, 0, 0.0f));
}

int prrtc_b200_smooth_cost_grad(const prrtc_robot_t* robot, const prrtc_world_t* world, int32_t dim,
                                const float* waypoints, int32_t n_paths, int32_t n_waypoints, float margin,
                                float beta, float w_len, float* cost, float* grad, void* ws, size_t ws_bytes,
                                void* stream) {
    if (n_paths == 0) return PRRTC_B200_OK;
    if (!robot || !world || !waypoints || !cost || n_paths < 0 || n_waypoints < 1 || !(beta > 0.0f))
        return PRRTC_B200_EARG;
    if (dim < 1 || dim > PRRTC_B200_DIM_MAX) return PRRTC_B200_EUNSUPPORTED;
    if (robot->n_joints < 1 || robot->n_joints > PRRTC_B200_MAX_JOINTS) return PRRTC_B200_EUNSUPPORTED;
    int rc = check_robot(*robot);
    if (rc) return rc;
    // the flat model: every sphere, every pair (no coarse gating in a smooth cost)
    const PackSrc s = make_pack(*robot, *world, dim, 0, 0.0f);
    const size_t stride = blob_stride(s);
    if (!ws || !aligned(ws, 256) || ws_bytes < stride) return PRRTC_B200_EWORKSPACE;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char* blob = static_cast<unsigned char*>(ws);
    cudaError_t e = launch_pack(s, 1, blob, stride, st);
    if (e != cudaSuccess) return cuda_fail(e);
    e = launch_smooth(blob, 0, world->self_pairs, 0, s.J, s.S, dim, waypoints, n_paths, n_waypoints, margin, beta,
                      w_len, cost, grad, st);
    return e == cudaSuccess ? PRRTC_B200_OK : cuda_fail(e);
}

size_t prrtc_b200_smooth_batch_workspace_size(const prrtc_batch_inputs_t* in) {
    if (!in || in->batch < 1) return 0;
    return (size_t)in->batch * blob_stride(make_batch_pack(in, 1, 0, 0.0f));
}

int prrtc_b200_smooth_cost_grad_batch(const prrtc_batch_inputs_t* in, int32_t dim, const float* waypoints,
                                      int32_t n_waypoints, float margin, float beta, float w_len, float* cost,
                                      float* grad, void* ws, size_t ws_bytes, void* stream) {
    if (!in) return PRRTC_B200_EARG;
    if (in->batch == 0) return PRRTC_B200_OK;
    if (in->batch < 0 || !waypoints || !cost || n_waypoints < 1 || !(beta > 0.0f)) return PRRTC_B200_EARG;
    if (dim < 1 || dim > PRRTC_B200_DIM_MAX) return PRRTC_B200_EUNSUPPORTED;
    if (in->robot.n_joints < 1 || in->robot.n_joints > PRRTC_B200_MAX_JOINTS) return PRRTC_B200_EUNSUPPORTED;
    int rc = check_robot(in->robot);
    if (rc) return rc;
    const PackSrc s = make_batch_pack(in, dim, 0, 0.0f);  // flat model, as the single-scene form
    const size_t stride = blob_stride(s);
    if (!ws || !aligned(ws, 256) || ws_bytes < (size_t)in->batch * stride) return PRRTC_B200_EWORKSPACE;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char* blobs = static_cast<unsigned char*>(ws);
    cudaError_t e = launch_pack(s, in->batch, blobs, stride, st);
    if (e != cudaSuccess) return cuda_fail(e);
    const size_t pstride = in->self_pairs_count ? (size_t)std::max(0, in->max_self_pairs) : 0;
    e = launch_smooth(blobs, stride, in->self_pairs, pstride, s.J, s.S, dim, waypoints, in->batch, n_waypoints,
                      margin, beta, w_len, cost, grad, st);
    return e == cudaSuccess ? PRRTC_B200_OK : cuda_fail(e);
}

// ---------------------------------------------------------------------------
// Collision check without allocation.  Some callers cannot call cudaMalloc or
// hand out scratch memory -- code running while another library captures the
// stream into a CUDA graph, real-time control loops that forbid allocation once
// started, plug-in hosts whose allocator is not reachable from the calling
// thread.  For them the packed scene lives in this file-scope device array.
// Every GPU that loads the library holds the array until the process exits.
// Each call rewrites the array completely (the pack kernel writes the header
// and every section the checker reads), so nothing has to be cleared between
// calls; calls that overlap on the GPU (different streams, or different host
// threads on one device) share the array and race.
static __device__ __align__(256) unsigned char g_noalloc_scene[PRRTC_B200_NOALLOC_SCENE_MAX];

static std::mutex g_noalloc_mutex;
// Device address of g_noalloc_scene per device ordinal, with the CUDA context it
// belongs to: the address is valid only in that context.
static unsigned char* g_noalloc_ptr[256];
static unsigned long long g_noalloc_ctx[256];  // context key of each cached address

// Host code cannot use g_noalloc_scene's name as a device address: resolve it
// with the device current, once per device and context.  A call made in a
// context other than the one of the cached address (another driver context made
// current, or the primary context re-created after cudaDeviceReset) resolves it
// again.
static int noalloc_scene_ptr(unsigned char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e);
    if (dev < 0 || dev >= 256) return PRRTC_B200_EUNSUPPORTED;
    unsigned long long key = current_context_key();
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev] || !key || key != g_noalloc_ctx[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scene);  // makes the device's primary context current if none is
        if (e != cudaSuccess) return cuda_fail(e);
        key = current_context_key();
        g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
        g_noalloc_ctx[dev] = key;
    }
    *out = g_noalloc_ptr[dev];
    return PRRTC_B200_OK;
}

int prrtc_b200_check_configs_noalloc(const prrtc_robot_t* robot, const prrtc_world_t* world, int32_t dim,
                                     const float* configs, int32_t n, int32_t mode, float margin,
                                     int32_t full_sweep, int32_t* verdicts, void* stream) {
    if (n == 0) return PRRTC_B200_OK;
    if (!robot || !world || !configs || !verdicts || n < 0 || mode < 0 || mode > 3) return PRRTC_B200_EARG;
    if (dim < 1 || dim > PRRTC_B200_DIM_MAX) return PRRTC_B200_EUNSUPPORTED;
    int rc = check_robot(*robot);
    if (rc) return rc;
    const PackSrc s = make_pack(*robot, *world, dim, mode, margin);
    const size_t stride = blob_stride(s);
    if (stride > (size_t)PRRTC_B200_NOALLOC_SCENE_MAX) return PRRTC_B200_ETOOLARGE;
    unsigned char* blob = nullptr;
    if ((rc = noalloc_scene_ptr(&blob))) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = launch_pack(s, 1, blob, stride, st);
    if (e != cudaSuccess) return cuda_fail(e);
    e = launch_check(blob, (int)stride, world->self_pairs, s.J, s.S, s.K, s.Q, dim, configs, n,
                     batch_sweep(mode, full_sweep), verdicts,
                     st);
    return e == cudaSuccess ? PRRTC_B200_OK : cuda_fail(e);
}

int prrtc_b200_fp32_probe(int32_t blocks, int32_t threads, int32_t iters, float* sink, void* stream) {
    if (blocks < 1 || threads < 32 || threads > 1024 || iters < 1 || !sink) return PRRTC_B200_EARG;
    cudaError_t e = launch_fp32_probe(blocks, threads, iters, sink, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? PRRTC_B200_OK : cuda_fail(e);
}

int prrtc_b200_fp32x2_probe(int32_t blocks, int32_t threads, int32_t iters, float* sink, void* stream) {
    if (blocks < 1 || threads < 32 || threads > 1024 || iters < 1 || !sink) return PRRTC_B200_EARG;
    cudaError_t e = launch_fp32x2_probe(blocks, threads, iters, sink, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? PRRTC_B200_OK : cuda_fail(e);
}

}  // extern "C"
