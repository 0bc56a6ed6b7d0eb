/*
 * prrtc_b200.h -- C-ABI of the B200 (sm_100a) pRRTC planner library.
 *
 * Plain pointers and sizes only: every buffer is DEVICE memory unless stated,
 * every call is asynchronous on the given cudaStream_t (passed as void*), and no
 * call allocates: scratch comes from a caller-provided workspace whose size the
 * matching *_workspace_size() function returns.  Return codes are 0 on success
 * and a negative PRRTC_B200_E* value otherwise (prrtc_b200_error_string()).
 *
 * Each entry point replaces one handler of the reference P-RRAX library
 * (paths relative to the P-RRAX project root):
 *   prrtc_b200_plan              <- PrrtcPlannerImpl / "prrtc_planner"
 *                                   cuda-rrtc/CUDA/prrtc_planner.cu:1069-1396, binding 2063-2117
 *   prrtc_b200_plan_batch        <- PrrtcPlannerBatchCtxImpl / "prrtc_planner_batch_ctx"
 *                                   prrtc_planner.cu:1643-1944, binding 1946-2005, and
 *                                   PrrtcPlannerBatchImpl / "prrtc_planner_batch" (shared world)
 *                                   prrtc_planner.cu:1404-1638, binding 2007-2061
 *   prrtc_b200_nearest_neighbor  <- PrrtcNearestNeighborImpl / "prrtc_nearest_neighbor"
 *                                   cuda-rrtc/CUDA/prrtc_nearest_neighbor.cu:80-141
 *   prrtc_b200_extend            <- PrrtcExtendImpl / "prrtc_extend"
 *   prrtc_b200_iteration         <- PrrtcIterationImpl / "prrtc_iteration" (legacy)
 *                                   cuda-rrtc/CUDA/prrtc_extend.cu:76-140
 *   prrtc_b200_extract_paths     <- _trace_path + cost, cuda-rrtc/jax/prrtc.py:556-640
 *   prrtc_b200_result_block      <- the device_get of every output and the per-result loop,
 *                                   cuda-rrtc/jax/prrtc.py:1399-1434
 *                                   (sizes, flags, paths): one block and one path copy
 *   prrtc_b200_check_configs     <- the collision checkers, prrtc_planner.cu:234-655
 *                                   (exposed as a batched primitive)
 *   prrtc_b200_fk / _halton      <- fk_single call sites (prrtc_planner.cu:509-522) and the
 *                                   Halton sampler (144-157, 747-788), exposed for parity tests
 *   prrtc_b200_choose_tree       <- the planner's tree-side balance rule
 *                                   (prrtc_planner.cu:790-824), exposed for parity tests
 *   prrtc_b200_radius_update     <- prrtc_radius_shrink_atomic / prrtc_radius_grow_atomic
 *                                   (prrtc_planner.cu:46-83), exposed for parity tests
 *   prrtc_b200_smooth_cost_grad  <- no reference counterpart: adjoint of the smooth
 *                                   collision + length cost for post-plan smoothing
 */
#ifndef PRRTC_B200_H
#define PRRTC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PRRTC_B200_OK 0
#define PRRTC_B200_EARG (-1)        /* invalid argument (shape, range, null pointer) */
#define PRRTC_B200_EWORKSPACE (-2)  /* workspace missing, too small or misaligned */
#define PRRTC_B200_ECUDA (-3)       /* a CUDA runtime call failed (prrtc_b200_last_cuda_error) */
#define PRRTC_B200_EUNSUPPORTED (-4)/* shape outside the supported limits */
#define PRRTC_B200_ETOOLARGE (-5)   /* scene larger than the no-allocation scene buffer */

#define PRRTC_B200_DIM_MAX 16        /* CONFIG_DIM_MAX, prrtc_helpers.cuh:10 */
#define PRRTC_B200_MAX_JOINTS 64     /* PRRTC_MAX_JOINTS, prrtc_planner.cu:31-33 */
#define PRRTC_B200_MAX_LINKS 64      /* PRRTC_MAX_LINKS, prrtc_planner.cu:215-218 */
#define PRRTC_B200_GRANULARITY_MAX 64/* PRRTC_BLOCK_THREADS_MAX, prrtc_planner.cu:43 */

/* Robot model: the 11 FK/sphere buffers and the 6 coarse buffers of the
 * collision_context contract (cuda-rrtc/jax/prrtc.py:397-459, README.md:74-113).
 * Zero counts mean "absent" exactly as zero-sized XLA buffers do. */
typedef struct {
    const float* fk_twists;            /* [n_joints,6]  (v, w) */
    const float* fk_parent_tf;         /* [n_joints,7]  (qw,qx,qy,qz, tx,ty,tz) */
    const int32_t* fk_parent_idx;      /* [n_joints] */
    const int32_t* fk_act_idx;         /* [n_joints] */
    const float* fk_mimic_mul;         /* [n_joints] */
    const float* fk_mimic_off;         /* [n_joints] */
    const int32_t* fk_mimic_act_idx;   /* [n_joints] */
    const int32_t* fk_topo_inv;        /* [n_joints] */
    int32_t n_joints;
    const int32_t* sphere_link_idx;    /* [n_spheres] */
    const float* sphere_local;         /* [n_spheres,3] */
    const float* sphere_radius;        /* [n_spheres] */
    int32_t n_spheres;
    const int32_t* coarse_sphere_link_idx; /* [n_coarse] */
    const float* coarse_sphere_local;  /* [n_coarse,3] */
    const float* coarse_sphere_radius; /* [n_coarse] */
    const int32_t* fine_link_offsets;  /* [n_coarse+1] */
    int32_t n_coarse;
    const int32_t* coarse_self_pairs;  /* [n_coarse_self_pairs,2] */
    const int32_t* self_pair_ranges;   /* [n_coarse_self_pairs,2] */
    int32_t n_coarse_self_pairs;
} prrtc_robot_t;

/* World geometry + self pairs of one problem (prrtc_planner.cu:171-175 row layouts). */
typedef struct {
    const float* world_spheres;     int32_t n_world_spheres;     /* [n,4]  x y z r */
    const float* world_capsules;    int32_t n_world_capsules;    /* [n,7]  p1 p2 r */
    const float* world_boxes;       int32_t n_world_boxes;       /* [n,15] c a1 a2 a3 hl */
    const float* world_halfspaces;  int32_t n_world_halfspaces;  /* [n,6]  n p */
    const int32_t* self_pairs;      int32_t n_self_pairs;        /* [n,2] */
} prrtc_world_t;

/* The 26 arguments of "prrtc_planner", in binding order. */
typedef struct {
    const float* start_config;   /* [dim] */
    const float* goal_configs;   /* [num_goals,dim] */
    int32_t num_goals;
    const float* min_vals;       /* [dim] */
    const float* max_vals;       /* [dim] */
    prrtc_robot_t robot;
    prrtc_world_t world;
} prrtc_inputs_t;

/* The 10 results of "prrtc_planner" (single) or of the batch targets ([B,...]). */
typedef struct {
    float* tree_a_configs;       /* [dim,max_nodes]            / [B,dim,max_nodes] */
    float* tree_b_configs;
    int32_t* tree_a_parents;     /* [max_nodes]                / [B,max_nodes] */
    int32_t* tree_b_parents;
    int32_t* tree_sizes;         /* [2]                        / [B,2] */
    int32_t* completed;          /* [2]                        / [B,2] */
    int32_t* iter_count;         /* [1]                        / [B,1] */
    int32_t* connection_info;    /* [3]                        / [B,3] */
    int32_t* solved_flag;        /* [1]  1 solved, 0, -1 failed / [B,1]; -2: stopped because a
                                    device-side wait ran out (see prrtc_tuning_t) */
    float* kernel_time_ms;       /* [1]                        / [B]  device-clock solve time */
} prrtc_outputs_t;

/* The 14 attributes of "prrtc_planner" (prrtc_planner.cu:2103-2116). */
typedef struct {
    int32_t max_iterations;
    float step_size;
    int32_t num_new_samples;     /* explorers per problem */
    int32_t balance_mode;
    float tree_ratio;
    int32_t dynamic_domain;
    float dd_alpha;
    float dd_radius;
    float dd_min_radius;
    int32_t dim;
    int32_t max_nodes;
    int32_t granularity;         /* waypoints per edge (power of two <= 64) */
    int32_t collision_mode;      /* 0 binary, 1 differentiable, 2 binary_coarse, 3 binary_coarse_coop */
    float collision_margin;
} prrtc_attrs_t;

/* Environment point cloud hashed into a uniform grid on the device by
 * prrtc_b200_point_cloud_build (views into that call's workspace, which must
 * outlive every use).  Every point is a sphere of radius r_env; a robot sphere
 * of radius r centred at c hits point p when |c - p| <= r + r_env (the
 * point-cloud validation of cuda-rrtc/jax/prrtc_robogpu.py:183-191, there on
 * RT cores through an external OptiX library).  Points and sphere centres with
 * a coordinate beyond +-1e4 m are ignored; a robot sphere whose bounding box
 * spans more than 512 grid cells counts as a hit. */
typedef struct {
    const float* points;          /* [n_points,4] device, bucket-sorted (x, y, z, unused) */
    const int32_t* bucket_start;  /* [n_buckets+1] device */
    int32_t n_points;
    int32_t n_buckets;            /* power of two */
    float cell;                   /* grid cell edge (m) */
    float r_env;
} prrtc_point_cloud_t;

/* Extensions (all-zero = defaults). */
typedef struct {
    float edge_resolution;       /* >0: an edge gets max(granularity, ceil(len/res)) waypoints */
    int32_t threads_per_explorer;/* threads of one explorer (one explorer per CTA): 32, 64, 128
                                    or 256 (default 128) */
    int32_t waypoint_chunk;      /* waypoints of an edge checked per CTA pass: 8, 16, 32 or 64
                                    (default 16) */
    int32_t resident_ctas;       /* batched planner grid (default: all resident CTAs) */
    uint64_t* stats;             /* optional device counters [4], accumulated: edges checked,
                                    configurations checked, FP32 flops of the collision work
                                    executed, nearest-neighbour nodes scanned */
    const prrtc_point_cloud_t* point_cloud; /* optional environment point cloud checked by the
                                    planner on top of the world geometry (shared by every
                                    problem of a batch) */
    int32_t tail_explorers;      /* batched planner: once every explorer slot has been taken,
                                    idle CTAs join problems still running as extra explorers
                                    (own Halton sequences); 0 = on (default), -1 = off, so
                                    every problem keeps exactly num_new_samples explorers */
    int32_t staging_wait_polls;  /* polls of each CTA's scene-staging wait before it gives up, after
                                    which the planner stops with solved_flag -2 on every open
                                    problem: 0 = default (about 4 million), > 0 = that many,
                                    < 0 = none (the wait gives up at once: tests the failure
                                    path without a fault) */
    int32_t ctas_per_sm;         /* batched planner: > 0 = at most that many CTAs per SM, with the
                                    shared-memory carve-out that just holds them, so the rest of
                                    the SM's unified L1 / shared memory serves as L1 for the
                                    trees, radii and scenes; 0 = as many as fit (default) */
    void* explore_events[2];     /* optional cudaEvent_t pair recorded on the stream right before
                                    and right after the planner kernel itself (not the fill,
                                    pack, init and finalize kernels around it), for timing that
                                    kernel alone; recorded as external event nodes when the
                                    call is captured into a CUDA graph.  NULL = none */
} prrtc_tuning_t;

size_t prrtc_b200_plan_workspace_size(const prrtc_inputs_t* in, const prrtc_attrs_t* attrs,
                                      const prrtc_tuning_t* tuning);
/* One planning problem.  Initialises the outputs (unused tree slots become NaN,
 * unused parents -1), packs the scene, runs the planner kernel and writes the
 * device-clock solve time.  Never blocks the host. */
int prrtc_b200_plan(const prrtc_inputs_t* in, const prrtc_outputs_t* out,
                    const prrtc_attrs_t* attrs, const prrtc_tuning_t* tuning,
                    void* workspace, size_t workspace_bytes, void* stream);

/* Batched planning: the arguments of "prrtc_planner_batch_ctx".  World tensors
 * are padded [B, max_n, feat] with per-problem counts [B] on the device; when a
 * count pointer is NULL every problem uses max_n rows of the unbatched world
 * ("prrtc_planner_batch").  goal_counts (optional, [B]) lets problems use fewer
 * than num_goals goals; problem_order (optional, [B]) is the order in which the
 * persistent planner starts problems (longest first balances uneven batches). */
typedef struct {
    int32_t batch;
    const float* start_configs;      /* [B,dim] */
    const float* goal_configs;       /* [B,num_goals,dim] */
    int32_t num_goals;
    const int32_t* goal_counts;      /* [B] or NULL */
    const float* min_vals;           /* [dim] */
    const float* max_vals;           /* [dim] */
    prrtc_robot_t robot;
    const float* world_spheres;      int32_t max_world_spheres;     const int32_t* world_spheres_count;
    const float* world_capsules;     int32_t max_world_capsules;    const int32_t* world_capsules_count;
    const float* world_boxes;        int32_t max_world_boxes;       const int32_t* world_boxes_count;
    const float* world_halfspaces;   int32_t max_world_halfspaces;  const int32_t* world_halfspaces_count;
    const int32_t* self_pairs;       int32_t max_self_pairs;        const int32_t* self_pairs_count;
    const int32_t* problem_order;    /* [B] or NULL */
    const int32_t* problem_capacity; /* [B] or NULL: each problem's tree capacity (clamped to
                                        [1, max_nodes]); its tree overflows (solved_flag -1)
                                        there, while the outputs keep the max_nodes row stride.
                                        Lets problems of different capacity share one launch. */
} prrtc_batch_inputs_t;

size_t prrtc_b200_plan_batch_workspace_size(const prrtc_batch_inputs_t* in, const prrtc_attrs_t* attrs,
                                            const prrtc_tuning_t* tuning);
/* Persistent batched planner: one launch, a per-problem work queue of explorer
 * slots, CTAs pop slots until the queue is empty. */
int prrtc_b200_plan_batch(const prrtc_batch_inputs_t* in, const prrtc_outputs_t* out,
                          const prrtc_attrs_t* attrs, const prrtc_tuning_t* tuning,
                          void* workspace, size_t workspace_bytes, void* stream);

/* Batched nearest neighbour of `batch` queries [batch,dim] in the SoA tree
 * [dim,max_nodes] over its first *tree_size nodes (read on the device, clamped
 * to [1,max_nodes]).  Ties go to the lowest index.  dists are Euclidean. */
size_t prrtc_b200_nearest_neighbor_workspace_size(int32_t batch);
int prrtc_b200_nearest_neighbor(const float* tree_configs, int32_t dim, int32_t max_nodes,
                                const int32_t* tree_size, const float* queries, int32_t batch,
                                int32_t* indices, float* dists,
                                void* workspace, size_t workspace_bytes, void* stream);

/* Step-limited extend (prrtc_extend.cu:14-73): new = near + (sample-near)*min(1, step/|.|). */
int prrtc_b200_extend(const float* tree_configs, int32_t dim, int32_t max_nodes,
                      const int32_t* nearest_indices, const float* samples, int32_t batch,
                      const float* step_size, float* new_configs, int32_t* parent_indices,
                      int32_t* valid_flags, void* stream);

/* Legacy single iteration ("prrtc_iteration", prrtc_iteration.cu:180-277; no
 * collision checking): resets tree_sizes = completed = {1,1} and solved_flag =
 * 0, then extends the smaller tree toward every sample (equal sizes: tree =
 * sample & 1) from its nearest completed node, appending the candidates to the
 * trees in place.  new_configs holds the float bits of each candidate.  The
 * tree choice and slot order are those of the reference's schedule in which
 * every sample reads the sizes before any inserts (slot 1 + sample/2). */
int prrtc_b200_iteration(float* tree_a_configs, float* tree_b_configs, int32_t* tree_a_parents,
                         int32_t* tree_b_parents, int32_t dim, int32_t max_nodes, const float* samples,
                         int32_t batch, int32_t* tree_sizes, int32_t* completed, const float* step_size,
                         int32_t* new_configs, int32_t* new_parents, int32_t* valid_flags,
                         int32_t* solved_flag, void* stream);

/* Collision verdicts of n configurations [n,dim] (1 = in collision) with the
 * checker of `collision_mode`.  full_sweep != 0 evaluates every pair with no
 * early exit (same verdicts; used to measure the kernel's FP32 throughput);
 * the flat checkers (modes 0 and 1) sweep fully either way, which measured
 * faster than their early exit, and the coarse-gated ones (2, 3) exit early
 * unless full_sweep is set. */
size_t prrtc_b200_check_configs_workspace_size(const prrtc_robot_t* robot, const prrtc_world_t* world);
int prrtc_b200_check_configs(const prrtc_robot_t* robot, const prrtc_world_t* world, int32_t dim,
                             const float* configs, int32_t n, int32_t collision_mode,
                             float collision_margin, int32_t full_sweep, int32_t* verdicts,
                             void* workspace, size_t workspace_bytes, void* stream);

/* Same verdicts as prrtc_b200_check_configs, with no workspace and no
 * allocation of any kind.  No counterpart in the reference: it serves callers
 * that cannot call cudaMalloc or provide scratch memory (work issued while
 * another library captures the stream into a CUDA graph, real-time loops that
 * forbid allocation after start-up, plug-in hosts without access to an
 * allocator).  The packed scene goes to a file-scope device array of
 * PRRTC_B200_NOALLOC_SCENE_MAX bytes that every GPU loading the library holds
 * until process exit; a larger scene returns PRRTC_B200_ETOOLARGE before any
 * CUDA call.  The first call on a device resolves the array's device address
 * (cudaGetSymbolAddress) with that device current, so make that first call
 * before any stream capture; the address is kept per device and CUDA context,
 * and a call in another context (a different driver context made current, or
 * the primary context re-created after cudaDeviceReset) resolves it again, so
 * that first call in a new context also belongs before any capture.  Every call
 * rewrites the header and every section of the array that the checker reads,
 * so nothing needs clearing between calls; calls that overlap on the GPU (other
 * streams or host threads on the same device) share the array and race --
 * serialise them. */
#define PRRTC_B200_NOALLOC_SCENE_MAX (256 * 1024)
int prrtc_b200_check_configs_noalloc(const prrtc_robot_t* robot, const prrtc_world_t* world, int32_t dim,
                                     const float* configs, int32_t n, int32_t collision_mode,
                                     float collision_margin, int32_t full_sweep, int32_t* verdicts,
                                     void* stream);

/* Point cloud [n_points,3] (device) -> hashed grid.  cell >= 1e-3 m (a cell
 * about the largest robot sphere radius + r_env keeps queries to <= 27 cells);
 * n_buckets a power of two <= 2^24, or 0 for the next power of two >= n_points
 * (at least 1024). */
size_t prrtc_b200_point_cloud_workspace_size(int32_t n_points, int32_t n_buckets);
int prrtc_b200_point_cloud_build(const float* points, int32_t n_points, float cell, float r_env,
                                 int32_t n_buckets, void* workspace, size_t workspace_bytes,
                                 prrtc_point_cloud_t* cloud, void* stream);

/* Edge validation (RoboGPUCollisionChecker.check_edges_collision_free, called at
 * cuda-rrtc/jax/prrtc_robogpu.py:183-191): edges [n_edges,granularity,dim] of
 * waypoints, free_flags [n_edges] = 1 when no waypoint collides with the world
 * geometry, the self pairs or the point cloud (cloud may be NULL). */
size_t prrtc_b200_check_edges_workspace_size(const prrtc_robot_t* robot, const prrtc_world_t* world,
                                             int32_t n_edges, int32_t granularity);
int prrtc_b200_check_edges(const prrtc_robot_t* robot, const prrtc_world_t* world,
                           const prrtc_point_cloud_t* cloud, int32_t dim, const float* edges,
                           int32_t n_edges, int32_t granularity, int32_t collision_mode,
                           float collision_margin, int32_t* free_flags, void* workspace,
                           size_t workspace_bytes, void* stream);

/* Forward kinematics: frames [n,n_joints,12] (row-major R then t) in output
 * frame order. */
int prrtc_b200_fk(const prrtc_robot_t* robot, int32_t dim, const float* configs, int32_t n,
                  float* frames, void* stream);

/* The first n Halton samples [n,dim] of explorer `explorer`, through the
 * planner's own device sampler. */
int prrtc_b200_halton(int32_t explorer, int32_t n, int32_t dim, const float* min_vals,
                      const float* max_vals, float* samples, void* stream);

/* The planner's tree-side rule (balance_mode 0-3) for n cases: explorer bid of
 * nblocks (one CUDA block each) with tree sizes sizes[2c], sizes[2c+1] and
 * iteration count local_iter[c] chooses tree_out[c*nblocks+bid] (0 = A, 1 = B);
 * vamp_in / vamp_out [n, nblocks] carry an explorer's balance_mode-2 side
 * before and after the choice. */
int prrtc_b200_choose_tree(int32_t balance_mode, int32_t n, const int32_t* sizes,
                           const int32_t* local_iter, const int32_t* vamp_in, int32_t nblocks,
                           float tree_ratio, int32_t* tree_out, int32_t* vamp_out, void* stream);

/* The planner's dynamic-domain radius updates on radii[] (FLT_MAX = unset):
 * update i is op[i] (0 = shrink after a failed extension from node idx[i], 1 = grow
 * after a successful one).  sequential = 0: one thread per update, so updates of
 * one node contend on its compare-and-swap loop; sequential != 0: applied in order.
 * err (optional, device int32): set to 1 if a loop's iteration guard ran out. */
int prrtc_b200_radius_update(float* radii, const int32_t* idx, const int32_t* op, int32_t n,
                             float dd_alpha, float dd_radius, float dd_min_radius,
                             int32_t sequential, int32_t* err, void* stream);

/* Root(A) -> connection -> root(B) paths of B solved problems ([B,...] planner
 * outputs) into paths [B,max_len,dim]; lengths [B] (0 when unsolved, -1 when
 * longer than max_len) and costs [B] (sum of segment norms). */
int prrtc_b200_extract_paths(int32_t batch, int32_t dim, int32_t max_nodes,
                             const float* tree_a_configs, const float* tree_b_configs,
                             const int32_t* tree_a_parents, const int32_t* tree_b_parents,
                             const int32_t* connection_info, const int32_t* solved_flag,
                             int32_t max_len, float* paths, int32_t* lengths, float* costs,
                             void* stream);

/* The scalars of B planner results gathered into one int32 block [B,16] for a
 * single device->host copy: columns 0-1 tree sizes, 2-3 completed flags, 4
 * iterations, 5-7 connection_info, 8 solved_flag, 9 kernel_ms (float bits), 10
 * path length and 11 path cost (float bits, from prrtc_b200_extract_paths), 12
 * the path's first waypoint in packed_paths or -1, 13-15 zero.  With packed_paths
 * (capacity packed_capacity waypoints of dim floats), the solved paths of
 * paths [B,max_len,dim] are also copied back to back, in problem order, into
 * packed_paths; a path past the capacity gets -1 in column 12 and stays only in
 * paths.  packed_paths may be NULL (block only). */
int prrtc_b200_result_block(int32_t batch, int32_t dim, int32_t max_len,
                            const int32_t* sizes, const int32_t* completed, const int32_t* iterations,
                            const int32_t* connection_info, const int32_t* solved_flag,
                            const float* kernel_ms, const int32_t* lengths, const float* costs,
                            const float* paths, int32_t* block, float* packed_paths,
                            int64_t packed_capacity, void* stream);

/* Smooth collision + length cost of P paths of W waypoints [P,W,dim] and its
 * gradient (hand-written adjoint through FK, link transforms recomputed):
 *   cost_p = sum_w sum_pairs softplus_beta(margin - d) + w_len * sum_w |q_{w+1}-q_w|^2
 * grad may be NULL (cost only). */
size_t prrtc_b200_smooth_workspace_size(const prrtc_robot_t* robot, const prrtc_world_t* world);
int prrtc_b200_smooth_cost_grad(const prrtc_robot_t* robot, const prrtc_world_t* world, int32_t dim,
                                const float* waypoints, int32_t n_paths, int32_t n_waypoints,
                                float margin, float beta, float w_len, float* cost, float* grad,
                                void* workspace, size_t workspace_bytes, void* stream);

/* The same cost and gradient for the paths of a batch, path p [W,dim] of
 * waypoints [batch,W,dim] against problem p's own world and self pairs, as
 * prrtc_b200_plan_batch reads them from `in` (robot, batch, the per-problem world
 * tables and counts; the start, goal, order and capacity fields are not used).
 * No reference counterpart (post-plan smoothing of a batch plan's paths). */
size_t prrtc_b200_smooth_batch_workspace_size(const prrtc_batch_inputs_t* in);
int prrtc_b200_smooth_cost_grad_batch(const prrtc_batch_inputs_t* in, int32_t dim, const float* waypoints,
                                      int32_t n_waypoints, float margin, float beta, float w_len,
                                      float* cost, float* grad, void* workspace, size_t workspace_bytes,
                                      void* stream);

/* Diagnostic: FP32 FFMA throughput probe (blocks x threads, iters x 8 independent
 * FFMA chains per thread); sink receives one value per block so the work is live.
 * Used to measure the FP32 roofline denominator. */
int prrtc_b200_fp32_probe(int32_t blocks, int32_t threads, int32_t iters, float* sink, void* stream);

/* Diagnostic: the same probe with packed FP32 FMAs (fma.rn.f32x2: iters x 8 chains
 * of two lanes per thread, twice the flops of prrtc_b200_fp32_probe per iteration).
 * The larger of the two rates is the FP32 roofline denominator. */
int prrtc_b200_fp32x2_probe(int32_t blocks, int32_t threads, int32_t iters, float* sink, void* stream);

const char* prrtc_b200_error_string(int code);
int prrtc_b200_last_cuda_error(void);
int prrtc_b200_version(void);

#ifdef __cplusplus
}
#endif
#endif
