/*
 * prrtc_oracle.h -- CPU restatement of the pRRTC hot path (TEST INFRASTRUCTURE).
 *
 * This library is the parity oracle for the B200 planner.  Only the test suite,
 * the smoke check and the CPU-baseline leg of the benchmark load it; the product
 * library (prrtc_b200) never links, calls or falls back to it.
 *
 * What it restates (reference paths relative to the P-RRAX project root):
 *   - Halton sampling + per-explorer prime shuffle   cuda-rrtc/CUDA/prrtc_planner.cu:144-157, 747-764, 784-788
 *   - tree-side balance modes                        prrtc_planner.cu:790-824
 *   - nearest neighbour (ties -> lowest index)       prrtc_planner.cu:841-862, 949-973
 *   - extend, dynamic domain                         prrtc_planner.cu:46-83, 864-881, 911-947
 *   - edge waypoints t=(k+1)/G                       prrtc_planner.cu:884-908, 996-1016
 *   - insert / connect / termination                 prrtc_planner.cu:925-1062
 *   - binary / differentiable / coarse checkers      prrtc_planner.cu:234-655
 *   - host-driven RRT-Connect (CPU path)             cuda-rrtc/jax/prrtc_robogpu.py:36-298
 *   - path tracing and cost                          cuda-rrtc/jax/prrtc.py:566, 588-640
 *
 * Forward kinematics and the primitive distances come from PyRoFFI in the
 * reference (fk_single, sphere_*_dist, colldist_from_sdf), whose source is not
 * available.  They are restated here from the geometry (product of exponentials,
 * exact point-primitive distances); parity at that boundary is UNPINNED.
 * Halton / nearest-neighbour / extend arithmetic is pinned against the
 * reference's own device code compiled from its sources (oracle/ref).
 *
 * Floating point: compiled with -ffp-contract=off.  Every place where nvcc
 * contracts the reference expression a + b*c into one FMA is written here as an
 * explicit fmaf(), so the float results are bit-identical to the device code.
 */
#ifndef PRRTC_ORACLE_H
#define PRRTC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_DIM_MAX 16
#define ORC_MAX_JOINTS 64
#define ORC_MAX_LINKS 64

/* A collision scene in the reference's collision_context layout
 * (cuda-rrtc/jax/prrtc.py:397-459, README.md:74-113).  Zero counts mean "absent". */
typedef struct {
    int dim;
    int n_joints;
    const float* twists;          /* [J,6]  (v, w) */
    const float* parent_tf;       /* [J,7]  (qw,qx,qy,qz, tx,ty,tz) */
    const int* parent_idx;        /* [J]    topological order, -1 = root */
    const int* act_idx;           /* [J] */
    const float* mimic_mul;       /* [J] */
    const float* mimic_off;       /* [J] */
    const int* mimic_act_idx;     /* [J] */
    const int* topo_inv;          /* [J]    output frame k = sorted joint topo_inv[k] */
    int n_spheres;
    const int* sphere_link_idx;   /* [S] */
    const float* sphere_local;    /* [S,3] */
    const float* sphere_radius;   /* [S] */
    int n_ws; const float* world_spheres;     /* [Ns,4]  x y z r */
    int n_wc; const float* world_capsules;    /* [Nc,7]  p1 p2 r */
    int n_wb; const float* world_boxes;       /* [Nb,15] c a1 a2 a3 hl */
    int n_wh; const float* world_halfspaces;  /* [Nh,6]  n p */
    int n_self; const int* self_pairs;        /* [P,2] */
    int n_coarse;
    const int* coarse_link;       /* [K] */
    const float* coarse_local;    /* [K,3] */
    const float* coarse_radius;   /* [K] */
    const int* fine_offsets;      /* [K+1] */
    int n_coarse_self;
    const int* coarse_self_pairs; /* [Q,2] */
    const int* self_pair_ranges;  /* [Q,2] */
    /* environment point cloud (the point-cloud edge validation of
     * prrtc_robogpu.py:183-191): every point is a sphere of radius r_env,
     * checked against every fine robot sphere by brute force */
    int n_points;
    const float* points;          /* [M,3] */
    float r_env;
} OrcScene;

/* Planner attributes: the 14 FFI attributes of prrtc_planner (prrtc_planner.cu:2103-2116)
 * plus edge_resolution (0 = exactly `granularity` waypoints per edge, as the reference). */
typedef struct {
    int max_iterations;
    float step_size;
    int num_new_samples;
    int balance_mode;
    float tree_ratio;
    int dynamic_domain;
    float dd_alpha;
    float dd_radius;
    float dd_min_radius;
    int dim;
    int max_nodes;
    int granularity;
    int collision_mode;
    float collision_margin;
    float edge_resolution;
} OrcPlanParams;

/* ---- sampling (prrtc_planner.cu:144-157, 747-764, 784-788) ---- */
float orc_halton_next(int base, int* state);
void orc_prime_order(int explorer, int out16[16]);
void orc_halton_sample(const int prime_order[16], int* states, int dim,
                       const float* lo, const float* hi, float* out);

/* ---- nearest neighbour: argmin over n nodes of SoA tree [dim][max_nodes].
 * NaN (unwritten) slots are skipped; ties go to the lowest index.  Returns the
 * index (or -1 when no node is valid) and writes the squared distance. ---- */
int orc_nearest(const float* tree, int max_nodes, int dim, int n, const float* q, float* dsq_out);
float orc_dist_sq(const float* tree, int max_nodes, int dim, int idx, const float* q);

/* ---- extend (prrtc_planner.cu:864-876) ---- */
void orc_extend(const float* base, const float* sample, int dim, float nd, float step, float* cand);
/* waypoint count for an edge of the given delta (edge_resolution extension) */
int orc_edge_waypoints(const float* delta, int dim, int granularity, float resolution);
/* waypoint k of G: base + ((k+1)/G) * delta, one fma per coordinate */
void orc_waypoint(const float* base, const float* delta, int dim, int k, int G, float* out);

/* Tree-side balance (prrtc_planner.cu:790-824): the tree (0 = A, 1 = B) explorer
 * bid of nblocks extends, given the sizes and its iteration count; *vamp is the
 * explorer's balance_mode-2 side, updated in place. */
int orc_choose_tree(int mode, int local_iter, int bid, int nblocks, int size_a, int size_b, float ratio_thr,
                    int* vamp);

/* Dynamic-domain radius updates (prrtc_planner.cu:46-83), FLT_MAX = unset. */
void orc_radius_shrink(float* radii, int idx, float alpha, float r0, float rmin);
void orc_radius_grow(float* radii, int idx, float alpha);

/* ---- forward kinematics: frames [J][12] = row-major R (9) then t (3), in the
 * output (original) frame order ---- */
void orc_fk_f64(const OrcScene* sc, const double* q, double* frames);
void orc_fk_f32(const OrcScene* sc, const float* q, float* frames);

/* ---- collision ----
 * mode: 0 binary, 1 differentiable (margin), 2 binary_coarse, 3 binary_coarse_coop
 * orc_config_in_collision evaluates the checker selected by `mode` in double
 * precision, literally following the reference control flow. */
int orc_config_in_collision(const OrcScene* sc, const float* q, int mode, float margin);
/* Minimum over every (robot sphere, primitive) and self pair of the signed
 * distance, in double precision.  For the verdict-exclusion band of the tests. */
double orc_min_distance(const OrcScene* sc, const float* q);
/* Edge check: G' waypoints t=(k+1)/G' between base and end (float arithmetic
 * bit-identical to the kernels), each checked by orc_config_in_collision. */
int orc_edge_in_collision(const OrcScene* sc, const float* base, const float* end,
                          int granularity, float resolution, int mode, float margin);
/* Batch verdicts for n configurations [n][dim]. */
void orc_check_configs(const OrcScene* sc, const float* configs, int n, int mode, float margin,
                       int32_t* verdict);

/* ---- sequential pRRTC: explorers run one iteration each in round-robin order.
 * Outputs mirror the 10 planner results (prrtc_planner.cu:2093-2102); trees are
 * SoA [dim][max_nodes], unused slots NaN.  Returns solved_flag (1/0/-1). ---- */
typedef struct {
    float* tree_a; float* tree_b;       /* [dim*max_nodes] */
    int* parents_a; int* parents_b;     /* [max_nodes] */
    int tree_sizes[2];
    int completed[2];
    int iter_count;
    int connection[3];
    int solved;
    int64_t edge_checks;                /* edges checked */
    int64_t config_checks;              /* waypoint configurations checked */
} OrcPlanOut;

int orc_prrtc_plan(const OrcScene* sc, const float* start, const float* goals, int n_goals,
                   const float* lo, const float* hi, const OrcPlanParams* p, OrcPlanOut* out);

/* Trace the path root(A) -> connection -> root(B) (prrtc.py:588-640).
 * Writes up to max_len rows [len][dim]; returns the length (or -1 if too long). */
int orc_trace_path(const float* tree_a, const float* tree_b, const int* pa, const int* pb,
                   int max_nodes, int dim, const int connection[3], float* path, int max_len);
float orc_path_cost(const float* path, int len, int dim);

/* ---- host-driven RRT-Connect (prrtc_robogpu.py:103-298) ----
 * Uniform samples from a splitmix64 stream seeded by `seed`; G waypoints per edge
 * with endpoints included; greedy connect of <= connect_max_steps.  n_threads > 1
 * spreads each iteration's batched edge checks over a thread pool. */
typedef struct {
    int solved;
    int iterations;
    int size_a, size_b;
    int path_len;
    float cost;
    int64_t config_checks;
} OrcHostOut;

int orc_rrtc_host_plan(const OrcScene* sc, const float* start, const float* goal,
                       const float* lo, const float* hi, int max_iterations, float step_size,
                       int num_new_samples, int granularity, int max_nodes, int connect_max_steps,
                       uint64_t seed, int mode, float margin, int n_threads,
                       float* path_out, int max_path, OrcHostOut* out);

/* ---- path re-validation: every edge subdivided into ceil(len/resolution)
 * segments, every point checked with the double-precision binary checker.
 * Returns 1 when the whole path is collision free; writes the smallest signed
 * distance met. ---- */
int orc_validate_path(const OrcScene* sc, const float* path, int len, float resolution,
                      double* min_dist);

/* ---- smoothing cost (double precision) over W waypoints [W][dim]:
 *   sum_w sum_pairs softplus_beta(margin - d)  +  w_len * sum_w |q_{w+1}-q_w|^2
 * with softplus_beta(x) = log(1 + exp(beta x)) / beta. ---- */
double orc_smooth_cost(const OrcScene* sc, const double* waypoints, int W,
                       float margin, float beta, float w_len);

#ifdef __cplusplus
}
#endif
#endif
