// kernels.h -- host-side launch interface between the C-ABI layer (capi.cu) and
// the kernel translation units.  Internal: not part of the public C-ABI.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace prrtc {

// Environment point cloud in a hashed uniform grid: points sorted by bucket,
// bucket b holding points [start[b], start[b+1]).  Cell (ix,iy,iz) =
// floor(p / cell) hashes to a bucket with the spatial hash of Teschner et al.
// (2003), three large primes XORed; cells that share a bucket only cost extra
// distance tests.  Every point is a sphere of radius r_env.
struct PcView {
    const float4* pts;  // [n] (x, y, z, unused)
    const int* start;   // [mask + 2]
    int n;              // 0 = no cloud
    int mask;           // buckets - 1 (power of two)
    float inv_cell;
    float r_env;
};


// Sources of the packed scene of every problem in a launch.  Robot tables are
// shared; world tables are either shared (count pointers null, n = max) or
// batched [B, max, feat] with per-problem device counts.
struct PackSrc {
    const float* twists; const float* ptf; const int32_t* parent; const int32_t* act;
    const float* mmul; const float* moff; const int32_t* mact; const int32_t* topo_inv; int J;
    const int32_t* sli; const float* sloc; const float* srad; int S;
    const int32_t* cli; const float* cloc; const float* crad; const int32_t* foff; int K;
    const int32_t* cpairs; const int32_t* cranges; int Q;
    const float* ws; int ws_max; const int32_t* ws_cnt;
    const float* wc; int wc_max; const int32_t* wc_cnt;
    const float* wb; int wb_max; const int32_t* wb_cnt;
    const float* wh; int wh_max; const int32_t* wh_cnt;
    const int32_t* sp; int sp_max; const int32_t* sp_cnt;
    int mode;
    float margin;
    int dim;
    int has_cloud;  // an environment point cloud is checked too (enables collision checking)
};

// Capacity in bytes of one problem's blob (multiple of 256).
size_t blob_stride(const PackSrc& s);
cudaError_t launch_pack(const PackSrc& s, int batch, unsigned char* blobs, size_t stride, cudaStream_t st);

struct PlanLaunch {
    // outputs ([B,...] contiguous, reference layout)
    float* tree_a; float* tree_b; int32_t* par_a; int32_t* par_b;
    int32_t* sizes; int32_t* completed; int32_t* iter_count; int32_t* connection; int32_t* solved;
    float* ktime;
    // inputs
    const float* starts; const float* goals; int num_goals; const int32_t* goal_counts;
    const float* lo; const float* hi;
    const int32_t* pairs; size_t pairs_stride;   // explicit self pairs (elements of int2 per problem)
    const int32_t* order;
    const int32_t* caps;                         // per-problem tree capacity (<= N) or null
    // workspace
    unsigned char* blobs; size_t blob_stride; int blob_cap;
    float* radii;                      // [B][2][N]
    unsigned long long* tstamp;        // [B][2]
    int32_t* queue;                    // [3]: head, error, tail-join ticket
    // shape
    int B, E, N, dim, J, S, K, Q;
    // attributes
    int max_iter, balance_mode, dd, granularity;
    float step, tree_ratio, dd_alpha, dd_radius, dd_min_radius, edge_res;
    // tuning
    int threads, cw, resident;
    int persistent;
    int tail_join;                     // persistent form: idle CTAs join running problems as extra explorers
    int wait_polls;                    // polls of the scene-staging wait before it gives up (0: default, <0: none)
    int ctas_per_sm;                   // persistent form: > 0 caps CTAs per SM and sizes the shared-memory carve-out
    cudaEvent_t explore_events[2];     // optional, recorded right before / after the planner kernel
    unsigned long long* stats;         // optional device counters (kStat*)
    PcView pc;                         // environment point cloud shared by every problem (pc.n = 0: none)
};

// Identity of the calling thread's current CUDA context (cuCtxGetId, else the
// handle), 0 when unknown (capi.cu).
unsigned long long current_context_key();

size_t plan_workspace_bytes(int B, int N, size_t blob_stride);
void plan_carve_workspace(PlanLaunch& L, void* ws, size_t blob_stride);
cudaError_t launch_plan(PlanLaunch& L, cudaStream_t st);
cudaError_t launch_extract_paths(int B, int dim, int N, const float* ta, const float* tb, const int32_t* pa,
                                 const int32_t* pb, const int32_t* conn, const int32_t* solved, int max_len,
                                 float* paths, int32_t* lengths, float* costs, cudaStream_t st);

// Columns of the [B,16] int32 result block.
enum : int {
    kBlkSizeA = 0, kBlkSizeB = 1, kBlkCompletedA = 2, kBlkCompletedB = 3, kBlkIterations = 4, kBlkConn = 5,
    kBlkSolved = 8, kBlkKernelMs = 9, kBlkLength = 10, kBlkCost = 11, kBlkOffset = 12
};

// Per-problem planner outputs that the result block gathers.
struct ResultSrc {
    const int32_t* sizes;      // [B,2]
    const int32_t* completed;  // [B,2]
    const int32_t* iterations; // [B]
    const int32_t* conn;       // [B,3]
    const int32_t* solved;     // [B]
    const float* kernel_ms;    // [B]
    const int32_t* lengths;    // [B]
    const float* costs;        // [B]
};
cudaError_t launch_result_block(int B, int dim, int max_len, const ResultSrc& R, int32_t* block,
                                const float* paths, float* packed, long long packed_cap, cudaStream_t st);

// primitives.cu
cudaError_t launch_nearest(const float* tree, int dim, int N, const int32_t* tree_size, const float* q, int batch,
                           int32_t* idx, float* dist, unsigned long long* keys, cudaStream_t st);
cudaError_t launch_extend(const float* tree, int dim, int N, const int32_t* nearest, const float* samples,
                          int batch, const float* step, float* out, int32_t* parents, int32_t* valid,
                          cudaStream_t st);
cudaError_t launch_iteration(float* ta, float* tb, int32_t* pa, int32_t* pb, int dim, int N, const float* samples,
                             int batch, int32_t* sizes, int32_t* completed, const float* step, int32_t* new_cfg,
                             int32_t* new_par, int32_t* valid, int32_t* solved, cudaStream_t st);
cudaError_t launch_check(const unsigned char* blob, int blob_cap, const int32_t* pairs, int J, int S, int K,
                         int Q, int dim, const float* configs, int n, int full_sweep, int32_t* verdicts,
                         cudaStream_t st, const PcView* pc = nullptr);

// pointcloud.cu
size_t pc_workspace_bytes(int n_points, int n_buckets);
// Hash n_points points [n,3] into n_buckets (power of two) buckets of cells of
// edge `cell`; fills `view` with pointers into the workspace.
cudaError_t launch_pc_build(const float* points, int n_points, float cell, float r_env, int n_buckets, void* ws,
                            PcView* view, cudaStream_t st);
cudaError_t launch_edge_reduce(const int32_t* verdicts, int n_edges, int G, int32_t* free_flags, cudaStream_t st);
struct FkTables {
    const float* twists; const float* ptf; const int32_t* parent; const int32_t* act;
    const float* mmul; const float* moff; const int32_t* mact; const int32_t* topo_inv; int J;
};
cudaError_t launch_fk(const FkTables& t, int dim, const float* configs, int n, float* frames, cudaStream_t st);
cudaError_t launch_halton(int explorer, int n, int dim, const float* lo, const float* hi, float* out,
                          cudaStream_t st);
cudaError_t launch_choose_tree(int mode, int n, const int32_t* sizes, const int32_t* local_iter,
                               const int32_t* vamp_in, int nblocks, float tree_ratio, int32_t* tree_out,
                               int32_t* vamp_out, cudaStream_t st);
cudaError_t launch_radius_update(float* radii, const int32_t* idx, const int32_t* op, int n, float alpha, float r0,
                                 float rmin, int sequential, int32_t* err, cudaStream_t st);

// smooth.cu
// Path p uses the scene at blob + p * blob_stride and the self pairs at
// pairs + 2 * p * pairs_stride (strides 0: one scene for every path).
cudaError_t launch_smooth(const unsigned char* blob, size_t blob_stride, const int32_t* pairs, size_t pairs_stride,
                          int J, int S, int dim, const float* wp, int P, int W, float margin, float beta, float w_len,
                          float* cost, float* grad, cudaStream_t st);

cudaError_t launch_fp32_probe(int blocks, int threads, int iters, float* sink, cudaStream_t st);
cudaError_t launch_fp32x2_probe(int blocks, int threads, int iters, float* sink, cudaStream_t st);

int device_sm_count();
size_t device_max_smem();

}  // namespace prrtc
