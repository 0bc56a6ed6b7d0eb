// pointcloud.cu -- environment point clouds for collision checking: a hashed
// uniform grid built on the device (count, scan, scatter), and the per-edge
// reduction of waypoint verdicts.  The queries themselves run inside the
// collision checker (pc_sphere_hits in prrtc_device.cuh), so the planner, the
// batched checker and the edge checker all see the cloud.
//
// The reference validates edges against a point cloud on RT cores through an
// external OptiX library (cuda-rrtc/jax/prrtc_robogpu.py:183-191, every point a
// sphere of radius r_env); this is the same sphere-vs-point test on the SMs.
#include <cuda_runtime.h>
#include <math.h>

#include "kernels.h"
#include "prrtc_device.cuh"

namespace prrtc {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanPer = 4;
constexpr int kScanTile = kScanThreads * kScanPer;

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct PcLayout {
    size_t start, count, sums, bkt, rnk, pts, bytes;
};

PcLayout pc_layout(int n, int H) {
    PcLayout L;
    const int nblk = (H + kScanTile - 1) / kScanTile;
    size_t o = 0;
    L.start = o; o += align256((size_t)(H + 1) * 4);
    L.count = o; o += align256((size_t)H * 4);
    L.sums = o; o += align256((size_t)nblk * 4);
    L.bkt = o; o += align256((size_t)n * 4);
    L.rnk = o; o += align256((size_t)n * 4);
    L.pts = o; o += align256((size_t)n * 16);
    L.bytes = o;
    return L;
}

__device__ __forceinline__ bool pc_inside(float x, float y, float z) {
    return fabsf(x) < kPcExtent && fabsf(y) < kPcExtent && fabsf(z) < kPcExtent;
}

// Bucket of every point and its rank inside the bucket (atomic ticket).
__global__ void pc_count_kernel(const float* __restrict__ p, int n, float inv, int mask, int* count, int* bkt,
                                int* rnk) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float x = p[(size_t)i * 3], y = p[(size_t)i * 3 + 1], z = p[(size_t)i * 3 + 2];
    if (!pc_inside(x, y, z)) {
        bkt[i] = -1;
        return;
    }
    const unsigned b = pc_hash((int)floorf(x * inv), (int)floorf(y * inv), (int)floorf(z * inv), mask);
    bkt[i] = (int)b;
    rnk[i] = atomicAdd(&count[b], 1);
}

// Exclusive scan of kScanPer values per thread over one CTA of kScanThreads
// (32 warps); returns the CTA total.
__device__ int cta_exclusive_scan(int v[kScanPer]) {
    __shared__ int warp_sums[32];
    __shared__ int total;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int sum = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        const int t = v[k];
        v[k] = sum;
        sum += t;
    }
    int inc = sum;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int o = __shfl_up_sync(0xffffffffu, inc, off);
        if (lane >= off) inc += o;
    }
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const int w = warp_sums[lane];
        int wi = w;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int o = __shfl_up_sync(0xffffffffu, wi, off);
            if (lane >= off) wi += o;
        }
        warp_sums[lane] = wi - w;
        if (lane == 31) total = wi;
    }
    __syncthreads();
    const int base = warp_sums[warp] + inc - sum;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) v[k] += base;
    const int t = total;
    __syncthreads();
    return t;
}

// Pass 1: tile-local exclusive prefix of the bucket counts, tile totals to sums.
__global__ void __launch_bounds__(kScanThreads) pc_scan_tiles_kernel(const int* count, int H, int* start, int* sums) {
    const int i0 = blockIdx.x * kScanTile + threadIdx.x * kScanPer;
    int v[kScanPer];
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) v[k] = i0 + k < H ? count[i0 + k] : 0;
    const int total = cta_exclusive_scan(v);
#pragma unroll
    for (int k = 0; k < kScanPer; ++k)
        if (i0 + k < H) start[i0 + k] = v[k];
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// Pass 2 (one CTA): exclusive prefix of the tile totals, in chunks of one CTA
// tile; start[H] = number of points kept.
__global__ void __launch_bounds__(kScanThreads) pc_scan_sums_kernel(int* sums, int nblk, int* start, int H) {
    int carry = 0;
    for (int c0 = 0; c0 < nblk; c0 += kScanTile) {
        const int i0 = c0 + threadIdx.x * kScanPer;
        int v[kScanPer];
#pragma unroll
        for (int k = 0; k < kScanPer; ++k) v[k] = i0 + k < nblk ? sums[i0 + k] : 0;
        const int total = cta_exclusive_scan(v);
#pragma unroll
        for (int k = 0; k < kScanPer; ++k)
            if (i0 + k < nblk) sums[i0 + k] = v[k] + carry;
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) start[H] = carry;
}

// Pass 3: add each tile's offset.
__global__ void pc_scan_add_kernel(int* start, int H, const int* sums) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < H) start[i] += sums[i / kScanTile];
}

__global__ void pc_scatter_kernel(const float* __restrict__ p, int n, const int* bkt, const int* rnk,
                                  const int* start, float4* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int b = bkt[i];
    if (b < 0) return;
    out[start[b] + rnk[i]] = make_float4(p[(size_t)i * 3], p[(size_t)i * 3 + 1], p[(size_t)i * 3 + 2], 0.0f);
}

// free[e] = 1 when none of the G waypoint verdicts of edge e is a hit.
__global__ void edge_reduce_kernel(const int32_t* v, int n_edges, int G, int32_t* free_flags) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_edges) return;
    int any = 0;
    for (int k = 0; k < G; ++k) any |= v[(size_t)e * G + k];
    free_flags[e] = any ? 0 : 1;
}

}  // namespace

size_t pc_workspace_bytes(int n_points, int n_buckets) { return pc_layout(n_points, n_buckets).bytes; }

cudaError_t launch_pc_build(const float* points, int n, float cell, float r_env, int H, void* ws, PcView* view,
                            cudaStream_t st) {
    const PcLayout L = pc_layout(n, H);
    unsigned char* w = static_cast<unsigned char*>(ws);
    int* start = reinterpret_cast<int*>(w + L.start);
    int* count = reinterpret_cast<int*>(w + L.count);
    int* sums = reinterpret_cast<int*>(w + L.sums);
    int* bkt = reinterpret_cast<int*>(w + L.bkt);
    int* rnk = reinterpret_cast<int*>(w + L.rnk);
    float4* pts = reinterpret_cast<float4*>(w + L.pts);
    const float inv = 1.0f / cell;
    const int nblk = (H + kScanTile - 1) / kScanTile;
    cudaError_t e = cudaMemsetAsync(count, 0, (size_t)H * 4, st);
    if (e != cudaSuccess) return e;
    if (n > 0) pc_count_kernel<<<(n + 255) / 256, 256, 0, st>>>(points, n, inv, H - 1, count, bkt, rnk);
    pc_scan_tiles_kernel<<<nblk, kScanThreads, 0, st>>>(count, H, start, sums);
    pc_scan_sums_kernel<<<1, kScanThreads, 0, st>>>(sums, nblk, start, H);
    pc_scan_add_kernel<<<(H + 255) / 256, 256, 0, st>>>(start, H, sums);
    if (n > 0) pc_scatter_kernel<<<(n + 255) / 256, 256, 0, st>>>(points, n, bkt, rnk, start, pts);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    view->pts = pts;
    view->start = start;
    view->n = n;
    view->mask = H - 1;
    view->inv_cell = inv;
    view->r_env = r_env;
    return cudaSuccess;
}

cudaError_t launch_edge_reduce(const int32_t* verdicts, int n_edges, int G, int32_t* free_flags, cudaStream_t st) {
    if (n_edges <= 0) return cudaSuccess;
    edge_reduce_kernel<<<(n_edges + 255) / 256, 256, 0, st>>>(verdicts, n_edges, G, free_flags);
    return cudaGetLastError();
}

}  // namespace prrtc
