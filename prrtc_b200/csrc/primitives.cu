// primitives.cu -- standalone kernels: batched nearest neighbour, extend, the
// batched FK + collision checker, FK and Halton sampling.  sm_100a.
#include <cuda_runtime.h>
#include <float.h>
#include <limits.h>
#include <math.h>

#include <algorithm>
#include <mutex>

#include "kernels.h"
#include "prrtc_device.cuh"

namespace prrtc {

// ============================================================================ nearest neighbour

// Grid (splits, batch): CTA (s, b) scans its slice of the tree for query b and
// folds its (dsq, index) minimum into keys[b] with a 64-bit atomicMin on
// (float bits << 32 | index) -- for non-negative floats the bit pattern orders
// like the value, so the minimum key is the lexicographic (dsq, lowest index)
// minimum.  NaN slots never win.
__global__ void __launch_bounds__(256) nn_kernel(const float* __restrict__ tree, int dim, int N,
                                                 const int32_t* tree_size, const float* __restrict__ q, int batch,
                                                 int slice, unsigned long long* keys) {
    const int b = blockIdx.y, tid = threadIdx.x, T = blockDim.x;
    int n = tree_size ? tree_size[0] : N;
    n = max(1, min(n, N));
    const int lo = blockIdx.x * slice;
    const int hi = min(n, lo + slice);
    float qr[kDimMax];
#pragma unroll
    for (int d = 0; d < kDimMax; ++d) qr[d] = d < dim ? q[(size_t)b * dim + d] : 0.0f;
    float best = INFINITY;
    int bi = INT_MAX;
    if ((N & 3) == 0 && (lo & 3) == 0 && (reinterpret_cast<uintptr_t>(tree) & 15) == 0) {
        const float4* t4 = reinterpret_cast<const float4*>(tree);
        const size_t row4 = (size_t)(N >> 2);
        const int g0 = lo >> 2, g1 = (hi + 3) >> 2;
        for (int g = g0 + tid; g < g1; g += T) {
            float4 v = __ldg(t4 + g);
            float dx = __fsub_rn(v.x, qr[0]), dy = __fsub_rn(v.y, qr[0]), dz = __fsub_rn(v.z, qr[0]),
                  dw = __fsub_rn(v.w, qr[0]);
            float ax = __fmul_rn(dx, dx), ay = __fmul_rn(dy, dy), az = __fmul_rn(dz, dz), aw = __fmul_rn(dw, dw);
#pragma unroll
            for (int d = 1; d < kDimMax; ++d) {
                if (d < dim) {
                    v = __ldg(t4 + d * row4 + g);
                    dx = __fsub_rn(v.x, qr[d]); dy = __fsub_rn(v.y, qr[d]);
                    dz = __fsub_rn(v.z, qr[d]); dw = __fsub_rn(v.w, qr[d]);
                    ax = __fmaf_rn(dx, dx, ax); ay = __fmaf_rn(dy, dy, ay);
                    az = __fmaf_rn(dz, dz, az); aw = __fmaf_rn(dw, dw, aw);
                }
            }
            const int i0 = g << 2;
            if (ax < best && i0 < hi) { best = ax; bi = i0; }
            if (ay < best && i0 + 1 < hi) { best = ay; bi = i0 + 1; }
            if (az < best && i0 + 2 < hi) { best = az; bi = i0 + 2; }
            if (aw < best && i0 + 3 < hi) { best = aw; bi = i0 + 3; }
        }
    } else {
        for (int i = lo + tid; i < hi; i += T) {
            float dd = __fsub_rn(__ldg(tree + i), qr[0]);
            float acc = __fmul_rn(dd, dd);
            for (int d = 1; d < dim; ++d) {
                dd = __fsub_rn(__ldg(tree + (size_t)d * N + i), qr[d]);
                acc = __fmaf_rn(dd, dd, acc);
            }
            if (acc < best) { best = acc; bi = i; }
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const float od = __shfl_xor_sync(0xffffffffu, best, off);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
        if (od < best || (od == best && oi < bi)) { best = od; bi = oi; }
    }
    if ((tid & 31) == 0 && bi != INT_MAX) {
        const unsigned long long key =
            ((unsigned long long)__float_as_uint(best) << 32) | (unsigned long long)(unsigned)bi;
        atomicMin(&keys[b], key);
    }
}

// Query-tiled form for batches: CTA (s, t) scans its slice once for QT queries
// of tile t.  Each thread keeps one 4-node column of every dimension in
// registers and evaluates all QT queries (held in shared memory) against it, so
// the tree is read once per QT queries instead of once per query.  Arithmetic
// per (node, query) is the same sub/mul/fma sequence as nn_kernel.
template <int QT>
__global__ void __launch_bounds__(256) nn_tiled_kernel(const float* __restrict__ tree, int dim, int N,
                                                       const int32_t* tree_size, const float* __restrict__ q,
                                                       int batch, int slice, unsigned long long* keys) {
    __shared__ __align__(16) float qs[QT][kDimMax];
    const int tid = threadIdx.x, T = blockDim.x;
    const int q0 = blockIdx.y * QT;
    for (int i = tid; i < QT * kDimMax; i += T) {
        const int qq = i / kDimMax, d = i - qq * kDimMax;
        qs[qq][d] = (q0 + qq < batch && d < dim) ? q[(size_t)(q0 + qq) * dim + d] : 0.0f;
    }
    __syncthreads();
    int n = tree_size ? tree_size[0] : N;
    n = max(1, min(n, N));
    const int lo = blockIdx.x * slice;
    const int hi = min(n, lo + slice);
    float best[QT];
    int bi[QT];
#pragma unroll
    for (int k = 0; k < QT; ++k) { best[k] = INFINITY; bi[k] = INT_MAX; }
    const float4* t4 = reinterpret_cast<const float4*>(tree);
    const size_t row4 = (size_t)(N >> 2);
    const int g0 = lo >> 2, g1 = (hi + 3) >> 2;
    for (int g = g0 + tid; g < g1; g += T) {
        float4 v[kDimMax];
#pragma unroll
        for (int d = 0; d < kDimMax; ++d)
            if (d < dim) v[d] = __ldg(t4 + d * row4 + g);
        const int i0 = g << 2;
#pragma unroll
        for (int k = 0; k < QT; ++k) {
            float dx = __fsub_rn(v[0].x, qs[k][0]), dy = __fsub_rn(v[0].y, qs[k][0]), dz = __fsub_rn(v[0].z, qs[k][0]),
                  dw = __fsub_rn(v[0].w, qs[k][0]);
            float ax = __fmul_rn(dx, dx), ay = __fmul_rn(dy, dy), az = __fmul_rn(dz, dz), aw = __fmul_rn(dw, dw);
#pragma unroll
            for (int d = 1; d < kDimMax; ++d) {
                if (d < dim) {
                    const float qd = qs[k][d];
                    dx = __fsub_rn(v[d].x, qd); dy = __fsub_rn(v[d].y, qd);
                    dz = __fsub_rn(v[d].z, qd); dw = __fsub_rn(v[d].w, qd);
                    ax = __fmaf_rn(dx, dx, ax); ay = __fmaf_rn(dy, dy, ay);
                    az = __fmaf_rn(dz, dz, az); aw = __fmaf_rn(dw, dw, aw);
                }
            }
            if (ax < best[k] && i0 < hi) { best[k] = ax; bi[k] = i0; }
            if (ay < best[k] && i0 + 1 < hi) { best[k] = ay; bi[k] = i0 + 1; }
            if (az < best[k] && i0 + 2 < hi) { best[k] = az; bi[k] = i0 + 2; }
            if (aw < best[k] && i0 + 3 < hi) { best[k] = aw; bi[k] = i0 + 3; }
        }
    }
#pragma unroll
    for (int k = 0; k < QT; ++k) {
        float bk = best[k];
        int ik = bi[k];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const float od = __shfl_xor_sync(0xffffffffu, bk, off);
            const int oi = __shfl_xor_sync(0xffffffffu, ik, off);
            if (od < bk || (od == bk && oi < ik)) { bk = od; ik = oi; }
        }
        if ((tid & 31) == 0 && ik != INT_MAX && q0 + k < batch) {
            const unsigned long long key =
                ((unsigned long long)__float_as_uint(bk) << 32) | (unsigned long long)(unsigned)ik;
            atomicMin(&keys[q0 + k], key);
        }
    }
}

__global__ void nn_decode_kernel(const unsigned long long* keys, int batch, int32_t* idx, float* dist) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= batch) return;
    const unsigned long long k = keys[b];
    if (k == ~0ull) {
        idx[b] = 0;
        dist[b] = INFINITY;
        return;
    }
    idx[b] = (int32_t)(k & 0xffffffffull);
    dist[b] = __fsqrt_rn(__uint_as_float((unsigned)(k >> 32)));
}

cudaError_t launch_nearest(const float* tree, int dim, int N, const int32_t* tree_size, const float* q, int batch,
                           int32_t* idx, float* dist, unsigned long long* keys, cudaStream_t st) {
    if (batch <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(keys, 0xFF, (size_t)batch * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    // enough CTAs to cover every SM several times; slices are multiples of 1024 nodes
    const int sms = device_sm_count();
    constexpr int kQT = 8;
    const bool tiled = batch >= 4 && (N & 3) == 0 && (reinterpret_cast<uintptr_t>(tree) & 15) == 0;
    const int tiles = tiled ? (batch + kQT - 1) / kQT : batch;
    int splits = std::max(1, (4 * sms + tiles - 1) / tiles);
    int slice = (N + splits - 1) / splits;
    slice = std::max(1024, (slice + 1023) & ~1023);
    splits = (N + slice - 1) / slice;
    if (tiled)
        nn_tiled_kernel<kQT><<<dim3(splits, tiles), 256, 0, st>>>(tree, dim, N, tree_size, q, batch, slice, keys);
    else
        nn_kernel<<<dim3(splits, batch), 256, 0, st>>>(tree, dim, N, tree_size, q, batch, slice, keys);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    nn_decode_kernel<<<(batch + 255) / 256, 256, 0, st>>>(keys, batch, idx, dist);
    return cudaGetLastError();
}

// ============================================================================ extend

// prrtc_extend.cu:14-73: new = near + (sample - near) * min(1, step / |sample - near|).
__global__ void extend_kernel(const float* tree, int dim, int N, const int32_t* nearest, const float* samples,
                              int batch, const float* step, float* out, int32_t* parents, int32_t* valid) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= batch) return;
    const int ni = nearest[b];
    const float s = step[0];
    float dsq = 0.0f;
    float nv[kDimMax], sv[kDimMax];
    for (int d = 0; d < dim; ++d) {
        nv[d] = tree[(size_t)d * N + ni];
        sv[d] = samples[(size_t)b * dim + d];
        const float df = __fsub_rn(sv[d], nv[d]);
        dsq = d == 0 ? __fmul_rn(df, df) : __fmaf_rn(df, df, dsq);
    }
    const float scale = fminf(1.0f, __fdiv_rn(s, __fsqrt_rn(dsq)));
    for (int d = 0; d < dim; ++d) out[(size_t)b * dim + d] = __fmaf_rn(__fsub_rn(sv[d], nv[d]), scale, nv[d]);
    parents[b] = ni;
    valid[b] = 1;
}

cudaError_t launch_extend(const float* tree, int dim, int N, const int32_t* nearest, const float* samples,
                          int batch, const float* step, float* out, int32_t* parents, int32_t* valid,
                          cudaStream_t st) {
    if (batch <= 0) return cudaSuccess;
    extend_kernel<<<(batch + 127) / 128, 128, 0, st>>>(tree, dim, N, nearest, samples, batch, step, out, parents,
                                                       valid);
    return cudaGetLastError();
}

// ============================================================================ legacy iteration

// prrtc_iteration.cu:21-167 (the "prrtc_iteration" target): every call first
// resets the state to one node per tree, then each sample extends the smaller
// tree (equal sizes: tree = sample & 1) from its nearest node among the
// `completed` ones and appends the step-limited candidate.  The reference reads
// the live sizes and appends with atomics, so its tree choice and slot order
// depend on scheduling; here every sample sees the sizes after the reset and
// the samples of a tree take its slots in sample order -- the schedule in which
// every block reads before any block inserts.  One warp per sample.
__global__ void iteration_kernel(float* ta, float* tb, int32_t* pa, int32_t* pb, int dim, int N,
                                 const float* __restrict__ samples, int batch, int32_t* sizes, int32_t* completed,
                                 const float* step_ptr, int32_t* new_cfg, int32_t* new_par, int32_t* valid,
                                 int32_t* solved) {
    // state after the reset (prrtc_iteration.cu:28-45): sizes = completed = {1, 1}
    const int n0 = (batch + 1) >> 1, n1 = batch >> 1;  // samples per tree under the tie rule
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const int room = max(0, N - 1);
        sizes[0] = completed[0] = 1 + min(n0, room);
        sizes[1] = completed[1] = 1 + min(n1, room);
        solved[0] = 0;
    }
    const int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (b >= batch) return;
    const int t = b & 1;
    float* tree = t == 0 ? ta : tb;
    int32_t* par = t == 0 ? pa : pb;
    const float* q = samples + (size_t)b * dim;
    // nearest among the completed nodes [0, 1): the root
    const int nn = 0;
    float dsq = 0.0f;
    for (int d = 0; d < dim; ++d) {
        const float df = __fsub_rn(tree[(size_t)d * N + nn], q[d]);
        dsq = d == 0 ? __fmul_rn(df, df) : __fmaf_rn(df, df, dsq);
    }
    const float nd = __fsqrt_rn(dsq);
    const float step = step_ptr[0];
    const float scale = nd > 1e-8f ? fminf(1.0f, __fdiv_rn(step, nd)) : 1.0f;
    const int idx = 1 + (b >> 1);  // this sample's slot in tree t
    const bool ok = idx < N;
    for (int d = lane; d < dim; d += 32) {
        const float nv = tree[(size_t)d * N + nn];
        const float c = __fmaf_rn(__fsub_rn(q[d], nv), scale, nv);
        new_cfg[(size_t)b * dim + d] = __float_as_int(c);
        if (ok) tree[(size_t)d * N + idx] = c;
    }
    if (lane == 0) {
        new_par[b] = nn;
        valid[b] = ok ? 1 : 0;
        if (ok) par[idx] = nn;
    }
}

cudaError_t launch_iteration(float* ta, float* tb, int32_t* pa, int32_t* pb, int dim, int N, const float* samples,
                             int batch, int32_t* sizes, int32_t* completed, const float* step, int32_t* new_cfg,
                             int32_t* new_par, int32_t* valid, int32_t* solved, cudaStream_t st) {
    const int blocks = std::max(1, (batch * 32 + 127) / 128);
    iteration_kernel<<<blocks, 128, 0, st>>>(ta, tb, pa, pb, dim, N, samples, batch, sizes, completed, step, new_cfg,
                                             new_par, valid, solved);
    return cudaGetLastError();
}

// ============================================================================ batched collision check

// Persistent over chunks of CW configurations; the scene is bulk-copied into
// shared memory once per CTA.  The wait is bounded: when it runs out, the CTA
// sets bit kBlobStagingTimeout of the blob header's `error` word (global
// memory), lets the copy land (second bounded wait) and reads the scene from
// global memory instead -- the verdicts are the same either way.
#ifndef PRRTC_CHECK_CW
#define PRRTC_CHECK_CW 32       // configurations per CTA pass of the batched checker
#endif
#ifndef PRRTC_CHECK_MINBLOCKS
#define PRRTC_CHECK_MINBLOCKS 4 // resident CTAs per SM the register allocation must allow (shared memory allows 4 at CW 32)
#endif

template <int CW, bool FULL>
__global__ void __launch_bounds__(128, PRRTC_CHECK_MINBLOCKS) check_kernel(const unsigned char* __restrict__ gblob, int blob_cap,
                                                    const int32_t* pairs, int J, int S, int K, int Q, int dim,
                                                    const float* __restrict__ configs, int n, int32_t* verdicts,
                                                    PcView pc) {
    extern __shared__ __align__(128) unsigned char dsm[];
    __shared__ __align__(8) uint64_t mbar;
    const int tid = threadIdx.x;
    const bool staged = blob_cap > 0;
    const CcBufs B = cc_bufs(dsm + (staged ? blob_cap : 0), J, S, K, Q, CW);
    Scene sc;
    if (staged) {
        const int bytes = min(reinterpret_cast<const BlobHeader*>(gblob)->used_bytes, blob_cap);
        if (tid == 0) mbar_init(&mbar);
        __syncthreads();
        uint32_t phase = 0;
        int* err = reinterpret_cast<int*>(const_cast<unsigned char*>(gblob) + offsetof(BlobHeader, error));
        const bool ok = stage_blob(dsm, gblob, bytes, &mbar, phase, err, kBlobStagingTimeout, kWaitLimit);
        sc = scene_view(ok ? dsm : gblob);
    } else {
        sc = scene_view(gblob);
    }
    sc.pairs = reinterpret_cast<const int2*>(pairs);
    sc.pc = pc;
    if (tid == 0) B.hit[0] = B.hit[1] = 0u;
    int par = 0;
    __syncthreads();
    for (int c0 = blockIdx.x * CW; c0 < n; c0 += gridDim.x * CW) {
        const int nw = min(CW, n - c0);
        for (int i = tid; i < nw * dim; i += blockDim.x) {
            const int w = i / dim, d = i - w * dim;
            B.q[w * kDimMax + d] = configs[(size_t)(c0 + w) * dim + d];
        }
        __syncthreads();
        const uint32_t hit = cc_chunk<FULL>(CtaGroup{}, sc, B, nw, false, par);
        for (int w = tid; w < nw; w += blockDim.x) verdicts[c0 + w] = (hit >> w) & 1u;
    }
}

// One candidate pass size of the batched checker: its kernel, dynamic shared
// memory (the scene staged when it fits), and resident CTAs per SM.
struct CheckLaunch {
    int cw = 0, blob_cap = 0, per_sm = 0;
    size_t dyn = 0;
};

// The largest dynamic shared-memory limit set on each check_kernel
// instantiation, per device and CUDA context.  The limit is only raised, never
// lowered, so a call on another host thread cannot shrink it between this
// call's check and its launch, and a call that needs no more than before sets
// nothing (setting an attribute while an earlier launch runs can make the host
// wait for that launch).
struct CheckAttrs {
    unsigned long long ctx = 0ull;  // context key (current_context_key)
    int max_dyn = -1;
};
constexpr int kCheckAttrDevices = 256;
static CheckAttrs g_check_attr[kCheckAttrDevices][6];  // [device][2 * (pass size: CW, CW/2, CW/4) + full]
static std::mutex g_check_attr_mutex;

template <class Kern>
static cudaError_t check_raise_dyn(Kern kern, int slot, size_t dyn) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long ctx = current_context_key();
    std::lock_guard<std::mutex> lock(g_check_attr_mutex);
    CheckAttrs dflt;
    CheckAttrs& c = (dev >= 0 && dev < kCheckAttrDevices && slot >= 0 && slot < 6) ? g_check_attr[dev][slot] : dflt;
    if (!ctx || c.ctx != ctx) {
        c = CheckAttrs{};
        c.ctx = ctx;
    }
    if ((int)dyn > c.max_dyn) {
        if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn)) != cudaSuccess)
            return e;
        c.max_dyn = (int)dyn;
    }
    return cudaSuccess;
}

template <int CW>
static cudaError_t check_option(int full_sweep, int J, int S, int K, int Q, int blob_cap, CheckLaunch& o) {
    const size_t cc = (size_t)cc_smem_bytes(J, S, K, Q, CW);
    size_t dyn = cc + (size_t)blob_cap;
    if (dyn + 64 > device_max_smem()) {
        blob_cap = 0;
        dyn = cc;
    }
    auto kern = full_sweep ? check_kernel<CW, true> : check_kernel<CW, false>;
    constexpr int size_idx = CW == PRRTC_CHECK_CW ? 0 : (2 * CW == PRRTC_CHECK_CW ? 1 : 2);
    cudaError_t e = check_raise_dyn(kern, 2 * size_idx + (full_sweep ? 1 : 0), dyn);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, dyn)) != cudaSuccess) return e;
    o.cw = CW;
    o.blob_cap = blob_cap;
    o.per_sm = per_sm;
    o.dyn = dyn;
    return cudaSuccess;
}

template <int CW>
static void check_go(const CheckLaunch& o, int full_sweep, const unsigned char* blob, const int32_t* pairs, int J,
                     int S, int K, int Q, int dim, const float* configs, int n, int32_t* verdicts, cudaStream_t st,
                     const PcView& cloud) {
    const long long chunks = (n + CW - 1) / CW;
    const long long grid = std::min<long long>(chunks, (long long)std::max(o.per_sm, 1) * device_sm_count());
    auto kern = full_sweep ? check_kernel<CW, true> : check_kernel<CW, false>;
    kern<<<(unsigned)grid, 128, o.dyn, st>>>(blob, o.blob_cap, pairs, J, S, K, Q, dim, configs, n, verdicts, cloud);
}

// Passes of PRRTC_CHECK_CW configurations, unless their buffers leave fewer
// than PRRTC_CHECK_MINBLOCKS CTAs per SM (large robots: the sphere centres and
// link frames of a pass grow with S and J); then half or a quarter as many
// configurations per pass, whichever keeps the most CTAs resident (the larger
// pass on a tie).  The dual arm with 120 spheres and 18 joints fits one CTA
// per SM at 32 configurations per pass, three at 16 and four at 8: 44.0 M
// checks/s at 32, 65.4 M at 8.
cudaError_t launch_check(const unsigned char* blob, int blob_cap, const int32_t* pairs, int J, int S, int K,
                         int Q, int dim, const float* configs, int n, int full_sweep, int32_t* verdicts,
                         cudaStream_t st, const PcView* pc) {
    if (n <= 0) return cudaSuccess;
    const PcView cloud = pc ? *pc : PcView{nullptr, nullptr, 0, 0, 0.0f, 0.0f};
    constexpr int CW = PRRTC_CHECK_CW;
    CheckLaunch best, o;
    cudaError_t e = check_option<CW>(full_sweep, J, S, K, Q, blob_cap, best);
    if (e != cudaSuccess) return e;
    if constexpr (CW / 2 >= 8) {
        if (best.per_sm < PRRTC_CHECK_MINBLOCKS) {
            if ((e = check_option<CW / 2>(full_sweep, J, S, K, Q, blob_cap, o)) != cudaSuccess) return e;
            if (o.per_sm > best.per_sm) best = o;
        }
    }
    if constexpr (CW / 4 >= 8) {
        if (best.per_sm < PRRTC_CHECK_MINBLOCKS) {
            if ((e = check_option<CW / 4>(full_sweep, J, S, K, Q, blob_cap, o)) != cudaSuccess) return e;
            if (o.per_sm > best.per_sm) best = o;
        }
    }
    if constexpr (CW / 2 >= 8) {
        if (best.cw == CW / 2) {
            check_go<CW / 2>(best, full_sweep, blob, pairs, J, S, K, Q, dim, configs, n, verdicts, st, cloud);
            return cudaGetLastError();
        }
    }
    if constexpr (CW / 4 >= 8) {
        if (best.cw == CW / 4) {
            check_go<CW / 4>(best, full_sweep, blob, pairs, J, S, K, Q, dim, configs, n, verdicts, st, cloud);
            return cudaGetLastError();
        }
    }
    check_go<CW>(best, full_sweep, blob, pairs, J, S, K, Q, dim, configs, n, verdicts, st, cloud);
    return cudaGetLastError();
}

// ============================================================================ FK

// One configuration per thread; link frames in thread-local memory (J <= 64),
// written in output frame order (frame k = sorted joint topo_inv[k]).
__global__ void fk_kernel(FkTables t, int dim, const float* configs, int n, float* frames) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int J = t.J;
    float q[kDimMax];
    for (int d = 0; d < dim; ++d) q[d] = configs[(size_t)c * dim + d];
    float W[kMaxJoints * 12];
    for (int j = 0; j < J; ++j) {
        const JointRec jr = make_joint_rec(j, t.ptf, t.twists, t.parent, t.act, t.mmul, t.moff, t.mact, dim);
        joint_local(jr, joint_value(jr, q), &W[j * 12]);
        const int p = jr.idx.x;
        if (p >= 0 && p < j) compose(&W[p * 12], &W[j * 12], &W[j * 12]);
    }
    for (int k = 0; k < J; ++k) {
        int s = t.topo_inv ? t.topo_inv[k] : k;
        if (s < 0 || s >= J) s = k;
        for (int i = 0; i < 12; ++i) frames[((size_t)c * J + k) * 12 + i] = W[s * 12 + i];
    }
}

cudaError_t launch_fk(const FkTables& t, int dim, const float* configs, int n, float* frames, cudaStream_t st) {
    if (n <= 0 || t.J <= 0) return cudaSuccess;
    fk_kernel<<<(n + 127) / 128, 128, 0, st>>>(t, dim, configs, n, frames);
    return cudaGetLastError();
}

// ============================================================================ Halton

__global__ void halton_kernel(int explorer, int n, int dim, const float* lo, const float* hi, float* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int order[16], st[kDimMax];
    prime_order(explorer, order);
    for (int d = 0; d < kDimMax; ++d) st[d] = 1;
    float row[kDimMax];
    for (int i = 0; i < n; ++i) {
        halton_sample(order, st, dim, lo, hi, row);
        for (int d = 0; d < dim; ++d) out[(size_t)i * dim + d] = row[d];
    }
}

cudaError_t launch_halton(int explorer, int n, int dim, const float* lo, const float* hi, float* out,
                          cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    halton_kernel<<<1, 32, 0, st>>>(explorer, n, dim, lo, hi, out);
    return cudaGetLastError();
}

// ============================================================================ planner rules

// Tree-side choice of the planner (choose_tree) for n cases at once: explorer
// bid = blockIdx.x of nblocks = gridDim.x, case c with tree sizes sizes[2c],
// sizes[2c+1], the explorer's iteration count local_iter[c] and its mode-2 side
// vamp_in[c * nblocks + bid]; writes the chosen tree and the updated side.
__global__ void choose_tree_kernel(int mode, int n, const int32_t* sizes, const int32_t* local_iter,
                                   const int32_t* vamp_in, float tree_ratio, int32_t* tree_out, int32_t* vamp_out) {
    const int bid = blockIdx.x, nblocks = gridDim.x;
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
        int vamp = vamp_in[(size_t)c * nblocks + bid];
        const int t = choose_tree(mode, local_iter[c], bid, nblocks, sizes[2 * c], sizes[2 * c + 1], tree_ratio, vamp);
        tree_out[(size_t)c * nblocks + bid] = t;
        vamp_out[(size_t)c * nblocks + bid] = vamp;
    }
}

cudaError_t launch_choose_tree(int mode, int n, const int32_t* sizes, const int32_t* local_iter,
                               const int32_t* vamp_in, int nblocks, float tree_ratio, int32_t* tree_out,
                               int32_t* vamp_out, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    choose_tree_kernel<<<nblocks, 128, 0, st>>>(mode, n, sizes, local_iter, vamp_in, tree_ratio, tree_out, vamp_out);
    return cudaGetLastError();
}

// Dynamic-domain radius updates of the planner (radius_shrink / radius_grow):
// update i is op[i] (0 shrink, 1 grow) on radii[idx[i]].  Concurrent: one
// thread per update, so updates of one index contend on its CAS loop;
// sequential: one thread applies them in order.
__global__ void radius_update_kernel(float* radii, const int32_t* idx, const int32_t* op, int n, float alpha,
                                     float r0, float rmin, int sequential, int32_t* err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (sequential) {
        if (i != 0) return;
        for (int k = 0; k < n; ++k) {
            if (op[k] == 0) radius_shrink(radii, idx[k], alpha, r0, rmin, err);
            else radius_grow(radii, idx[k], alpha, err);
        }
        return;
    }
    if (i >= n) return;
    if (op[i] == 0) radius_shrink(radii, idx[i], alpha, r0, rmin, err);
    else radius_grow(radii, idx[i], alpha, err);
}

cudaError_t launch_radius_update(float* radii, const int32_t* idx, const int32_t* op, int n, float alpha, float r0,
                                 float rmin, int sequential, int32_t* err, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    radius_update_kernel<<<sequential ? 1 : (n + 127) / 128, sequential ? 32 : 128, 0, st>>>(
        radii, idx, op, n, alpha, r0, rmin, sequential, err);
    return cudaGetLastError();
}

// ============================================================================ FP32 probe

// 8 independent FFMA chains per thread: the FP32 pipe stays busy without
// dependency stalls.  2 * 8 * iters flops per thread.
__global__ void fp32_probe_kernel(int iters, float* sink) {
    float a0 = threadIdx.x * 1e-7f, a1 = a0 + 1e-7f, a2 = a0 + 2e-7f, a3 = a0 + 3e-7f;
    float a4 = a0 + 4e-7f, a5 = a0 + 5e-7f, a6 = a0 + 6e-7f, a7 = a0 + 7e-7f;
    const float m = 0.999999f, c = 1e-7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            a0 = fmaf(a0, m, c); a1 = fmaf(a1, m, c); a2 = fmaf(a2, m, c); a3 = fmaf(a3, m, c);
            a4 = fmaf(a4, m, c); a5 = fmaf(a5, m, c); a6 = fmaf(a6, m, c); a7 = fmaf(a7, m, c);
        }
    }
    const float r = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (r == 12345.0f) sink[blockIdx.x] = r;  // never true; keeps the chains live
}

cudaError_t launch_fp32_probe(int blocks, int threads, int iters, float* sink, cudaStream_t st) {
    fp32_probe_kernel<<<blocks, threads, 0, st>>>(iters, sink);
    return cudaGetLastError();
}

// The same with packed FP32 (fma.rn.f32x2, sm_100): 8 independent chains of two
// lanes each per thread, 2 * 2 * 8 * 16 * iters flops per thread.  Measures
// whether one packed instruction delivers two FP32 FMAs per lane per issue
// slot, i.e. which FP32 peak a kernel built from packed FMAs runs against.
__device__ __forceinline__ unsigned long long pack2(float lo, float hi) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}

__global__ void fp32x2_probe_kernel(int iters, float* sink) {
    const float b = threadIdx.x * 1e-7f;
    unsigned long long a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = pack2(b + (2 * k) * 1e-7f, b + (2 * k + 1) * 1e-7f);
    const unsigned long long m = pack2(0.999999f, 0.999999f), c = pack2(1e-7f, 1e-7f);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
#pragma unroll
            for (int k = 0; k < 8; ++k) asm volatile("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(a[k]) : "l"(m), "l"(c));
        }
    }
    float r = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float lo, hi;
        asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a[k]));
        r += lo + hi;
    }
    if (r == 12345.0f) sink[blockIdx.x] = r;  // never true; keeps the chains live
}

cudaError_t launch_fp32x2_probe(int blocks, int threads, int iters, float* sink, cudaStream_t st) {
    fp32x2_probe_kernel<<<blocks, threads, 0, st>>>(iters, sink);
    return cudaGetLastError();
}

}  // namespace prrtc
