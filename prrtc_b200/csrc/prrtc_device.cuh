// prrtc_device.cuh -- device building blocks of the B200 pRRTC planner (sm_100a).
//
// Layout of one packed scene ("blob"): a 128-byte header followed by 16-byte
// aligned sections (joints, fine spheres, coarse groups, sphere chunks, world
// primitives pre-conditioned for the tests, self-collision work items, coarse
// self pairs).  A planner CTA copies its blob into shared memory with one bulk
// TMA copy, so every table lookup of the collision check is a shared-memory
// read (broadcast for world primitives).
//
// Collision semantics follow the reference checkers (cuda-rrtc/CUDA/
// prrtc_planner.cu:234-655): a configuration is in collision when any robot
// sphere is within `inflate` of a world primitive or another sphere of an active
// self pair.  inflate = 0 is the binary checker (d <= 0, 252-303); inflate =
// margin is the differentiable checker, whose verdict "sum of margin penalties
// < 0" (386) holds exactly when some distance is below the margin.  Coarse
// gating (426-499, 540-655) only skips work whose verdict is known to be "free".
#pragma once

#include <cuda_runtime.h>
#include <float.h>
#include <stddef.h>
#include <stdint.h>

#include "kernels.h"

namespace prrtc {

constexpr int kDimMax = 16;
constexpr int kMaxJoints = 64;
constexpr int kMaxLinks = 64;
constexpr int kObsChunk = 32;    // world primitives per work item
#ifndef PRRTC_SPH_CHUNK
#define PRRTC_SPH_CHUNK 8
#endif
constexpr int kSphChunk = PRRTC_SPH_CHUNK;  // fine spheres held in registers per work item
constexpr int kPairChunk = 32;   // explicit self pairs per work item
constexpr float kFar = 1.0e18f;  // centre of a sphere that can never collide
// Box records are stored scaled by 1/kBoxScale (a power of two, so the scaling
// is exact): the checker's relu(|l| - h) becomes a saturating add, exact for
// any distance below kBoxScale metres (robot spheres must be smaller than that).
constexpr float kBoxScale = 1024.0f;
constexpr float kBoxInv = 1.0f / 1024.0f;

// FP32 operations per primitive test as issued by the functions below (FFMA = 2,
// FADD/FMUL = 1; min/max/abs and the MUFU of sin/cos/sqrt are not counted).
constexpr int kFlopSphere = 8, kFlopCapsule = 23, kFlopBox = 26, kFlopHalfspace = 6;
constexpr int kFlopPair = 8, kFlopPairExplicit = 11;
constexpr int kFlopXform = 18;                  // one sphere centre
constexpr int kFlopJointLocal = 90, kFlopJointChain = 63;

// Device counters of the collision work (optional): [0] edges checked,
// [1] configurations checked, [2] FP32 flops executed by primitive tests,
// transforms and FK, [3] nearest-neighbour nodes scanned.
enum { kStatEdges = 0, kStatConfigs = 1, kStatFlops = 2, kStatNnNodes = 3, kStatCount = 4 };

// ----------------------------------------------------------------------------- blob

struct BlobHeader {
    int32_t J, dim, S, S_pad;
    int32_t K, Q, Ns, Nc;
    int32_t Nb, Nh, n_sch, n_items;
    int32_t n_och, gated, enabled, inflate_bits;
    int32_t o_joint, o_sph, o_sfr, o_grp;
    int32_t o_sch, o_ws, o_wc, o_wb;
    int32_t o_wh, o_item, o_cpair, used_bytes;
    int32_t P, cap_bytes, error, pad0;
};
static_assert(sizeof(BlobHeader) == 128, "header must stay 128 bytes");
// Bits of BlobHeader::error: the pack kernel's self-pair item list overflowed
// (the flat pair list is used instead), a checker CTA's scene-staging wait ran
// out (it read the scene from global memory instead).  Neither changes a verdict.
constexpr int kBlobItemOverflow = 1;
constexpr int kBlobStagingTimeout = 2;

struct JointRec {     // 96 bytes
    float4 r0, r1, r2;  // parent transform rows: (R0x R0y R0z tx) ...
    float4 tv;          // twist linear part, .w = mimic_mul
    float4 tw;          // twist angular part, .w = mimic_off
    int4 idx;           // parent, act_idx, mimic_act_idx, kind (0 screw, 1 revolute, 2 prismatic, 3 fixed)
};

__host__ __device__ inline int align16(int x) { return (x + 15) & ~15; }
__host__ __device__ inline int cdiv(int a, int b) { return (a + b - 1) / b; }
__host__ __device__ inline int odd_pad(int s) { return s | 1; }

// Capacity of a blob for the given (maximum) counts.  Layout offsets are
// computed by the pack kernel with the same arithmetic.
struct BlobLayout {
    int o_joint, o_sph, o_sfr, o_grp, o_sch, o_ws, o_wc, o_wb, o_wh, o_item, o_cpair, bytes;
    int sch_cap, item_cap;
};

__host__ __device__ inline BlobLayout blob_layout(int J, int S, int K, int Q, int P, int Ns, int Nc,
                                                  int Nb, int Nh) {
    BlobLayout L;
    int off = (int)sizeof(BlobHeader);
    L.sch_cap = cdiv(S, kSphChunk) + K + 1;
    L.item_cap = cdiv(P, kSphChunk) + 2 * Q + cdiv(P, kPairChunk) + 2;
    L.o_joint = off; off += J * (int)sizeof(JointRec);
    L.o_sph = off;   off += S * 16;
    L.o_sfr = off;   off += align16(S * 4);
    L.o_grp = off;   off += K * 32;
    L.o_sch = off;   off += L.sch_cap * 16;
    L.o_ws = off;    off += Ns * 32;
    L.o_wc = off;    off += Nc * 48;
    L.o_wb = off;    off += Nb * 64;
    L.o_wh = off;    off += Nh * 16;
    L.o_item = off;  off += L.item_cap * 16;
    L.o_cpair = off; off += align16(Q * 8);
    L.bytes = align16(off);
    return L;
}

constexpr float kPcExtent = 1.0e4f;  // points and sphere centres beyond +-10 km are ignored
constexpr int kPcMaxCells = 512;     // a sphere spanning more grid cells is reported as a hit
constexpr int kFlopPoint = 8;        // 3 FADD + FMUL + 2 FFMA per point test

__device__ __forceinline__ unsigned pc_hash(int x, int y, int z, int mask) {
    return ((unsigned)x * 73856093u ^ (unsigned)y * 19349663u ^ (unsigned)z * 83492791u) & (unsigned)mask;
}

struct Scene {  // typed view of a blob (shared or global memory)
    const BlobHeader* h;
    const JointRec* joints;
    const float4* sph;
    const int* sfr;
    const float4* grp;   // [K][2]: (c, r) then int4 bits (frame, s0, s1, 0)
    const int4* sch;
    const float4* ws;    // [Ns][2]: (-2x,-2y,-2z,-2r), (x,y,z, x^2+y^2+z^2-r^2)
    const float4* wc;    // [Nc][3]: (p1, r), (d/|d|^2, -p1.d/|d|^2), (d, 0)   with d = p2 - p1
    const float4* wb;    // [Nb][4]: (a1, -a1.c), (a2, -a2.c), (a3, -a3.c), (h1, h2, h3, 0)
    const float4* wh;    // [Nh]:    (n, -n.p)
    const int4* item;
    const int2* cpair;
    const int2* pairs;   // explicit self-pair list (global memory), for non-block items
    PcView pc;           // environment point cloud (global memory), pc.n == 0 when absent
};

__device__ __forceinline__ Scene scene_view(const unsigned char* b) {
    Scene s;
    s.h = reinterpret_cast<const BlobHeader*>(b);
    s.joints = reinterpret_cast<const JointRec*>(b + s.h->o_joint);
    s.sph = reinterpret_cast<const float4*>(b + s.h->o_sph);
    s.sfr = reinterpret_cast<const int*>(b + s.h->o_sfr);
    s.grp = reinterpret_cast<const float4*>(b + s.h->o_grp);
    s.sch = reinterpret_cast<const int4*>(b + s.h->o_sch);
    s.ws = reinterpret_cast<const float4*>(b + s.h->o_ws);
    s.wc = reinterpret_cast<const float4*>(b + s.h->o_wc);
    s.wb = reinterpret_cast<const float4*>(b + s.h->o_wb);
    s.wh = reinterpret_cast<const float4*>(b + s.h->o_wh);
    s.item = reinterpret_cast<const int4*>(b + s.h->o_item);
    s.cpair = reinterpret_cast<const int2*>(b + s.h->o_cpair);
    s.pairs = nullptr;
    s.pc = PcView{nullptr, nullptr, 0, 0, 0.0f, 0.0f};
    return s;
}

// Sphere c (c.w = radius + inflation) against the point cloud: any point p with
// |c - p| <= c.w + r_env.  Visits every grid cell the sphere's bounding box
// touches; a box of more than kPcMaxCells cells is conservatively a hit.  With
// |c| < kPcExtent, 0 <= R < 1e3 and a cell of at least 1 mm every cell index
// stays below 2^31 in magnitude.
__device__ inline bool pc_sphere_hits(const PcView& pc, float4 c, bool full_sweep, unsigned long long& flops) {
    if (!(fabsf(c.x) < kPcExtent && fabsf(c.y) < kPcExtent && fabsf(c.z) < kPcExtent)) return false;
    const float R = c.w + pc.r_env;
    if (!(R >= 0.0f)) return false;  // negative or NaN radius: touches nothing
    if (!(R < 1.0e3f)) return true;  // a sphere of 1 km or more is conservatively a hit
    const float R2 = R * R;
    const int x0 = (int)floorf((c.x - R) * pc.inv_cell), x1 = (int)floorf((c.x + R) * pc.inv_cell);
    const int y0 = (int)floorf((c.y - R) * pc.inv_cell), y1 = (int)floorf((c.y + R) * pc.inv_cell);
    const int z0 = (int)floorf((c.z - R) * pc.inv_cell), z1 = (int)floorf((c.z + R) * pc.inv_cell);
    const long long cells = ((long long)x1 - x0 + 1) * ((long long)y1 - y0 + 1) * ((long long)z1 - z0 + 1);
    if (cells > kPcMaxCells) return true;
    bool hit = false;
    for (int z = z0; z <= z1; ++z)
        for (int y = y0; y <= y1; ++y)
            for (int x = x0; x <= x1; ++x) {
                const unsigned b = pc_hash(x, y, z, pc.mask);
                const int p1 = __ldg(&pc.start[b + 1]);
                int p = __ldg(&pc.start[b]);
                flops += (unsigned long long)(p1 - p) * kFlopPoint;
                for (; p < p1; ++p) {
                    const float4 q = __ldg(&pc.pts[p]);
                    const float dx = c.x - q.x, dy = c.y - q.y, dz = c.z - q.z;
                    hit |= fmaf(dx, dx, fmaf(dy, dy, dz * dz)) <= R2;
                    if (hit && !full_sweep) return true;
                }
            }
    return hit;
}

// ----------------------------------------------------------------------------- small helpers

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ int ld_volatile(const int* p) { return *reinterpret_cast<const volatile int*>(p); }

// ----------------------------------------------------------------------------- scene staging

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* mbar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_addr(mbar)), "r"(parity)
        : "memory");
    return done != 0;
}

constexpr int kWaitLimit = 1 << 22;

// Bulk-copy `bytes` (multiple of 16; both addresses 16-byte aligned) from global
// memory into shared memory (cp.async.bulk, no multicast) and wait for
// completion with a bounded spin of `first_limit` polls.  All threads of the CTA
// call it.  Returns false (uniformly) if the wait ran out, after OR-ing
// `err_code` into *err (when given) and giving the copy a second bounded wait
// to land, so that no copy still targets shared memory the CTA goes on to
// reuse or leaves.
__device__ inline bool stage_blob(unsigned char* dst, const unsigned char* src, int bytes, uint64_t* mbar,
                                  uint32_t& phase, int* err, int err_code, int first_limit) {
    __syncthreads();  // previous readers of dst are done
    if (threadIdx.x == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        uint64_t state;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 %0, [%1], %2;"
                     : "=l"(state)
                     : "r"(smem_addr(mbar)), "r"(bytes)
                     : "memory");
        (void)state;
        for (int off = 0; off < bytes; off += 16384) {
            const int n = min(16384, bytes - off);
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_addr(dst + off)),
                "l"(src + off), "r"(n), "r"(smem_addr(mbar))
                : "memory");
        }
    }
    bool ok = false;
    for (int i = 0; i < first_limit && !ok; ++i) ok = mbar_try_wait(mbar, phase);
    const bool all_ok = __syncthreads_and(ok ? 1 : 0) != 0;
    if (!all_ok) {
        // the wait ran out: report it, then let the copy land (bounded) before
        // the CTA stops using -- or leaves -- its shared memory
        if (threadIdx.x == 0 && err) atomicOr(err, err_code);
        for (int i = 0; i < kWaitLimit && !ok; ++i) ok = mbar_try_wait(mbar, phase);
        __syncthreads();
    }
    phase ^= 1u;
    return all_ok;
}

// Dynamic-domain radius updates (prrtc_planner.cu:46-83).  As in the
// reference, FLT_MAX means "unset": a failed extension from an unset node sets
// its radius to r0, otherwise shrinks it by (1 - alpha) down to rmin; a
// successful one grows a set radius by (1 + alpha).  Concurrent updates of one
// node are compare-and-swap loops.  Every CAS round lets at least one contender
// through, so a loop ends after as many rounds as there are contenders; the
// guard only bounds it, and a guard that runs out sets *err (when given).
constexpr int kCasGuard = 1 << 20;

__device__ __forceinline__ bool radius_unset(float r) { return r == FLT_MAX; }

__device__ inline void radius_shrink(float* radii, int idx, float alpha, float r0, float rmin, int* err) {
    int* ri = reinterpret_cast<int*>(&radii[idx]);
    int old_i = atomicAdd(ri, 0);
    for (int guard = 0;; ++guard) {
        if (guard == kCasGuard) {
            if (err) atomicExch(err, 1);
            return;
        }
        const float old_r = __int_as_float(old_i);
        const float new_r = radius_unset(old_r) ? r0 : fmaxf(old_r * (1.0f - alpha), rmin);
        const int prev = atomicCAS(ri, old_i, __float_as_int(new_r));
        if (prev == old_i) return;
        old_i = prev;
    }
}

__device__ inline void radius_grow(float* radii, int idx, float alpha, int* err) {
    int* ri = reinterpret_cast<int*>(&radii[idx]);
    int old_i = atomicAdd(ri, 0);
    for (int guard = 0;; ++guard) {
        if (guard == kCasGuard) {
            if (err) atomicExch(err, 1);
            return;
        }
        const float old_r = __int_as_float(old_i);
        if (radius_unset(old_r)) return;
        const int prev = atomicCAS(ri, old_i, __float_as_int(old_r * (1.0f + alpha)));
        if (prev == old_i) return;
        old_i = prev;
    }
}

// Tree side of an explorer's next extension (prrtc_planner.cu:790-824);
// nblocks = explorers of the problem, bid = this explorer's index among them.
//   mode 0, or the first iteration: the first half of the explorers extend tree A;
//   mode 1: while the sizes differ by fewer than 1.5 nblocks, the first
//           nblocks * (1 - |A| / (|A| + |B|)) explorers take A, else A iff the A
//           share is below tree_ratio;
//   mode 2: the explorer toggles its own side whenever |t - o| / t < tree_ratio
//           for its current side t (`vamp` is that per-explorer state);
//   mode 3: the smaller tree (A on ties).
__device__ __forceinline__ int choose_tree(int mode, int local_iter, int bid, int nblocks, int size_a, int size_b,
                                           float thr, int& vamp) {
    const int total = size_a + size_b;
    if (mode == 0 || local_iter == 1) return (bid < (nblocks / 2)) ? 0 : 1;
    if (mode == 1) {
        const int diff = size_a >= size_b ? size_a - size_b : size_b - size_a;
        const float ratio = total > 0 ? __fdiv_rn((float)size_a, (float)total) : 0.5f;
        if (diff < (int)(1.5f * (float)nblocks)) return (bid < (int)((float)nblocks * (1.0f - ratio))) ? 0 : 1;
        return ratio < thr ? 0 : 1;
    }
    if (mode == 2) {
        const int o_id = 1 - vamp;
        const int t_sz = vamp == 0 ? size_a : size_b;
        const int o_sz = o_id == 0 ? size_a : size_b;
        const float r = t_sz > 0 ? fabsf(__fdiv_rn((float)(t_sz - o_sz), (float)t_sz)) : 0.0f;
        if (r < thr) vamp = 1 - vamp;
        return vamp;
    }
    return size_a <= size_b ? 0 : 1;
}

// ----------------------------------------------------------------------------- sampling

// Halton radical inverse (prrtc_planner.cu:144-157): IEEE divide, one FMA per digit.
__device__ __forceinline__ float halton_next(int base, int& state) {
    float fraction = 1.0f, result = 0.0f;
    int n = state;
    const float fb = (float)base;
    while (n > 0) {
        fraction = __fdiv_rn(fraction, fb);
        result = __fmaf_rn(fraction, (float)(n % base), result);
        n /= base;
    }
    state = state + 1;
    return result;
}

// Per-explorer prime order (prrtc_planner.cu:747-758).
__device__ inline void prime_order(int explorer, int* out16) {
    int p[16] = {3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59};
    if (explorer != 0) {
        unsigned int rng = (unsigned int)explorer * 1664525u + 1013904223u;
        for (int i = 15; i > 0; --i) {
            rng = rng * 1664525u + 1013904223u;
            const int j = (int)(rng % (unsigned int)(i + 1));
            const int t = p[i];
            p[i] = p[j];
            p[j] = t;
        }
    }
#pragma unroll
    for (int d = 0; d < 16; ++d) out16[d] = p[d];
}

// Sample (784-788): min + val * (max - min) as one FMA.
__device__ __forceinline__ void halton_sample(const int* order, int* states, int dim, const float* lo,
                                              const float* hi, float* out) {
    for (int d = 0; d < dim; ++d) {
        const float val = halton_next(order[d & 15], states[d]);
        out[d] = __fmaf_rn(val, __fsub_rn(hi[d], lo[d]), lo[d]);
    }
}

// Waypoint count: `granularity`, raised to ceil(|delta|/res) when res > 0.
__device__ __forceinline__ int edge_waypoints(const float* delta, int dim, int G, float res) {
    if (!(res > 0.0f)) return G;
    float s = __fmul_rn(delta[0], delta[0]);
    for (int d = 1; d < dim; ++d) s = __fmaf_rn(delta[d], delta[d], s);
    const int n = (int)ceilf(__fdiv_rn(__fsqrt_rn(s), res));
    return n > G ? n : G;
}

// ----------------------------------------------------------------------------- FK

// out = a o b ([R|t] as 12 floats, R row-major)
__device__ __forceinline__ void compose(const float* a, const float* b, float* out) {
    float o[12];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int j = 0; j < 3; ++j) o[i * 3 + j] = fmaf(a[i * 3 + 0], b[j], fmaf(a[i * 3 + 1], b[3 + j], a[i * 3 + 2] * b[6 + j]));
        o[9 + i] = fmaf(a[i * 3 + 0], b[9], fmaf(a[i * 3 + 1], b[10], fmaf(a[i * 3 + 2], b[11], a[9 + i])));
    }
#pragma unroll
    for (int i = 0; i < 12; ++i) out[i] = o[i];
}

__device__ __forceinline__ float joint_value(const JointRec& jr, const float* q) {
    if (jr.idx.z >= 0) return fmaf(jr.tv.w, q[jr.idx.z], jr.tw.w);
    if (jr.idx.y >= 0) return q[jr.idx.y];
    return 0.0f;
}

// Local transform parent_tf o exp(twist * v) of one joint, written as 12 floats.
__device__ inline void joint_local(const JointRec& jr, float v, float* out) {
    const float P[12] = {jr.r0.x, jr.r0.y, jr.r0.z, jr.r1.x, jr.r1.y, jr.r1.z,
                         jr.r2.x, jr.r2.y, jr.r2.z, jr.r0.w, jr.r1.w, jr.r2.w};
    const int kind = jr.idx.w;
    if (kind == 3) {
#pragma unroll
        for (int i = 0; i < 12; ++i) out[i] = P[i];
        return;
    }
    float E[12];
    if (kind == 2) {  // pure translation along v
        E[0] = 1; E[1] = 0; E[2] = 0; E[3] = 0; E[4] = 1; E[5] = 0; E[6] = 0; E[7] = 0; E[8] = 1;
        E[9] = jr.tv.x * v; E[10] = jr.tv.y * v; E[11] = jr.tv.z * v;
    } else {
        const float wx = jr.tw.x * v, wy = jr.tw.y * v, wz = jr.tw.z * v;
        const float th2 = fmaf(wx, wx, fmaf(wy, wy, wz * wz));
        const float th = sqrtf(th2);
        float A, B, Cc;
        if (kind == 1) {  // unit axis: th = |v|, R = I + sin(v) K + (1-cos(v)) K^2 with K from the axis
            float s, c;
            sincosf(v, &s, &c);
            const float ax = jr.tw.x, ay = jr.tw.y, az = jr.tw.z;
            const float oc = 1.0f - c;
            E[0] = fmaf(oc, ax * ax - 1.0f, 1.0f); E[1] = fmaf(oc, ax * ay, -s * az); E[2] = fmaf(oc, ax * az, s * ay);
            E[3] = fmaf(oc, ay * ax, s * az); E[4] = fmaf(oc, ay * ay - 1.0f, 1.0f); E[5] = fmaf(oc, ay * az, -s * ax);
            E[6] = fmaf(oc, az * ax, -s * ay); E[7] = fmaf(oc, az * ay, s * ax); E[8] = fmaf(oc, az * az - 1.0f, 1.0f);
            E[9] = 0; E[10] = 0; E[11] = 0;
        } else {
            if (th < 1e-4f) {
                A = 1.0f - th2 * (1.0f / 6.0f);
                B = 0.5f - th2 * (1.0f / 24.0f);
                Cc = (1.0f / 6.0f) - th2 * (1.0f / 120.0f);
            } else {
                float s, c;
                sincosf(th, &s, &c);
                A = s / th;
                B = (1.0f - c) / th2;
                Cc = (th - s) / (th2 * th);
            }
            const float K[9] = {0, -wz, wy, wz, 0, -wx, -wy, wx, 0};
            const float K2[9] = {wx * wx - th2, wx * wy, wx * wz, wy * wx, wy * wy - th2, wy * wz,
                                 wz * wx, wz * wy, wz * wz - th2};
            float V[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                E[i] = fmaf(A, K[i], B * K2[i]);
                V[i] = fmaf(B, K[i], Cc * K2[i]);
            }
            E[0] += 1.0f; E[4] += 1.0f; E[8] += 1.0f;
            V[0] += 1.0f; V[4] += 1.0f; V[8] += 1.0f;
            const float vx = jr.tv.x * v, vy = jr.tv.y * v, vz = jr.tv.z * v;
            E[9] = fmaf(V[0], vx, fmaf(V[1], vy, V[2] * vz));
            E[10] = fmaf(V[3], vx, fmaf(V[4], vy, V[5] * vz));
            E[11] = fmaf(V[6], vx, fmaf(V[7], vy, V[8] * vz));
        }
    }
    compose(P, E, out);
}

// Joint record from the reference tables: parent_tf quaternion (normalised) as a
// rotation matrix, twist split into linear/angular parts, joint kind.
__device__ inline JointRec make_joint_rec(int j, const float* ptf, const float* twists, const int32_t* parent,
                                          const int32_t* act, const float* mmul, const float* moff,
                                          const int32_t* mact, int dim) {
    const float* q = &ptf[j * 7];
    float w = q[0], x = q[1], y = q[2], z = q[3];
    const float n = sqrtf(w * w + x * x + y * y + z * z);
    if (n > 0.0f) { w /= n; x /= n; y /= n; z /= n; } else { w = 1.0f; x = y = z = 0.0f; }
    JointRec r;
    r.r0 = make_float4(1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y), q[4]);
    r.r1 = make_float4(2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x), q[5]);
    r.r2 = make_float4(2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y), q[6]);
    const float* tw = &twists[j * 6];
    r.tv = make_float4(tw[0], tw[1], tw[2], mmul ? mmul[j] : 1.0f);
    r.tw = make_float4(tw[3], tw[4], tw[5], moff ? moff[j] : 0.0f);
    const float vn = sqrtf(tw[0] * tw[0] + tw[1] * tw[1] + tw[2] * tw[2]);
    const float wn = sqrtf(tw[3] * tw[3] + tw[4] * tw[4] + tw[5] * tw[5]);
    int kind = 0;
    if (vn < 1e-12f && wn < 1e-12f) kind = 3;
    else if (wn < 1e-12f) kind = 2;
    else if (vn < 1e-12f && fabsf(wn - 1.0f) < 1e-6f) kind = 1;
    int a = act ? act[j] : -1;
    int ma = mact ? mact[j] : -1;
    if (a >= dim) a = -1;
    if (ma >= dim) ma = -1;
    int par = parent ? parent[j] : -1;
    if (par >= j) par = -1;
    r.idx = make_int4(par, a, ma, kind);
    return r;
}

// ----------------------------------------------------------------------------- primitive tests

__device__ __forceinline__ float4 xform_point(const float* F, float4 l) {
    float4 r;
    r.x = fmaf(F[0], l.x, fmaf(F[1], l.y, fmaf(F[2], l.z, F[9])));
    r.y = fmaf(F[3], l.x, fmaf(F[4], l.y, fmaf(F[5], l.z, F[10])));
    r.z = fmaf(F[6], l.x, fmaf(F[7], l.y, fmaf(F[8], l.z, F[11])));
    r.w = l.w;
    return r;
}

// FFMA-dense tests.  Every test yields a value that is <= 0 exactly when the
// pair is within its threshold; a work item keeps the minimum over its spheres
// and compares once per obstacle.
//
// Sphere-sphere: |c-o|^2 - (rc+ro)^2 = (|c|^2 - rc^2) + (|o|^2 - ro^2) - 2 c.o - 2 rc ro.
// With A = |c|^2 - rc^2 per robot sphere and the obstacle stored as
// O = (-2o, -2ro), B = |o|^2 - ro^2, the per-pair part is four FMAs:
// g = A + c.O, and the pair collides iff g <= -B.
__device__ __forceinline__ float sphere_A(float4 c) { return fmaf(c.x, c.x, fmaf(c.y, c.y, fmaf(c.z, c.z, -c.w * c.w))); }

// Per-sphere running minima.  Each test below returns a value h whose
// comparison with a per-sphere threshold decides a hit; a work item keeps one
// running minimum per sphere over all obstacles of a type (independent FFMA
// chains, no cross-sphere reduction per obstacle) and compares once per group
// of obstacles:
//   sphere     h = B + O.(c, r)        (O = -2(o, r_o), B = |o|^2 - r_o^2),  hit iff h <= -(|c|^2 - r^2)
//   capsule    h = |e|^2 - (r + r_c)^2 (e = c - p1 - t d, t = sat(d'.c + off)), hit iff h <= 0
//   box        h = |max(|l| - hl, 0)|^2 (l = box-frame coordinates),         hit iff h <= r^2
//              (computed in units of kBoxScale metres: h/kBoxScale^2 against (r/kBoxScale)^2)
//   halfspace  h = n.c - n.p                                                  hit iff h <= r
// Three-input minimum (PTX min.f32 with three sources, sm_100): folds two
// obstacles into a running minimum with one instruction.
__device__ __forceinline__ float fmin3(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

template <int NS>
__device__ __forceinline__ void h_sphere(float (&h)[NS], const float4 (&c)[NS], float4 O, float B) {
#pragma unroll
    for (int k = 0; k < NS; ++k) h[k] = fmaf(c[k].x, O.x, fmaf(c[k].y, O.y, fmaf(c[k].z, O.z, fmaf(c[k].w, O.w, B))));
}

template <int NS>
__device__ __forceinline__ void h_capsule(float (&h)[NS], const float4 (&c)[NS], float4 p1r, float4 dp, float4 d) {
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        const float t = __saturatef(fmaf(dp.x, c[k].x, fmaf(dp.y, c[k].y, fmaf(dp.z, c[k].z, dp.w))));
        const float ex = fmaf(-t, d.x, c[k].x - p1r.x);
        const float ey = fmaf(-t, d.y, c[k].y - p1r.y);
        const float ez = fmaf(-t, d.z, c[k].z - p1r.z);
        const float s = c[k].w + p1r.w;
        h[k] = fmaf(ex, ex, fmaf(ey, ey, fmaf(ez, ez, -s * s)));
    }
}

// Box rows and half extents arrive scaled by kBoxInv, so l/kBoxScale and
// h/kBoxScale: sat(|l| - h) is relu(|l| - h)/kBoxScale (one saturating add
// instead of a subtract and a max) and h is |q|^2/kBoxScale^2, bit for bit.
template <int NS>
__device__ __forceinline__ void h_box(float (&h)[NS], const float4 (&c)[NS], float4 a1, float4 a2, float4 a3,
                                      float4 hl) {
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        const float q1 = __saturatef(fabsf(fmaf(a1.x, c[k].x, fmaf(a1.y, c[k].y, fmaf(a1.z, c[k].z, a1.w)))) - hl.x);
        const float q2 = __saturatef(fabsf(fmaf(a2.x, c[k].x, fmaf(a2.y, c[k].y, fmaf(a2.z, c[k].z, a2.w)))) - hl.y);
        const float q3 = __saturatef(fabsf(fmaf(a3.x, c[k].x, fmaf(a3.y, c[k].y, fmaf(a3.z, c[k].z, a3.w)))) - hl.z);
        h[k] = fmaf(q1, q1, fmaf(q2, q2, q3 * q3));
    }
}

template <int NS>
__device__ __forceinline__ void h_halfspace(float (&h)[NS], const float4 (&c)[NS], float4 hs) {
#pragma unroll
    for (int k = 0; k < NS; ++k) h[k] = fmaf(hs.x, c[k].x, fmaf(hs.y, c[k].y, fmaf(hs.z, c[k].z, hs.w)));
}

template <int NS>
__device__ __forceinline__ void fold1(float (&m)[NS], const float (&h)[NS]) {
#pragma unroll
    for (int k = 0; k < NS; ++k) m[k] = fminf(m[k], h[k]);
}

template <int NS>
__device__ __forceinline__ void fold2(float (&m)[NS], const float (&h1)[NS], const float (&h2)[NS]) {
#pragma unroll
    for (int k = 0; k < NS; ++k) m[k] = fmin3(m[k], h1[k], h2[k]);
}

template <int NS>
__device__ __forceinline__ bool any_le(const float (&m)[NS], const float (&thr)[NS]) {
    bool r = false;
#pragma unroll
    for (int k = 0; k < NS; ++k) r |= m[k] <= thr[k];
    return r;
}

template <int NS>
__device__ __forceinline__ void fill(float (&m)[NS], float v) {
#pragma unroll
    for (int k = 0; k < NS; ++k) m[k] = v;
}

// An absent sphere (chunk padding, or a sphere whose frame does not exist):
// NaN centre and radius.  Every test value h is then NaN, which fminf / min.f32
// skip, or its threshold is NaN, which no comparison passes -- whatever the
// obstacle's orientation (a far-away finite centre would still fall on the
// negative side of some halfspaces).
__device__ __forceinline__ float4 absent_sphere() {
    const float n = __int_as_float(0x7fc00000);
    return make_float4(n, n, n, n);
}

// World obstacles form one list in type order (spheres, capsules, boxes,
// halfspaces).  Work items take contiguous ranges of that list of roughly equal
// cost; the weights are the issue slots of one sphere test of each type.
constexpr int kCostSphere = 5, kCostCapsule = 15, kCostBox = 19, kCostHalfspace = 5;

__device__ __forceinline__ int world_cost(const BlobHeader& h) {
    return kCostSphere * h.Ns + kCostCapsule * h.Nc + kCostBox * h.Nb + kCostHalfspace * h.Nh;
}

// First obstacle (combined index) whose cost offset is >= x.
__device__ __forceinline__ int world_index_at(const BlobHeader& h, int x) {
    int base = 0, cbase = 0;
    const int n[4] = {h.Ns, h.Nc, h.Nb, h.Nh};
    const int w[4] = {kCostSphere, kCostCapsule, kCostBox, kCostHalfspace};
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const int span = n[t] * w[t];
        if (x <= cbase + span) return base + (x - cbase + w[t] - 1) / w[t];
        base += n[t];
        cbase += span;
    }
    return base;
}

// Obstacles [j0, j1) of the combined list against NS sphere centres held in
// registers (c.w = radius + inflation; padding spheres are absent_sphere()).  FULL:
// test every obstacle; otherwise stop at the first group of kHitCheck
// obstacles that holds a hit.  flops accumulates the FP32 flops of the tests
// executed (NS_real real spheres per test).
constexpr int kHitCheck = 8;

// One sphere chunk against obstacles [lo, hi) of one type: running minimum per
// sphere; FULL && PAIRS folds two obstacles per three-input minimum, otherwise
// one obstacle at a time, with a hit check every kHitCheck obstacles unless
// FULL.  Returns whether some sphere reached its threshold; `done` = obstacles
// tested.
template <int NS, bool FULL, bool PAIRS, class Test>
__device__ __forceinline__ bool sweep_type(float (&m)[NS], const float (&thr)[NS], int lo, int hi, Test test,
                                           int& done) {
    fill(m, INFINITY);
    int o = lo;
    if constexpr (FULL && PAIRS) {  // throughput form: two obstacles per fold
        for (; o + 1 < hi; o += 2) {
            float h1[NS], h2[NS];
            test(h1, o);
            test(h2, o + 1);
            fold2(m, h1, h2);
        }
    } else {  // one obstacle per fold (fewer live registers), early exit unless FULL
        for (; o < hi; ++o) {
            float h1[NS];
            test(h1, o);
            fold1(m, h1);
            if (!FULL && ((o - lo) & (kHitCheck - 1)) == kHitCheck - 1 && any_le(m, thr)) {
                done = o + 1 - lo;
                return true;
            }
        }
    }
    if (o < hi) {
        float h1[NS];
        test(h1, o);
        fold1(m, h1);
    }
    done = hi - lo;
    return any_le(m, thr);
}

template <int NS>
__device__ __forceinline__ uint32_t le_mask(const float (&m)[NS], const float (&thr)[NS]) {
    uint32_t r = 0u;
#pragma unroll
    for (int k = 0; k < NS; ++k) r |= (m[k] <= thr[k] ? 1u : 0u) << k;
    return r;
}

// Returns the spheres found in collision as a bit mask (bit k = s[k]).  With
// !FULL the sweep stops at the first group of obstacles holding a hit, so the
// mask is then non-zero but may be incomplete.  PAIRS folds world spheres two
// at a time; capsules and boxes, whose tests hold more operands, fold one at a
// time (measured faster in the full sweep: less code, no register spill in the
// loop).
template <int NS, bool FULL, bool PAIRS = FULL>
__device__ __forceinline__ uint32_t obstacles_vs_spheres(const Scene& sc, int j0, int j1, const float4 (&s)[NS],
                                                         int ns_real, unsigned long long& flops) {
    const BlobHeader& h = *sc.h;
    float m[NS], thr[NS];
    uint32_t mask = 0u;
    int done = 0;
    int lo = max(j0, 0), hi = min(j1, h.Ns);
    if (lo < hi) {
#pragma unroll
        for (int k = 0; k < NS; ++k) thr[k] = -sphere_A(s[k]);
        const float4* ws = sc.ws;
        if (sweep_type<NS, FULL, PAIRS>(m, thr, lo, hi, [&](float (&v)[NS], int o) { h_sphere<NS>(v, s, ws[2 * o], ws[2 * o + 1].w); }, done))
            mask |= le_mask(m, thr);
        flops += (unsigned long long)done * ns_real * kFlopSphere;
        if (!FULL && mask) return mask;
    }
    int base = h.Ns;
    lo = max(j0, base) - base;
    hi = min(j1, base + h.Nc) - base;
    if (lo < hi) {
        fill(thr, 0.0f);
        const float4* wc = sc.wc;
        if (sweep_type<NS, FULL, false>(m, thr, lo, hi, [&](float (&v)[NS], int o) { h_capsule<NS>(v, s, wc[3 * o], wc[3 * o + 1], wc[3 * o + 2]); }, done))
            mask |= le_mask(m, thr);
        flops += (unsigned long long)done * ns_real * kFlopCapsule;
        if (!FULL && mask) return mask;
    }
    base += h.Nc;
    lo = max(j0, base) - base;
    hi = min(j1, base + h.Nb) - base;
    if (lo < hi) {
#pragma unroll
        for (int k = 0; k < NS; ++k) thr[k] = (s[k].w * kBoxInv) * (s[k].w * kBoxInv);
        const float4* wb = sc.wb;
        if (sweep_type<NS, FULL, false>(m, thr, lo, hi, [&](float (&v)[NS], int o) { h_box<NS>(v, s, wb[4 * o], wb[4 * o + 1], wb[4 * o + 2], wb[4 * o + 3]); }, done))
            mask |= le_mask(m, thr);
        flops += (unsigned long long)done * ns_real * kFlopBox;
        if (!FULL && mask) return mask;
    }
    base += h.Nb;
    lo = max(j0, base) - base;
    hi = min(j1, base + h.Nh) - base;
    if (lo < hi) {
#pragma unroll
        for (int k = 0; k < NS; ++k) thr[k] = s[k].w;
        const float4* wh = sc.wh;
        if (sweep_type<NS, true, false>(m, thr, lo, hi, [&](float (&v)[NS], int o) { h_halfspace<NS>(v, s, wh[o]); }, done))
            mask |= le_mask(m, thr);
        flops += (unsigned long long)done * ns_real * kFlopHalfspace;
    }
    return mask;
}

// ----------------------------------------------------------------------------- thread groups

// The checker, the nearest-neighbour scan and the explorer loop run on a whole
// CTA (one explorer per CTA); the group type supplies the rank, size and
// barrier.
struct CtaGroup {
    __device__ __forceinline__ int rank() const { return threadIdx.x; }
    __device__ __forceinline__ int size() const { return blockDim.x; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
};

// ----------------------------------------------------------------------------- CTA-cooperative check

// Shared-memory work buffers of the collision check for a chunk of CW waypoints.
struct CcBufs {
    float* q;        // [CW][kDimMax]
    float* pose;     // [CW][J][12]
    float4* ctr;     // [CW][S_pad]
    float4* cctr;    // [CW][K]
    uint32_t* dirty; // [CW][KW]
    uint32_t* gate;  // [CW][QW]
    uint32_t* hit;   // [4]: two alternating result words, two work-list counters
    int* bounds;     // [2][kMaxParts + 1] first obstacle of each world part (fine pass, coarse pass)
    unsigned long long* stats;  // optional device counters (kStat*), may be null
    int listcap;     // ints the work lists may use in `pose` once the centres are placed
};

constexpr int kMaxParts = 256;  // world parts per chunk (cost-balanced obstacle ranges)

__host__ __device__ inline int cc_smem_bytes(int J, int S, int K, int Q, int CW) {
    const int S_pad = odd_pad(S);
    const int KW = cdiv(K > 0 ? K : 1, 32), QW = cdiv(Q > 0 ? Q : 1, 32);
    int b = 0;
    b += align16(CW * kDimMax * 4);
    b += align16(CW * J * 48);
    b += CW * S_pad * 16;
    b += CW * K * 16;
    b += align16(CW * KW * 4);
    b += align16(CW * QW * 4);
    b += 16;
    b += align16(2 * (kMaxParts + 1) * 4);
    return b;
}

__device__ inline CcBufs cc_bufs(unsigned char* base, int J, int S, int K, int Q, int CW) {
    const int S_pad = odd_pad(S);
    const int KW = cdiv(K > 0 ? K : 1, 32), QW = cdiv(Q > 0 ? Q : 1, 32);
    CcBufs b;
    unsigned char* p = base;
    b.q = reinterpret_cast<float*>(p);        p += align16(CW * kDimMax * 4);
    b.pose = reinterpret_cast<float*>(p);     p += align16(CW * J * 48);
    b.ctr = reinterpret_cast<float4*>(p);     p += CW * S_pad * 16;
    b.cctr = reinterpret_cast<float4*>(p);    p += CW * K * 16;
    b.dirty = reinterpret_cast<uint32_t*>(p); p += align16(CW * KW * 4);
    b.gate = reinterpret_cast<uint32_t*>(p);  p += align16(CW * QW * 4);
    b.hit = reinterpret_cast<uint32_t*>(p);    p += 16;
    b.bounds = reinterpret_cast<int*>(p);
    b.stats = nullptr;
    b.listcap = CW * J * 12;
    return b;
}

// Sphere centres of waypoint w (fine, and coarse when gated) from its frames in
// B.pose: spheres first, first + step, ... of this caller.
__device__ __forceinline__ void cc_centres(const Scene& sc, const CcBufs& B, int w, int first, int step, int J, int S,
                                           int S_pad, int K, bool gated, float inflate) {
    for (int s = first; s < S; s += step) {
        const int f = sc.sfr[s];
        float4 l = sc.sph[s];
        l.w += inflate;
        B.ctr[w * S_pad + s] = f >= 0 ? xform_point(&B.pose[(w * J + f) * 12], l) : absent_sphere();
    }
    if (gated) {
        for (int k = first; k < K; k += step) {
            float4 l = sc.grp[2 * k];
            l.w += inflate;
            const int f = __float_as_int(sc.grp[2 * k + 1].x);
            B.cctr[w * K + k] = f >= 0 ? xform_point(&B.pose[(w * J + f) * 12], l) : absent_sphere();
        }
    }
}

// Waypoints of an edge computed where they are needed instead of staged in
// B.q: waypoint w of pass c is base + t*delta with t = (c + w*nchunk + 1)/G,
// the same bits as the staged form.
struct EdgeSrc {
    const float* base;
    const float* delta;
    int G, nchunk, c;
};

__device__ __forceinline__ float cc_q(const CcBufs& B, const EdgeSrc* e, int w, int d) {
    if (!e) return B.q[w * kDimMax + d];
    const float t = __fdiv_rn((float)(e->c + w * e->nchunk + 1), (float)e->G);
    return __fmaf_rn(t, e->delta[d], e->base[d]);
}

// joint_value of waypoint w
__device__ __forceinline__ float cc_joint_value(const JointRec& jr, const CcBufs& B, const EdgeSrc* e, int w) {
    if (jr.idx.z >= 0) return fmaf(jr.tv.w, cc_q(B, e, w, jr.idx.z), jr.tw.w);
    if (jr.idx.y >= 0) return cc_q(B, e, w, jr.idx.y);
    return 0.0f;
}

// Collision check of nw (<= CW <= 32) configurations: B.q, or the waypoints of
// `edge` when given.  Every thread of the group must call it, with the same
// `par`, which the call flips: B.hit holds two words used on alternate calls,
// so a call clears the other word after its first barrier and no barrier is
// needed between one call's read of its result and the next call.  Both
// words must be zero (and `par` 0) before the first call.  edge_mode: stop all work at the first hit
// (the whole edge is rejected).  Otherwise each configuration stops at its own
// first hit, or never with full_sweep.  Returns the hit bit mask (bit w =
// configuration w in collision).
template <bool FULL_SWEEP, class G>
__device__ inline uint32_t cc_chunk(const G& g, const Scene& sc, const CcBufs& B, int nw, bool edge_mode, int& par,
                                    const EdgeSrc* edge = nullptr) {
    constexpr bool full_sweep = FULL_SWEEP;
    const BlobHeader& h = *sc.h;
    const int tid = g.rank(), T = g.size();
    const int J = h.J, S = h.S, S_pad = h.S_pad, K = h.K, Q = h.Q;
    const bool gated = h.gated != 0;
    const float inflate = __int_as_float(h.inflate_bits);
    const int KW = cdiv(K > 0 ? K : 1, 32), QW = cdiv(Q > 0 ? Q : 1, 32);
    uint32_t* hw = B.hit + par;
    volatile uint32_t* vhit = hw;
    par ^= 1;

    if (!h.enabled) {
        g.sync();
        return 0u;
    }
    // World work is split into n_parts ranges of the combined obstacle list with
    // about equal cost, enough parts for roughly two world items per thread; the
    // range bounds are computed once per chunk.
    const int n_obs = h.Ns + h.Nc + h.Nb + h.Nh;
    const int ctot = world_cost(h);
    // A full sweep (throughput) takes at most one world item per thread, and
    // whole-world items once there are more (sphere chunk, waypoint) pairs
    // than threads: measured faster than finer parts, whose fixed cost per
    // item outweighs the better spread.  Early-exit checks (latency) take
    // about two items per thread.
    const int n_parts = n_obs == 0 ? 0
                        : full_sweep ? min(kMaxParts, max(1, min(T / max(1, nw * h.n_sch), cdiv(n_obs, 4))))
                                     : min(kMaxParts, max(1, min(cdiv(2 * T, max(1, nw * h.n_sch)), cdiv(n_obs, 4))));
    // coarse pass: one item = up to 8 coarse spheres of a waypoint over a part
    const int KC = cdiv(K, 8);
    const int n_parts_c =
        (n_obs == 0 || !gated) ? 0 : min(kMaxParts, max(1, min(cdiv(2 * T, max(1, nw * KC)), cdiv(n_obs, 4))));
    int* bounds_c = B.bounds + (kMaxParts + 1);
    if (n_parts > 0)
        for (int i = tid; i <= n_parts; i += T) B.bounds[i] = world_index_at(h, (int)((long long)i * ctot / n_parts));
    if (n_parts_c > 0)
        for (int i = tid; i <= n_parts_c; i += T)
            bounds_c[i] = world_index_at(h, (int)((long long)i * ctot / n_parts_c));
    if (gated) {
        for (int i = tid; i < nw * KW; i += T) B.dirty[i] = 0u;
        for (int i = tid; i < nw * QW; i += T) B.gate[i] = 0u;
    }
    if (J <= 32) {
        // A+B in registers: a warp segment of SEG lanes per waypoint, lane j
        // computes joint j's local transform, then pointer jumping composes
        // the chain -- each round T_j = T_anc(j) o T_j, anc(j) = anc(anc(j)),
        // ancestors read with shuffles -- in ceil(log2 J) rounds with no
        // barrier.  Parents precede their children (pack order).
        const int SEG = J <= 8 ? 8 : (J <= 16 ? 16 : 32);
        const int per_warp = 32 / SEG, n_warps = T >> 5, warp = tid >> 5, lane = tid & 31;
        const int sub = lane / SEG, j = lane - sub * SEG;
        const int rounds = J <= 1 ? 0 : 32 - __clz(J - 1);
        for (int w0 = warp * per_warp; w0 < nw; w0 += n_warps * per_warp) {
            const int w = w0 + sub;
            const bool act = j < J && w < nw;
            float X[12] = {1.0f, 0.0f, 0.0f, 0.0f, 1.0f, 0.0f, 0.0f, 0.0f, 1.0f, 0.0f, 0.0f, 0.0f};
            int a = -1;
            if (act) {
                const JointRec& jr = sc.joints[j];
                joint_local(jr, cc_joint_value(jr, B, edge, w), X);
                const int p = jr.idx.x;
                a = (p >= 0 && p < j) ? p : -1;
            }
            for (int r = 0; r < rounds; ++r) {
                const int src = lane - j + max(a, 0);
                float Y[12];
#pragma unroll
                for (int i = 0; i < 12; ++i) Y[i] = __shfl_sync(0xffffffffu, X[i], src);
                const int aa = __shfl_sync(0xffffffffu, a, src);
                if (a >= 0) {
                    compose(Y, X, X);
                    a = aa;
                }
            }
            if (act) {
                float* P = &B.pose[(w * J + j) * 12];
#pragma unroll
                for (int i = 0; i < 12; ++i) P[i] = X[i];
            }
            __syncwarp();
            // C, fused: the segment that composed waypoint w's frames places its
            // sphere centres (warp-local data, so no CTA barrier in between)
            if (w < nw) cc_centres(sc, B, w, j, SEG, J, S, S_pad, K, gated, inflate);
        }
    } else {
        // A: local joint transforms, one (waypoint, joint) per thread
        for (int it = tid; it < nw * J; it += T) {
            const int w = it / J, j = it - w * J;
            const JointRec& jr = sc.joints[j];
            joint_local(jr, cc_joint_value(jr, B, edge, w), &B.pose[(w * J + j) * 12]);
        }
        g.sync();
        // B: chain composition in topological order, one waypoint per thread
        for (int w = tid; w < nw; w += T) {
            float* P = &B.pose[w * J * 12];
            for (int j = 0; j < J; ++j) {
                const int p = sc.joints[j].idx.x;
                if (p >= 0 && p < j) compose(&P[p * 12], &P[j * 12], &P[j * 12]);
            }
        }
        g.sync();
        // C: sphere centres, one (waypoint, sphere) per thread
        for (int it = tid; it < nw * T; it += T) cc_centres(sc, B, it / T, it % T, T, J, S, S_pad, K, gated, inflate);
    }
    g.sync();
    // every thread has read the other word's previous result by now
    if (tid == 0) {
        B.hit[par] = 0u;  // par was flipped: this is the word the next call uses
        B.hit[2] = B.hit[3] = 0u;  // work-list counters
    }
    unsigned long long flops = 0;
    // D: coarse pre-pass -> dirty groups and touching coarse self pairs
    if (gated) {
        const int n_cw = nw * KC * n_parts_c;
        for (int it = tid; it < n_cw + nw * Q; it += T) {
            if (it < n_cw) {
                const int part = it / (nw * KC), r = it - part * (nw * KC);
                const int kc = r / nw, w = r - kc * nw;
                const int k0 = kc * 8, nk = min(8, K - k0);
                float4 s[8];
#pragma unroll
                for (int m = 0; m < 8; ++m) s[m] = m < nk ? B.cctr[w * K + k0 + m] : absent_sphere();
                const uint32_t hitk =
                    obstacles_vs_spheres<8, true, false>(sc, bounds_c[part], bounds_c[part + 1], s, nk, flops);
                // 8 | 32: a chunk's bits never straddle two words
                if (hitk) atomicOr(&B.dirty[w * KW + (k0 >> 5)], hitk << (k0 & 31));
            } else {
                const int r = it - n_cw;
                const int qq = r / nw, w = r - qq * nw;
                const int2 cp = sc.cpair[qq];
                if (cp.x < 0 || cp.y < 0 || cp.x >= K || cp.y >= K) continue;
                const float4 a = B.cctr[w * K + cp.x], b = B.cctr[w * K + cp.y];
                const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
                const float t = a.w + b.w - inflate;
                if (fmaf(dx, dx, fmaf(dy, dy, dz * dz)) <= t * t) atomicOr(&B.gate[w * QW + (qq >> 5)], 1u << (qq & 31));
                flops += kFlopPairExplicit;
            }
        }
        g.sync();
    }
    // E0 (gated early-exit checks): the coarse pass leaves only a few (sphere
    // chunk, waypoint) pairs dirty and a few self items touching, and dealing all
    // items out by index gave the few threads holding real work a long tail that
    // the rest of the CTA waited for at the final barrier.  Compact the live
    // pairs and items into lists (in `pose`, free once the centres are placed),
    // then spread them: every dirty pair's obstacle list is cut into n_sub
    // cost-balanced ranges so that the world work makes about two items per
    // thread.
    const bool compact = gated && !full_sweep && nw * (h.n_sch + h.n_items) <= B.listcap;
    int* wl = reinterpret_cast<int*>(B.pose);  // (sphere chunk << 8 | waypoint) of dirty pairs
    int* sl = wl + nw * h.n_sch;               // (self item << 8 | waypoint) of touching items
    if (compact) {
        for (int i = tid; i < nw * h.n_sch; i += T) {
            const int si = i / nw, w = i - si * nw;
            const int4 ch = sc.sch[si];
            if (ch.z < 0 || (B.dirty[w * KW + (ch.z >> 5)] & (1u << (ch.z & 31)))) wl[atomicAdd(&B.hit[2], 1u)] = (si << 8) | w;
        }
        for (int i = tid; i < nw * h.n_items; i += T) {
            const int ii = i / nw, w = i - ii * nw;
            const int4 item = sc.item[ii];
            if (item.w < 0 || (B.gate[w * QW + (item.w >> 5)] & (1u << (item.w & 31)))) sl[atomicAdd(&B.hit[3], 1u)] = (ii << 8) | w;
        }
        g.sync();
    }
    const int Lw = compact ? (int)B.hit[2] : 0, Ls = compact ? (int)B.hit[3] : 0;
    const int n_sub = Lw > 0 ? min(max(1, cdiv(2 * T, Lw)), max(1, cdiv(n_obs, 4))) : 0;
    // E: fine work items.  World: (obstacle chunk, sphere chunk, waypoint) with the
    // obstacle chunk slowest so a warp reads the same primitive (broadcast); from
    // the list: (obstacle range, list entry), range slowest.  Self: (item,
    // waypoint), or the listed ones.
    const int n_world = compact ? Lw * n_sub : nw * h.n_sch * n_parts;
    const int n_self = compact ? Ls : nw * h.n_items;
    const int n_total = n_world + n_self + (sc.pc.n > 0 ? nw * S : 0);
    auto run_item = [&](int it) {
        int w;
        bool hit = false;
        if (it < n_world) {
            int si, j0, j1;
            if (compact) {
                const int p = it / Lw, ent = wl[it - p * Lw];
                si = ent >> 8;
                w = ent & 255;
                if (edge_mode ? (*vhit != 0u) : ((*vhit >> w) & 1u)) return;
                j0 = world_index_at(h, (int)((long long)p * ctot / n_sub));
                j1 = world_index_at(h, (int)((long long)(p + 1) * ctot / n_sub));
            } else {
                const int part = it / (nw * h.n_sch), r = it - part * (nw * h.n_sch);
                si = r / nw;
                w = r - si * nw;
                if (!full_sweep && (edge_mode ? (*vhit != 0u) : ((*vhit >> w) & 1u))) return;
                const int4 chk = sc.sch[si];
                if (gated && chk.z >= 0 && !(B.dirty[w * KW + (chk.z >> 5)] & (1u << (chk.z & 31)))) return;
                j0 = B.bounds[part];
                j1 = B.bounds[part + 1];
            }
            const int4 ch = sc.sch[si];
            float4 s[kSphChunk];
#pragma unroll
            for (int m = 0; m < kSphChunk; ++m) s[m] = (m < ch.y) ? B.ctr[w * S_pad + ch.x + m] : absent_sphere();
            hit = (full_sweep ? obstacles_vs_spheres<kSphChunk, true>(sc, j0, j1, s, ch.y, flops)
                              : obstacles_vs_spheres<kSphChunk, false>(sc, j0, j1, s, ch.y, flops)) != 0u;
        } else if (it >= n_world + n_self) {  // point cloud: (sphere, waypoint)
            const int r = it - n_world - n_self;
            const int si = r / nw;
            w = r - si * nw;
            if (!full_sweep && (edge_mode ? (*vhit != 0u) : ((*vhit >> w) & 1u))) return;
            hit = pc_sphere_hits(sc.pc, B.ctr[w * S_pad + si], full_sweep, flops);
        } else {
            const int r = it - n_world;
            int ii;
            if (compact) {
                const int ent = sl[r];
                ii = ent >> 8;
                w = ent & 255;
            } else {
                ii = r / nw;
                w = r - ii * nw;
            }
            if (!full_sweep && (edge_mode ? (*vhit != 0u) : ((*vhit >> w) & 1u))) return;
            const int4 item = sc.item[ii];
            if (!compact && gated && item.w >= 0 && !(B.gate[w * QW + (item.w >> 5)] & (1u << (item.w & 31)))) return;
            const float4* C = &B.ctr[w * S_pad];
            if (item.y >= 0) {  // dense block: spheres [a0, a0+na) x [b0, b0+nb)
                // self pairs use radius rho = r + inflate/2 per sphere, so the pair
                // threshold is r_i + r_j + inflate
                const int na = item.z >> 16, nb = item.z & 0xffff;
                const float half = 0.5f * inflate;
                float4 a[kSphChunk];
                float thr[kSphChunk], mn[kSphChunk];
#pragma unroll
                for (int m = 0; m < kSphChunk; ++m) {
                    a[m] = (m < na) ? C[item.x + m] : absent_sphere();
                    a[m].w -= half;
                    thr[m] = -sphere_A(a[m]);
                    mn[m] = INFINITY;
                }
                auto pair_h = [&](float (&v)[kSphChunk], int j) {
                    float4 b = C[item.y + j];
                    b.w -= half;
                    h_sphere<kSphChunk>(v, a, make_float4(-2.0f * b.x, -2.0f * b.y, -2.0f * b.z, -2.0f * b.w),
                                        sphere_A(b));
                };
                // a full sweep folds two partner spheres per three-input
                // minimum; early exit folds one at a time and checks after
                // every four (measured faster for each)
                int bb = 0;
                if constexpr (FULL_SWEEP) {
                    for (; bb + 1 < nb; bb += 2) {
                        float h1[kSphChunk], h2[kSphChunk];
                        pair_h(h1, bb);
                        pair_h(h2, bb + 1);
                        fold2(mn, h1, h2);
                    }
                }
                for (; bb < nb; ++bb) {
                    float h1[kSphChunk];
                    pair_h(h1, bb);
                    fold1(mn, h1);
                    if (!full_sweep && (bb & 3) == 3 && any_le(mn, thr)) { ++bb; break; }
                }
                hit |= any_le(mn, thr);
                flops += (unsigned long long)bb * na * kFlopPair;
            } else {  // explicit pairs [p0, p0+count) of the pair list (global memory)
                const int p1 = min(item.x + item.z, h.P);
                for (int p = item.x; p < p1; ++p) {
                    const int2 pr = __ldg(&sc.pairs[p]);
                    if (pr.x < 0 || pr.y < 0 || pr.x >= S || pr.y >= S) continue;
                    const float4 a = C[pr.x], b = C[pr.y];
                    const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
                    const float t = a.w + b.w - inflate;
                    hit |= fmaf(dx, dx, fmaf(dy, dy, dz * dz)) <= t * t;
                    flops += kFlopPairExplicit;
                    if (hit && !full_sweep) break;
                }
            }
        }
        // one shared-memory atomic per warp: OR the hit bits of the active lanes
        const unsigned active = __activemask();
        // bit w per configuration (nw <= 32 outside edge mode); an edge only needs
        // the word to become non-zero, which bit w & 31 does for chunks of 64
        const unsigned bits = __reduce_or_sync(active, hit ? (1u << (w & 31)) : 0u);
        if (bits && (threadIdx.x & 31) == (__ffs(active) - 1)) atomicOr(hw, bits);
    };
    for (int it = tid; it < n_total; it += T) run_item(it);
    if (B.stats) {
        if (tid == 0) {
            unsigned long long fk = (unsigned long long)nw * (J * (kFlopJointLocal + kFlopJointChain) + S * kFlopXform);
            if (gated) fk += (unsigned long long)nw * K * kFlopXform;
            flops += fk;
            atomicAdd(&B.stats[kStatConfigs], (unsigned long long)nw);
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) flops += __shfl_xor_sync(0xffffffffu, flops, off);
        if ((tid & 31) == 0 && flops) atomicAdd(&B.stats[kStatFlops], flops);
    }
    g.sync();
    return *vhit;
}

}  // namespace prrtc
