// smooth.cu -- hand-written adjoint of the post-plan smoothing cost.  sm_100a.
//
// For a path of W waypoints q_w (dim each):
//   C = sum_w sum_pairs softplus_beta(margin - d_pair(q_w)) + w_len * sum_w |q_{w+1} - q_w|^2
// over every (robot sphere, world primitive) pair and every self pair, with
// softplus_beta(x) = log(1 + exp(beta x)) / beta.
//
// Backward pass per waypoint, one warp per waypoint, nothing stored between the
// forward and backward sweeps except per-sphere centres:
//   1. recompute FK (joint-local transforms in parallel over lanes, chain
//      composition on lane 0) and the sphere centres c_s;
//   2. g_s = dC/dc_s from every pair: -sigmoid(beta (m - d)) * dd/dc_s;
//   3. per frame f: G_f = sum g_s, M_f = sum c_s x g_s over its spheres, then
//      folded into parents in reverse topological order (subtree sums);
//   4. joint j with world pose (R_j, t_j) and twist (v, w):
//        dC/dv_j = (R_j w) . (M_j - t_j x G_j) + (R_j v) . G_j
//      (a point p below joint j moves with dp/dv_j = (R_j w) x (p - t_j) + R_j v);
//   5. dC/dq_a = sum over joints driven by a of dv_j/dq_a * dC/dv_j (1 for an
//      actuated joint, mimic_mul for a mimic joint) plus the length term.
#include <cuda_runtime.h>
#include <math.h>

#include "kernels.h"
#include "prrtc_device.cuh"

namespace prrtc {

// softplus_beta(x) and sigmoid(beta x) from one exponential: with z = beta x
// and e = exp(-|z|), softplus_beta = (max(z, 0) + log1p(e)) / beta and
// sigmoid = 1/(1+e) for z >= 0, e/(1+e) otherwise.  Below z = kTailZ a pair
// adds less than exp(kTailZ)/beta (below 1e-15 for beta >= 1) to the cost and
// to every gradient entry; its sigmoid is reported as 0 so that callers can
// skip the gradient scatter.
constexpr float kTailZ = -34.0f;

// log1p(e) for e in [0, 1] without branches: log1p(e) = 2 atanh(s) with
// s = e / (2 + e) in [0, 1/3], and atanh(s) = s + s^3/3 + s^5/5 + ... summed
// to s^15 (the first omitted term is below 1.5e-9 of the sum for s <= 1/3).
__device__ __forceinline__ float log1p_unit(float e) {
    const float s = __fdividef(e, 2.0f + e);
    const float s2 = s * s;
    float p = 1.0f / 15.0f;
    p = fmaf(p, s2, 1.0f / 13.0f);
    p = fmaf(p, s2, 1.0f / 11.0f);
    p = fmaf(p, s2, 1.0f / 9.0f);
    p = fmaf(p, s2, 1.0f / 7.0f);
    p = fmaf(p, s2, 1.0f / 5.0f);
    p = fmaf(p, s2, 1.0f / 3.0f);
    p = fmaf(p, s2, 1.0f);
    return 2.0f * s * p;
}

struct SmoothArgs {
    const unsigned char* blob;
    const int2* pairs;
    size_t blob_stride;   // bytes between the scenes of consecutive paths (0: one scene for every path)
    size_t pairs_stride;  // int2 between the self-pair lists of consecutive paths (0: shared list)
    int J, S, dim;
    const float* wp;
    int P, W;
    float margin, beta, w_len;
    float* cost;
    float* grad;
};

// per-warp shared memory: pose J*12, ctr S*4, g S*4, acc J*8, dv J, q dim (padded)
__host__ __device__ inline int smooth_warp_floats(int J, int S) {
    return (J * 12 + S * 4 + S * 4 + J * 8 + J + kDimMax + 3) & ~3;  // keep every warp slice 16-byte aligned
}

// Accumulate the cost term of a pair at distance d.  sig = sigmoid(beta
// (margin - d)) is the factor of -dd/dc in the gradient (0 for a skipped pair).
__device__ __forceinline__ void pair_term(float d, float margin, float beta, float inv_beta, float& cost,
                                          float& sig) {
    const float z = beta * (margin - d);
    const float e = __expf(-fabsf(z));
    cost = fmaf(fmaxf(z, 0.0f) + log1p_unit(e), inv_beta, cost);
    const float r = __fdividef(1.0f, 1.0f + e);
    sig = z >= kTailZ ? (z >= 0.0f ? r : e * r) : 0.0f;
}

// |v| and 1/|v| (0 and 0 for v = 0) from one reciprocal square root
__device__ __forceinline__ void norm_rnorm(float d2, float& n, float& rn) {
    rn = d2 > 0.0f ? rsqrtf(d2) : 0.0f;
    n = d2 * rn;
}

template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32) smooth_kernel(SmoothArgs a) {
    extern __shared__ __align__(16) float smf[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * WARPS + warp;
    if (c >= a.P * a.W) return;
    const int p = c / a.W, w = c - p * a.W;
    const Scene sc = scene_view(a.blob + (size_t)p * a.blob_stride);
    const int2* pairs = a.pairs + (size_t)p * a.pairs_stride;
    const BlobHeader& h = *sc.h;
    const int J = a.J, S = a.S, dim = a.dim;
    float* base = smf + (size_t)warp * smooth_warp_floats(J, S);
    float* pose = base;
    float4* ctr = reinterpret_cast<float4*>(pose + J * 12);
    float4* g = ctr + S;
    float* acc = reinterpret_cast<float*>(g + S);  // [J][8]: G xyz, M xyz
    float* dv = acc + J * 8;
    float* q = dv + J;
    const float* qw = a.wp + ((size_t)p * a.W + w) * dim;
    if (lane < dim) q[lane] = qw[lane];
    __syncwarp();
    // 1. FK (recomputed) and centres
    for (int j = lane; j < J; j += 32) {
        const JointRec& jr = sc.joints[j];
        joint_local(jr, joint_value(jr, q), &pose[j * 12]);
    }
    __syncwarp();
    if (lane == 0) {
        for (int j = 0; j < J; ++j) {
            const int pj = sc.joints[j].idx.x;
            if (pj >= 0 && pj < j) compose(&pose[pj * 12], &pose[j * 12], &pose[j * 12]);
        }
    }
    __syncwarp();
    for (int s = lane; s < S; s += 32) {
        const int f = sc.sfr[s];
        const float4 l = sc.sph[s];
        ctr[s] = f >= 0 ? xform_point(&pose[f * 12], l) : make_float4(kFar, kFar, kFar, l.w);
        g[s] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    for (int i = lane; i < J * 8; i += 32) acc[i] = 0.0f;
    __syncwarp();
    // 2a. world pairs: one sphere per lane
    float cost = 0.0f;
    const float inv_beta = 1.0f / a.beta;
    for (int s = lane; s < S; s += 32) {
        if (sc.sfr[s] < 0) continue;
        const float4 cs = ctr[s];
        const float r = cs.w;
        float gx = 0.0f, gy = 0.0f, gz = 0.0f;
        for (int o = 0; o < h.Ns; ++o) {
            const float4 o1 = sc.ws[2 * o + 1];
            const float4 ob = make_float4(o1.x, o1.y, o1.z, -0.5f * sc.ws[2 * o].w);
            const float dx = cs.x - ob.x, dy = cs.y - ob.y, dz = cs.z - ob.z;
            float n, rn, sig;
            norm_rnorm(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), n, rn);
            pair_term(n - r - ob.w, a.margin, a.beta, inv_beta, cost, sig);
            const float k = -sig * rn;
            gx = fmaf(k, dx, gx); gy = fmaf(k, dy, gy); gz = fmaf(k, dz, gz);
        }
        for (int o = 0; o < h.Nc; ++o) {
            const float4 p1 = sc.wc[3 * o], dp = sc.wc[3 * o + 1], dl = sc.wc[3 * o + 2];
            const float wx = cs.x - p1.x, wy = cs.y - p1.y, wz = cs.z - p1.z;
            const float t = __saturatef(fmaf(dp.x, cs.x, fmaf(dp.y, cs.y, fmaf(dp.z, cs.z, dp.w))));
            const float ex = fmaf(-t, dl.x, wx), ey = fmaf(-t, dl.y, wy), ez = fmaf(-t, dl.z, wz);
            float n, rn, sig;
            norm_rnorm(fmaf(ex, ex, fmaf(ey, ey, ez * ez)), n, rn);
            pair_term(n - r - p1.w, a.margin, a.beta, inv_beta, cost, sig);
            const float k = -sig * rn;
            gx = fmaf(k, ex, gx); gy = fmaf(k, ey, gy); gz = fmaf(k, ez, gz);
        }
        for (int o = 0; o < h.Nb; ++o) {
            // records are stored scaled by 1/kBoxScale (a power of two): undo exactly
            float4 ax[3] = {sc.wb[4 * o], sc.wb[4 * o + 1], sc.wb[4 * o + 2]};
#pragma unroll
            for (int k = 0; k < 3; ++k)
                ax[k] = make_float4(ax[k].x * kBoxScale, ax[k].y * kBoxScale, ax[k].z * kBoxScale, ax[k].w * kBoxScale);
            float4 hl = sc.wb[4 * o + 3];
            hl = make_float4(hl.x * kBoxScale, hl.y * kBoxScale, hl.z * kBoxScale, 0.0f);
            const float hh[3] = {hl.x, hl.y, hl.z};
            // signed distance to the box without branches: outside, |max(q, 0)|
            // with gradient sum_k sign(l_k) max(q_k, 0)/n a_k; inside, the
            // largest q_k (first axis on ties) with gradient sign(l_k) a_k
            float l[3], qv[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                l[k] = fmaf(ax[k].x, cs.x, fmaf(ax[k].y, cs.y, fmaf(ax[k].z, cs.z, ax[k].w)));
                qv[k] = fabsf(l[k]) - hh[k];
            }
            const float p0 = fmaxf(qv[0], 0.0f), p1 = fmaxf(qv[1], 0.0f), p2 = fmaxf(qv[2], 0.0f);
            const float out2 = fmaf(p0, p0, fmaf(p1, p1, p2 * p2));
            float n, rn;
            norm_rnorm(out2, n, rn);
            const float qmax = fmaxf(qv[0], fmaxf(qv[1], qv[2]));
            const bool outside = out2 > 0.0f;
            const float d = (outside ? n : qmax) - r;
            const bool k0 = qv[0] == qmax, k1 = !k0 && qv[1] == qmax, k2 = !k0 && !k1;
            const float c0 = copysignf(outside ? p0 * rn : (k0 ? 1.0f : 0.0f), l[0]);
            const float c1 = copysignf(outside ? p1 * rn : (k1 ? 1.0f : 0.0f), l[1]);
            const float c2 = copysignf(outside ? p2 * rn : (k2 ? 1.0f : 0.0f), l[2]);
            const float ddx = fmaf(c0, ax[0].x, fmaf(c1, ax[1].x, c2 * ax[2].x));
            const float ddy = fmaf(c0, ax[0].y, fmaf(c1, ax[1].y, c2 * ax[2].y));
            const float ddz = fmaf(c0, ax[0].z, fmaf(c1, ax[1].z, c2 * ax[2].z));
            float sig;
            pair_term(d, a.margin, a.beta, inv_beta, cost, sig);
            gx = fmaf(-sig, ddx, gx); gy = fmaf(-sig, ddy, gy); gz = fmaf(-sig, ddz, gz);
        }
        for (int o = 0; o < h.Nh; ++o) {
            const float4 hs = sc.wh[o];
            const float d = fmaf(hs.x, cs.x, fmaf(hs.y, cs.y, fmaf(hs.z, cs.z, hs.w))) - r;
            float sig;
            pair_term(d, a.margin, a.beta, inv_beta, cost, sig);
            gx = fmaf(-sig, hs.x, gx); gy = fmaf(-sig, hs.y, gy); gz = fmaf(-sig, hs.z, gz);
        }
        g[s] = make_float4(gx, gy, gz, 0.0f);
    }
    __syncwarp();
    // 2b. self pairs (explicit list): shared-memory atomics into both spheres
    for (int k = lane; k < h.P; k += 32) {
        const int2 pr = __ldg(&pairs[k]);
        if (pr.x < 0 || pr.y < 0 || pr.x >= S || pr.y >= S) continue;
        if (sc.sfr[pr.x] < 0 || sc.sfr[pr.y] < 0) continue;
        const float4 ci = ctr[pr.x], cj = ctr[pr.y];
        const float dx = ci.x - cj.x, dy = ci.y - cj.y, dz = ci.z - cj.z;
        float n, rn, sig;
        norm_rnorm(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), n, rn);
        pair_term(n - ci.w - cj.w, a.margin, a.beta, inv_beta, cost, sig);
        if (sig == 0.0f) continue;  // nothing to add
        const float kk = -sig * rn;
        atomicAdd(&g[pr.x].x, kk * dx); atomicAdd(&g[pr.x].y, kk * dy); atomicAdd(&g[pr.x].z, kk * dz);
        atomicAdd(&g[pr.y].x, -kk * dx); atomicAdd(&g[pr.y].y, -kk * dy); atomicAdd(&g[pr.y].z, -kk * dz);
    }
    __syncwarp();
    // 3. frame sums
    for (int s = lane; s < S; s += 32) {
        const int f = sc.sfr[s];
        if (f < 0) continue;
        const float4 cs = ctr[s], gs = g[s];
        float* A = &acc[f * 8];
        atomicAdd(&A[0], gs.x); atomicAdd(&A[1], gs.y); atomicAdd(&A[2], gs.z);
        atomicAdd(&A[3], cs.y * gs.z - cs.z * gs.y);
        atomicAdd(&A[4], cs.z * gs.x - cs.x * gs.z);
        atomicAdd(&A[5], cs.x * gs.y - cs.y * gs.x);
    }
    __syncwarp();
    // 4. reverse sweep
    if (lane == 0) {
        for (int j = J - 1; j >= 0; --j) {
            const JointRec& jr = sc.joints[j];
            const float* F = &pose[j * 12];
            float* A = &acc[j * 8];
            const float wx = fmaf(F[0], jr.tw.x, fmaf(F[1], jr.tw.y, F[2] * jr.tw.z));
            const float wy = fmaf(F[3], jr.tw.x, fmaf(F[4], jr.tw.y, F[5] * jr.tw.z));
            const float wz = fmaf(F[6], jr.tw.x, fmaf(F[7], jr.tw.y, F[8] * jr.tw.z));
            const float vx = fmaf(F[0], jr.tv.x, fmaf(F[1], jr.tv.y, F[2] * jr.tv.z));
            const float vy = fmaf(F[3], jr.tv.x, fmaf(F[4], jr.tv.y, F[5] * jr.tv.z));
            const float vz = fmaf(F[6], jr.tv.x, fmaf(F[7], jr.tv.y, F[8] * jr.tv.z));
            const float tx = F[9], ty = F[10], tz = F[11];
            const float mx = A[3] - (ty * A[2] - tz * A[1]);
            const float my = A[4] - (tz * A[0] - tx * A[2]);
            const float mz = A[5] - (tx * A[1] - ty * A[0]);
            dv[j] = wx * mx + wy * my + wz * mz + vx * A[0] + vy * A[1] + vz * A[2];
            const int pj = jr.idx.x;
            if (pj >= 0 && pj < j) {
                float* B = &acc[pj * 8];
#pragma unroll
                for (int i = 0; i < 6; ++i) B[i] += A[i];
            }
        }
    }
    __syncwarp();
    // 5. joint-space gradient + length term
    float lenc = 0.0f;
    if (lane < dim) {
        float gq = 0.0f;
        for (int j = 0; j < J; ++j) {
            const JointRec& jr = sc.joints[j];
            if (jr.idx.z >= 0) {
                if (jr.idx.z == lane) gq = fmaf(jr.tv.w, dv[j], gq);
            } else if (jr.idx.y == lane) {
                gq += dv[j];
            }
        }
        const float qc = q[lane];
        if (w + 1 < a.W) {
            const float dn = a.wp[((size_t)p * a.W + w + 1) * dim + lane] - qc;
            gq -= 2.0f * a.w_len * dn;
            lenc = a.w_len * dn * dn;
        }
        if (w > 0) {
            const float dp = qc - a.wp[((size_t)p * a.W + w - 1) * dim + lane];
            gq += 2.0f * a.w_len * dp;
        }
        if (a.grad) a.grad[((size_t)p * a.W + w) * dim + lane] = gq;
    }
    cost += lenc;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) cost += __shfl_xor_sync(0xffffffffu, cost, off);
    if (lane == 0) atomicAdd(&a.cost[p], cost);
}

cudaError_t launch_smooth(const unsigned char* blob, size_t blob_stride, const int32_t* pairs, size_t pairs_stride,
                          int J, int S, int dim, const float* wp, int P, int W, float margin, float beta, float w_len,
                          float* cost, float* grad, cudaStream_t st) {
    if (P <= 0 || W <= 0) return cudaSuccess;
    constexpr int WARPS = 4;
    cudaError_t e = cudaMemsetAsync(cost, 0, (size_t)P * sizeof(float), st);
    if (e != cudaSuccess) return e;
    const size_t smem = (size_t)WARPS * smooth_warp_floats(J, S) * sizeof(float);
    if (smem > 48 * 1024) {
        if ((e = cudaFuncSetAttribute(smooth_kernel<WARPS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem)) != cudaSuccess)
            return e;
    }
    SmoothArgs a{blob, reinterpret_cast<const int2*>(pairs), blob_stride, pairs_stride, J, S, dim, wp, P, W,
                 margin, beta, w_len, cost, grad};
    const long long n = (long long)P * W;
    smooth_kernel<WARPS><<<(unsigned)((n + WARPS - 1) / WARPS), WARPS * 32, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace prrtc
