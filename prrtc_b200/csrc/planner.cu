// planner.cu -- scene packing, the pRRTC explorer kernel (plain and persistent
// batched launch), output initialisation, device-clock timing and path
// extraction.  sm_100a.
//
// Algorithm: the reference's prrtc_planner_kernel (cuda-rrtc/CUDA/
// prrtc_planner.cu:675-1066).  Each explorer samples its Halton stream, picks a
// tree by balance mode, finds the nearest node, extends by step_size, checks the
// edge, inserts, then connects toward the other tree in ceil(d/step) checked
// sub-edges; the first explorer whose connect completes solves the problem.
//
// B200 design:
//  * an explorer is a CTA of 64-256 threads; nearest neighbour is a CTA scan of
//    the SoA tree with 128-bit L2-coherent loads and a lexicographic (dsq, idx)
//    warp-shuffle argmin (ties to the lowest index);
//  * an edge's waypoints are checked cooperatively by the whole CTA (FK per
//    waypoint, sphere centres, then (waypoint x sphere-chunk x obstacle-chunk)
//    and (waypoint x self-block) work items) against the scene staged in shared
//    memory by one bulk TMA copy;
//  * tree slots are pre-filled with NaN, so a reader scanning [0, tree_size)
//    never uses a half-written node (its squared distance is NaN and loses every
//    comparison); this replaces the reference's `completed` counter as the scan
//    bound, whose count-not-prefix semantics let a reader see an unwritten slot;
//  * the batched form is one persistent launch: CTAs pop (problem, explorer)
//    slots from a queue ordered by the caller (longest problems first).
#include <cuda_runtime.h>
#include <float.h>
#include <limits.h>
#include <math.h>

#include <algorithm>
#include <mutex>

#include "kernels.h"
#include "prrtc_device.cuh"

namespace prrtc {

#ifndef PRRTC_EXPLORE_MINBLOCKS
#define PRRTC_EXPLORE_MINBLOCKS 2  // resident 256-thread explorer CTAs per SM the register allocation must allow
#endif

// ============================================================================ pack

size_t blob_stride(const PackSrc& s) {
    const BlobLayout L = blob_layout(s.J, s.S, s.K, s.Q, s.sp_max, s.ws_max, s.wc_max, s.wb_max, s.wh_max);
    return ((size_t)L.bytes + 255) & ~(size_t)255;
}

__device__ __forceinline__ int clampi(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }

// One CTA per problem.  Converts the reference collision_context buffers into
// the packed blob (see prrtc_device.cuh).  Dynamic shared memory: Q ints.
__global__ void pack_kernel(PackSrc s, unsigned char* blobs, size_t stride, int cap) {
    extern __shared__ int s_dense[];
    const int b = blockIdx.x, tid = threadIdx.x, T = blockDim.x;
    unsigned char* blob = blobs + (size_t)b * stride;
    BlobHeader* h = reinterpret_cast<BlobHeader*>(blob);
    const int Ns = s.ws_cnt ? clampi(s.ws_cnt[b], 0, s.ws_max) : s.ws_max;
    const int Nc = s.wc_cnt ? clampi(s.wc_cnt[b], 0, s.wc_max) : s.wc_max;
    const int Nb = s.wb_cnt ? clampi(s.wb_cnt[b], 0, s.wb_max) : s.wb_max;
    const int Nh = s.wh_cnt ? clampi(s.wh_cnt[b], 0, s.wh_max) : s.wh_max;
    const int P = s.sp_cnt ? clampi(s.sp_cnt[b], 0, s.sp_max) : s.sp_max;
    // a table is batched [B, max, feat] exactly when its count pointer is set
    const float* ws = s.ws + (s.ws_cnt ? (size_t)b * s.ws_max * 4 : 0);
    const float* wc = s.wc + (s.wc_cnt ? (size_t)b * s.wc_max * 7 : 0);
    const float* wbx = s.wb + (s.wb_cnt ? (size_t)b * s.wb_max * 15 : 0);
    const float* wh = s.wh + (s.wh_cnt ? (size_t)b * s.wh_max * 6 : 0);
    const int* sp = s.sp + (s.sp_cnt ? (size_t)b * s.sp_max * 2 : 0);
    const int J = s.J, S = s.S, K = s.K, Q = s.Q;
    const BlobLayout L = blob_layout(J, S, K, Q, s.sp_max, s.ws_max, s.wc_max, s.wb_max, s.wh_max);

    // reference enable rules (prrtc_planner.cu:505-506, 1156-1157, 1173, 741-743)
    const bool enabled =
        J > 0 && J <= kMaxJoints && S > 0 && (Ns > 0 || Nc > 0 || Nb > 0 || Nh > 0 || P > 0 || s.has_cloud);
    const bool coarse_ok = K > 0 && K <= kMaxLinks && s.foff != nullptr;
    bool gated = enabled && coarse_ok && (s.mode == 2 || (s.mode == 3 && J <= 16));

    JointRec* jr = reinterpret_cast<JointRec*>(blob + L.o_joint);
    for (int j = tid; j < J; j += T)
        jr[j] = make_joint_rec(j, s.ptf, s.twists, s.parent, s.act, s.mmul, s.moff, s.mact, s.dim);
    float4* sph = reinterpret_cast<float4*>(blob + L.o_sph);
    int* sfr = reinterpret_cast<int*>(blob + L.o_sfr);
    for (int i = tid; i < S; i += T) {
        sph[i] = make_float4(s.sloc[i * 3], s.sloc[i * 3 + 1], s.sloc[i * 3 + 2], s.srad[i]);
        const int li = s.sli[i];
        int f = (li >= 0 && li < J) ? (s.topo_inv ? s.topo_inv[li] : li) : -1;
        sfr[i] = (f >= 0 && f < J) ? f : -1;
    }
    float4* grp = reinterpret_cast<float4*>(blob + L.o_grp);
    for (int k = tid; k < K; k += T) {
        grp[2 * k] = make_float4(s.cloc[k * 3], s.cloc[k * 3 + 1], s.cloc[k * 3 + 2], s.crad[k]);
        const int li = s.cli[k];
        int f = (li >= 0 && li < J) ? (s.topo_inv ? s.topo_inv[li] : li) : -1;
        if (f >= J) f = -1;
        const int s0 = s.foff ? clampi(s.foff[k], 0, S) : 0;
        const int s1 = s.foff ? clampi(s.foff[k + 1], 0, S) : 0;
        grp[2 * k + 1] = make_float4(__int_as_float(f), __int_as_float(s0), __int_as_float(s1), 0.0f);
    }
    // world primitives, pre-conditioned for the FMA-form tests (prrtc_device.cuh)
    float4* o_ws = reinterpret_cast<float4*>(blob + L.o_ws);
    for (int i = tid; i < Ns; i += T) {
        const float x = ws[i * 4], y = ws[i * 4 + 1], z = ws[i * 4 + 2], r = ws[i * 4 + 3];
        o_ws[2 * i] = make_float4(-2.0f * x, -2.0f * y, -2.0f * z, -2.0f * r);
        o_ws[2 * i + 1] = make_float4(x, y, z, fmaf(x, x, fmaf(y, y, fmaf(z, z, -r * r))));
    }
    float4* o_wc = reinterpret_cast<float4*>(blob + L.o_wc);
    for (int i = tid; i < Nc; i += T) {
        const float* c = &wc[i * 7];
        const float dx = c[3] - c[0], dy = c[4] - c[1], dz = c[5] - c[2];
        const float l2 = dx * dx + dy * dy + dz * dz;
        const float il2 = l2 > 0.0f ? 1.0f / l2 : 0.0f;
        const float px = dx * il2, py = dy * il2, pz = dz * il2;
        o_wc[3 * i] = make_float4(c[0], c[1], c[2], c[6]);
        o_wc[3 * i + 1] = make_float4(px, py, pz, -(px * c[0] + py * c[1] + pz * c[2]));
        o_wc[3 * i + 2] = make_float4(dx, dy, dz, 0.0f);
    }
    float4* o_wb = reinterpret_cast<float4*>(blob + L.o_wb);
    for (int i = tid; i < Nb; i += T) {
        const float* c = &wbx[i * 15];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float ax = c[3 + 3 * k], ay = c[4 + 3 * k], az = c[5 + 3 * k];
            const float off = -(ax * c[0] + ay * c[1] + az * c[2]);
            o_wb[4 * i + k] = make_float4(ax * kBoxInv, ay * kBoxInv, az * kBoxInv, off * kBoxInv);
        }
        o_wb[4 * i + 3] = make_float4(c[12] * kBoxInv, c[13] * kBoxInv, c[14] * kBoxInv, 0.0f);
    }
    float4* o_wh = reinterpret_cast<float4*>(blob + L.o_wh);
    for (int i = tid; i < Nh; i += T) {
        const float* c = &wh[i * 6];
        o_wh[i] = make_float4(c[0], c[1], c[2], -(c[0] * c[3] + c[1] * c[4] + c[2] * c[5]));
    }
    int2* cp = reinterpret_cast<int2*>(blob + L.o_cpair);
    for (int q = tid; q < Q; q += T) cp[q] = make_int2(s.cpairs[2 * q], s.cpairs[2 * q + 1]);
    // dense-block detection: coarse pair q's range is the row-major product of
    // its two groups' fine ranges
    for (int q = tid; q < Q; q += T) {
        int dense = 0;
        if (coarse_ok && s.cranges) {
            const int ci = s.cpairs[2 * q], cj = s.cpairs[2 * q + 1];
            const int r0 = s.cranges[2 * q], r1 = s.cranges[2 * q + 1];
            if (ci >= 0 && cj >= 0 && ci < K && cj < K && r0 >= 0 && r1 <= P && r0 <= r1) {
                const int a0 = clampi(s.foff[ci], 0, S), a1 = clampi(s.foff[ci + 1], 0, S);
                const int b0 = clampi(s.foff[cj], 0, S), b1 = clampi(s.foff[cj + 1], 0, S);
                const int na = a1 - a0, nb = b1 - b0;
                if (na > 0 && nb > 0 && nb <= 0xffff && r1 - r0 == na * nb) {
                    dense = 1;
                    for (int m = 0; m < na * nb && dense; ++m) {
                        const int pi = sp[2 * (r0 + m)], pj = sp[2 * (r0 + m) + 1];
                        if (pi != a0 + m / nb || pj != b0 + m % nb) dense = 0;
                    }
                }
            }
        }
        s_dense[q] = dense;
    }
    __syncthreads();
    if (tid == 0) {
        int4* sch = reinterpret_cast<int4*>(blob + L.o_sch);
        int n_sch = 0;
        if (gated) {
            for (int k = 0; k < K; ++k) {
                const int s0 = clampi(s.foff[k], 0, S), s1 = clampi(s.foff[k + 1], 0, S);
                for (int a = s0; a < s1 && n_sch < L.sch_cap; a += kSphChunk)
                    sch[n_sch++] = make_int4(a, min(kSphChunk, s1 - a), k, 0);
            }
        } else {
            for (int a = 0; a < S && n_sch < L.sch_cap; a += kSphChunk)
                sch[n_sch++] = make_int4(a, min(kSphChunk, S - a), -1, 0);
        }
        int4* item = reinterpret_cast<int4*>(blob + L.o_item);
        int n_items = 0;
        bool use_ranges = gated;
        if (!gated && coarse_ok && s.cranges && Q > 0) {
            // flat checker: reuse the range decomposition when the ranges tile [0, P)
            int cursor = 0;
            use_ranges = true;
            for (int q = 0; q < Q; ++q) {
                if (s.cranges[2 * q] != cursor) { use_ranges = false; break; }
                cursor = s.cranges[2 * q + 1];
            }
            if (cursor != P) use_ranges = false;
        }
        bool overflow = false;
        if (use_ranges) {
            for (int q = 0; q < Q && !overflow; ++q) {
                const int gate = gated ? q : -1;
                const int r0 = clampi(s.cranges[2 * q], 0, P), r1 = clampi(s.cranges[2 * q + 1], 0, P);
                if (s_dense[q]) {
                    const int ci = s.cpairs[2 * q], cj = s.cpairs[2 * q + 1];
                    const int a0 = clampi(s.foff[ci], 0, S), a1 = clampi(s.foff[ci + 1], 0, S);
                    const int b0 = clampi(s.foff[cj], 0, S), b1 = clampi(s.foff[cj + 1], 0, S);
                    for (int a = a0; a < a1; a += kSphChunk) {
                        if (n_items >= L.item_cap) { overflow = true; break; }
                        item[n_items++] = make_int4(a, b0, (min(kSphChunk, a1 - a) << 16) | (b1 - b0), gate);
                    }
                } else {
                    for (int p = r0; p < r1; p += kPairChunk) {
                        if (n_items >= L.item_cap) { overflow = true; break; }
                        item[n_items++] = make_int4(p, -1, min(kPairChunk, r1 - p), gate);
                    }
                }
            }
        }
        if (!use_ranges || overflow) {
            n_items = 0;
            for (int p = 0; p < P; p += kPairChunk) item[n_items++] = make_int4(p, -1, min(kPairChunk, P - p), -1);
            if (overflow) {  // fall back to the flat sweep; verdicts are identical
                gated = false;
            }
        }
        BlobHeader hd;
        hd.J = J; hd.dim = s.dim; hd.S = S; hd.S_pad = odd_pad(S);
        hd.K = K; hd.Q = Q; hd.Ns = Ns; hd.Nc = Nc;
        hd.Nb = Nb; hd.Nh = Nh; hd.n_sch = n_sch; hd.n_items = n_items;
        hd.n_och = cdiv(Ns, kObsChunk) + cdiv(Nc, kObsChunk) + cdiv(Nb, kObsChunk) + cdiv(Nh, kObsChunk);
        hd.gated = gated ? 1 : 0;
        hd.enabled = enabled ? 1 : 0;
        hd.inflate_bits = __float_as_int(s.mode == 1 ? s.margin : 0.0f);
        hd.o_joint = L.o_joint; hd.o_sph = L.o_sph; hd.o_sfr = L.o_sfr; hd.o_grp = L.o_grp;
        hd.o_sch = L.o_sch; hd.o_ws = L.o_ws; hd.o_wc = L.o_wc; hd.o_wb = L.o_wb;
        hd.o_wh = L.o_wh; hd.o_item = L.o_item; hd.o_cpair = L.o_cpair; hd.used_bytes = L.bytes;
        hd.P = P; hd.cap_bytes = cap; hd.error = overflow ? kBlobItemOverflow : 0; hd.pad0 = 0;
        *h = hd;
    }
}

cudaError_t launch_pack(const PackSrc& s, int batch, unsigned char* blobs, size_t stride, cudaStream_t st) {
    if (batch <= 0) return cudaSuccess;
    const size_t smem = (size_t)std::max(s.Q, 1) * sizeof(int);
    pack_kernel<<<batch, 256, smem, st>>>(s, blobs, stride, (int)stride);
    return cudaGetLastError();
}

// ============================================================================ helpers

// ============================================================================ nearest neighbour

// Group-wide argmin of the squared distance from q (shared memory) over nodes
// [0, n) of the SoA tree (row stride N).  dsq = d0*d0, then fma(dd, dd, dsq) in
// dimension order -- bit-identical to the reference's `dsq += diff*diff`
// (prrtc_planner.cu:845-849) under nvcc's default contraction.  Result:
// red_d[0], red_i[0] (INT_MAX when no valid node).
template <class G>
__device__ void group_nearest(const G& grp, const float* __restrict__ tree, int N, int dim, int n, const float* q,
                              float* red_d, int* red_i) {
    const int tid = grp.rank(), T = grp.size();
    float best = INFINITY;
    int bi = INT_MAX;
    float qr[kDimMax];
#pragma unroll
    for (int d = 0; d < kDimMax; ++d) qr[d] = d < dim ? q[d] : 0.0f;
    if ((N & 3) == 0 && (reinterpret_cast<uintptr_t>(tree) & 15) == 0) {
        const int n4 = (n + 3) >> 2;
        const float4* t4 = reinterpret_cast<const float4*>(tree);
        const size_t row4 = (size_t)(N >> 2);
        for (int g = tid; g < n4; g += T) {
            float4 v = __ldcg(t4 + g);
            float dx = __fsub_rn(v.x, qr[0]), dy = __fsub_rn(v.y, qr[0]), dz = __fsub_rn(v.z, qr[0]),
                  dw = __fsub_rn(v.w, qr[0]);
            float ax = __fmul_rn(dx, dx), ay = __fmul_rn(dy, dy), az = __fmul_rn(dz, dz), aw = __fmul_rn(dw, dw);
#pragma unroll
            for (int d = 1; d < kDimMax; ++d) {
                if (d < dim) {
                    v = __ldcg(t4 + d * row4 + g);
                    dx = __fsub_rn(v.x, qr[d]); dy = __fsub_rn(v.y, qr[d]);
                    dz = __fsub_rn(v.z, qr[d]); dw = __fsub_rn(v.w, qr[d]);
                    ax = __fmaf_rn(dx, dx, ax); ay = __fmaf_rn(dy, dy, ay);
                    az = __fmaf_rn(dz, dz, az); aw = __fmaf_rn(dw, dw, aw);
                }
            }
            const int i0 = g << 2;
            if (ax < best && i0 < n) { best = ax; bi = i0; }
            if (ay < best && i0 + 1 < n) { best = ay; bi = i0 + 1; }
            if (az < best && i0 + 2 < n) { best = az; bi = i0 + 2; }
            if (aw < best && i0 + 3 < n) { best = aw; bi = i0 + 3; }
        }
    } else {
        for (int i = tid; i < n; i += T) {
            float dd = __fsub_rn(__ldcg(tree + i), qr[0]);
            float acc = __fmul_rn(dd, dd);
            for (int d = 1; d < dim; ++d) {
                dd = __fsub_rn(__ldcg(tree + (size_t)d * N + i), qr[d]);
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
    const int warp = tid >> 5, lane = tid & 31, nwarp = (T + 31) >> 5;
    if (lane == 0) { red_d[warp] = best; red_i[warp] = bi; }
    grp.sync();
    if (warp == 0) {
        best = lane < nwarp ? red_d[lane] : INFINITY;
        bi = lane < nwarp ? red_i[lane] : INT_MAX;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const float od = __shfl_xor_sync(0xffffffffu, best, off);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
            if (od < best || (od == best && oi < bi)) { best = od; bi = oi; }
        }
        if (lane == 0) { red_d[0] = best; red_i[0] = bi; }
    }
    grp.sync();
}

// ============================================================================ explorer

struct Prob {
    int cap;  // this problem's tree capacity (<= the row stride N)
    float* tree[2];
    int* par[2];
    float* radii[2];
    int* sizes;
    int* completed;
    int* iter_count;
    int* conn;
    int* solved;
    unsigned long long* ts;
};

__device__ __forceinline__ Prob prob_ptrs(const PlanLaunch& L, int b) {
    Prob p;
    p.cap = L.caps ? max(1, min(L.caps[b], L.N)) : L.N;
    const size_t tn = (size_t)L.dim * L.N;
    p.tree[0] = L.tree_a + (size_t)b * tn;
    p.tree[1] = L.tree_b + (size_t)b * tn;
    p.par[0] = L.par_a + (size_t)b * L.N;
    p.par[1] = L.par_b + (size_t)b * L.N;
    p.radii[0] = L.radii + (size_t)b * 2 * L.N;
    p.radii[1] = p.radii[0] + L.N;
    p.sizes = L.sizes + 2 * b;
    p.completed = L.completed + 2 * b;
    p.iter_count = L.iter_count + b;
    p.conn = L.connection + 3 * b;
    p.solved = L.solved + b;
    p.ts = L.tstamp + 2 * b;
    return p;
}

struct ExplorerSmem {
    float sample[kDimMax], base[kDimMax], cand[kDimMax], delta[kDimMax], curr[kDimMax], vec[kDimMax];
    float red_d[32];
    int red_i[32];
    int order[16];
    int halton[kDimMax];
    int stop, t, n_t, n_o, nn, skip, new_idx, n_ext, ext_parent, ext_idx, G1, G2, vamp, cnn, abort_;
    int slot, problem, join_e;
};

// Tail join: once every explorer slot has been taken, a CTA that runs out of
// work picks a problem that is still running -- round-robin over the problems
// from a global ticket -- and runs an extra explorer on it (explorer index
// E + ticket: its own Halton sequence).  The hardest problems of a batch thus
// end with every idle CTA exploring them instead of E explorers and an idle
// GPU.  Returns the problem, or -1 when none is running.
__device__ int tail_join_pick(const PlanLaunch& L, int* e_out) {
    const int k = atomicAdd(&L.queue[2], 1);
    *e_out = L.E + k;
    for (int i = 0; i < L.B; ++i) {
        const int pi = (int)(((long long)k + i) % L.B);
        const int bb = L.order ? L.order[pi] : pi;
        if (ld_volatile(&L.solved[bb]) == 0) return bb;
    }
    return -1;
}

// Edge [base, base+delta] at waypoints t = (k+1)/G (prrtc_planner.cu:899-903).
// The G waypoints are visited in nchunk interleaved passes -- pass c checks
// waypoints c, c+nchunk, c+2*nchunk, ... -- so the first pass already samples
// the whole edge and a colliding edge usually stops after one pass.  The
// verdict (any waypoint in collision) does not depend on the order.
// The waypoints are computed inside the checker's FK step (no staging pass).
template <class Grp>
__device__ bool group_edge_collides(const Grp& grp, const Scene& sc, const CcBufs& B, const float* base,
                                    const float* delta, int G, int CW, int& par) {
    if (B.stats && grp.rank() == 0) atomicAdd(&B.stats[kStatEdges], 1ull);
    const int nchunk = (G + CW - 1) / CW;
    for (int c = 0; c < nchunk; ++c) {
        const int nw = (G - c + nchunk - 1) / nchunk;  // waypoints c, c+nchunk, ... below G
        const EdgeSrc e{base, delta, G, nchunk, c};
        if (cc_chunk<false>(grp, sc, B, nw, true, par, &e) != 0u) return true;
    }
    return false;
}

__device__ __forceinline__ void stamp_end(const Prob& P) {
    atomicCAS(&P.ts[1], 0ull, globaltimer());
}

// One explorer (problem P, index e of E) until the problem terminates or the
// explorer exits.  All threads of the group call it.
template <class Grp>
__device__ void run_explorer(const Grp& grp, const PlanLaunch& L, const Prob& P, const Scene& sc, const CcBufs& B,
                             ExplorerSmem& X, int e) {
    const int tid = grp.rank();
    const int dim = L.dim, N = L.N;
    if (tid == 0) {
        prime_order(e, X.order);
        for (int d = 0; d < kDimMax; ++d) X.halton[d] = 1;
        X.vamp = 0;
        B.hit[0] = B.hit[1] = 0u;  // the checker's two result words
    }
    grp.sync();
    int par = 0;  // which hit word the next checker call uses (same in every thread)
    int local_iter = 0;
    // The per-iteration scalar work runs on warp 0 with one lane per dimension
    // (Halton digits, extend, connect vector); lane 0 does the rest.  Every lane
    // repeats lane 0's arithmetic for its own dimension, so results are the
    // same bits as a sequential loop.
    while (true) {
        ++local_iter;
        if (tid < 32) {
            const int lane = tid;
            int stop = 0, sa = 0, sb = 0;
            if (lane == 0) {
                // the three loads go out together: one round trip, not three
                const int sv = ld_volatile(P.solved);
                sa = ld_volatile(&P.sizes[0]);
                sb = ld_volatile(&P.sizes[1]);
                stop = sv != 0;
                if (!stop && local_iter > L.max_iter) {
                    if (atomicCAS(P.solved, 0, -1) == 0) stamp_end(P);
                    atomicMax(P.iter_count, local_iter);
                    stop = 1;
                }
            }
            stop = __shfl_sync(0xffffffffu, stop, 0);
            if (!stop) {
                if (lane < dim) {  // halton_sample, one dimension per lane
                    const float val = halton_next(X.order[lane & 15], X.halton[lane]);
                    X.sample[lane] = __fmaf_rn(val, __fsub_rn(L.hi[lane], L.lo[lane]), L.lo[lane]);
                }
                if (lane == 0) {
                    const int t = choose_tree(L.balance_mode, local_iter, e % L.E, L.E, sa, sb, L.tree_ratio, X.vamp);
                    X.t = t;
                    X.n_t = min(t == 0 ? sa : sb, P.cap);
                }
            }
            if (lane == 0) X.stop = stop;
        }
        grp.sync();
        if (X.stop) break;
        const int t = X.t, o = 1 - t;
        group_nearest(grp, P.tree[t], N, dim, X.n_t, X.sample, X.red_d, X.red_i);
        if (tid < 32) {
            const int lane = tid;
            const int nn = X.red_i[0];
            int skip = nn == INT_MAX;
            if (!skip) {
                // radius and node loads issued together (one round trip)
                const float rad = L.dd ? __ldcg(&P.radii[t][nn]) : 0.0f;
                const float bv = lane < dim ? __ldcg(&P.tree[t][(size_t)lane * N + nn]) : 0.0f;
                const float nd = __fsqrt_rn(X.red_d[0]);
                skip = L.dd && (rad < nd);
                if (!skip) {
                    const float scl = nd > 1e-8f ? fminf(1.0f, __fdiv_rn(L.step, nd)) : 1.0f;
                    if (lane < dim) {
                        X.base[lane] = bv;
                        const float c = __fmaf_rn(__fsub_rn(X.sample[lane], bv), scl, bv);
                        X.cand[lane] = c;
                        X.delta[lane] = __fsub_rn(c, bv);
                    }
                    __syncwarp();
                    if (lane == 0) X.G1 = edge_waypoints(X.delta, dim, L.granularity, L.edge_res);
                }
            }
            if (lane == 0) {
                if (L.stats) atomicAdd(&L.stats[kStatNnNodes], (unsigned long long)X.n_t);
                X.nn = nn;
                X.skip = skip;
            }
        }
        grp.sync();
        if (X.skip) continue;
        if (group_edge_collides(grp, sc, B, X.base, X.delta, X.G1, L.cw, par)) {
            if (tid == 0 && L.dd) radius_shrink(P.radii[t], X.nn, L.dd_alpha, L.dd_radius, L.dd_min_radius, &L.queue[1]);
            continue;
        }
        // insert (prrtc_planner.cu:925-947).  The other tree's size for the
        // connect scan is read together with the slot claim (one round trip
        // instead of two; any node published by then is scanned, as in the
        // reference's read after its insert).  The nearest node's radius grows
        // on another warp while the connect scan runs: nothing in this
        // iteration reads it.
        if (tid == 0) {
            const int so = ld_volatile(&P.sizes[o]);
            const int idx = atomicAdd(&P.sizes[t], 1);
            if (idx >= P.cap) {
                if (atomicCAS(P.solved, 0, -1) == 0) stamp_end(P);
                X.new_idx = -1;
            } else {
                P.par[t][idx] = X.nn;
                X.new_idx = idx;
            }
            X.n_o = min(so, P.cap);
        }
        grp.sync();
        if (X.new_idx < 0) break;
        if (tid < dim) __stcg(&P.tree[t][(size_t)tid * N + X.new_idx], X.cand[tid]);
        if (tid == 0) atomicAdd(&P.completed[t], 1);
        if (L.dd && tid == (grp.size() > 32 ? 32 : 0)) radius_grow(P.radii[t], X.nn, L.dd_alpha, &L.queue[1]);
        // connect (prrtc_planner.cu:949-1043); group_nearest's first barrier
        // follows the scan, so X.cand / X.n_o written above are visible
        group_nearest(grp, P.tree[o], N, dim, X.n_o, X.cand, X.red_d, X.red_i);
        if (tid < 32) {
            const int lane = tid;
            const int cnn = X.red_i[0];
            int n_ext = 0;
            if (cnn != INT_MAX) {
                const float cd = __fsqrt_rn(X.red_d[0]);
                if (L.step > 1e-8f && cd > 1e-8f) n_ext = (int)ceilf(__fdiv_rn(cd, L.step));
                if (lane < dim) {
                    const float c = X.cand[lane];
                    X.curr[lane] = c;
                    X.vec[lane] = n_ext > 0 ? __fdiv_rn(__fsub_rn(__ldcg(&P.tree[o][(size_t)lane * N + cnn]), c),
                                                        (float)n_ext)
                                            : 0.0f;
                }
                __syncwarp();
                if (lane == 0) X.G2 = edge_waypoints(X.vec, dim, L.granularity, L.edge_res);
            } else {
                n_ext = -1;
            }
            if (lane == 0) {
                if (L.stats) atomicAdd(&L.stats[kStatNnNodes], (unsigned long long)X.n_o);
                X.cnn = cnn;
                X.n_ext = n_ext;
                X.ext_parent = X.new_idx;
                X.abort_ = 0;
            }
        }
        grp.sync();
        bool failed = X.n_ext < 0;
        const int n_ext = X.n_ext;
        for (int ext = 0; ext < n_ext && !failed; ++ext) {
            if (X.abort_) { failed = true; break; }
            if (group_edge_collides(grp, sc, B, X.curr, X.vec, X.G2, L.cw, par)) { failed = true; break; }
            if (tid < 32) {
                const int lane = tid;
                int eidx = 0;
                if (lane == 0) {
                    // whether another explorer solved the problem meanwhile, read with the claim
                    X.abort_ = ld_volatile(P.solved) != 0;
                    eidx = atomicAdd(&P.sizes[t], 1);
                }
                eidx = __shfl_sync(0xffffffffu, eidx, 0);
                if (eidx >= P.cap) {
                    if (lane == 0) {
                        if (atomicCAS(P.solved, 0, -1) == 0) stamp_end(P);
                        X.ext_idx = -1;
                    }
                } else {
                    if (lane < dim) X.curr[lane] = __fadd_rn(X.curr[lane], X.vec[lane]);
                    if (lane == 0) {
                        P.par[t][eidx] = X.ext_parent;
                        X.ext_parent = eidx;
                        X.ext_idx = eidx;
                    }
                }
            }
            grp.sync();
            if (X.ext_idx < 0) { failed = true; break; }
            if (tid < dim) __stcg(&P.tree[t][(size_t)tid * N + X.ext_idx], X.curr[tid]);
            if (tid == 0) atomicAdd(&P.completed[t], 1);
            // no barrier: the next sub-edge check only reads X.curr / X.vec, and
            // warp 0 next writes them after that check's barriers
        }
        if (!failed) {  // connection found (prrtc_planner.cu:1045-1062)
            if (tid == 0) {
                if (atomicCAS(P.solved, 0, 1) == 0) {
                    if (t == 0) { P.conn[0] = X.ext_parent; P.conn[1] = X.cnn; }
                    else { P.conn[0] = X.cnn; P.conn[1] = X.ext_parent; }
                    P.conn[2] = t;
                    stamp_end(P);
                }
                atomicMax(P.iter_count, local_iter);
            }
            break;
        }
    }
    grp.sync();
}

// Plain form: grid = E explorers of problem blockIdx.y.  Persistent form: CTAs
// pop (problem, explorer) slots until the queue is empty.
__global__ void __launch_bounds__(256, PRRTC_EXPLORE_MINBLOCKS) explore_kernel(PlanLaunch L) {
    extern __shared__ __align__(128) unsigned char dsm[];
    __shared__ ExplorerSmem X;
    __shared__ __align__(8) uint64_t mbar;
    const int tid = threadIdx.x;
    const bool staged = L.blob_cap > 0;
    unsigned char* blob_sm = dsm;
    CcBufs B = cc_bufs(dsm + (staged ? L.blob_cap : 0), L.J, L.S, L.K, L.Q, L.cw);
    B.stats = L.stats;
    if (tid == 0) mbar_init(&mbar);
    __syncthreads();
    uint32_t phase = 0;
    int cur = -1;
    Scene sc;
    const int total = L.persistent ? L.B * L.E : 1;
    for (int iter = 0;; ++iter) {
        int b, e;
        if (L.persistent) {
            if (tid == 0) {
                int slot = atomicAdd(&L.queue[0], 1);
                // skip the explorers of problems that already terminated
                while (slot < total) {
                    const int pi = slot / L.E;
                    const int bb = L.order ? L.order[pi] : pi;
                    if (ld_volatile(&L.solved[bb]) == 0) break;
                    slot = atomicAdd(&L.queue[0], 1);
                }
                X.slot = slot;
                X.problem = -1;
                if (slot >= total && L.tail_join) X.problem = tail_join_pick(L, &X.join_e);
            }
            __syncthreads();
            const int slot = X.slot;
            if (slot < total) {
                const int pi = slot / L.E;
                b = L.order ? L.order[pi] : pi;
                e = slot - pi * L.E;
            } else {
                if (X.problem < 0) break;
                b = X.problem;
                e = X.join_e;
            }
        } else {
            if (iter > 0) break;
            b = blockIdx.y;
            e = blockIdx.x;
        }
        const unsigned char* gblob = L.blobs + (size_t)b * L.blob_stride;
        if (b != cur) {
            if (staged) {
                const int bytes = reinterpret_cast<const BlobHeader*>(gblob)->used_bytes;
                if (!stage_blob(blob_sm, gblob, min(bytes, L.blob_cap), &mbar, phase, &L.queue[1], 1,
                                L.wait_polls == 0 ? kWaitLimit : max(L.wait_polls, 0)))
                    break;
                sc = scene_view(blob_sm);
            } else {
                sc = scene_view(gblob);
            }
            sc.pairs = reinterpret_cast<const int2*>(L.pairs) + (size_t)b * L.pairs_stride;
            sc.pc = L.pc;
            cur = b;
        }
        const Prob P = prob_ptrs(L, b);
        if (L.persistent && tid == 0) atomicCAS(&P.ts[0], 0ull, globaltimer());
        run_explorer(CtaGroup{}, L, P, sc, B, X, e);
    }
}

// Slot initialisation (the reference's memsets and FLT_MAX fill,
// prrtc_planner.cu:1192-1202, 85-95): slots [0, cap_b) of problem b's rows --
// two trees of dim rows, two parent rows, two radius rows -- become
// 0xFFFFFFFF in the trees and parents (a NaN tree slot, skipped by the
// nearest-neighbour scan until written; parent -1) and FLT_MAX in the radii
// (unset).  Only the problem's own
// capacity is written; words [cap_b, N) of its rows are never read by the
// planner and keep whatever they held.  A CTA writes 16 KB chunks of one row
// (uint4 stores when every row starts 16-byte aligned, N % 4 == 0); blockIdx.y
// strides over problems, blockIdx.x over a problem's (row, chunk) items.
constexpr int kFillChunk = 4096;  // 32-bit words per fill item

__device__ __forceinline__ uint32_t* fill_row(const PlanLaunch& L, int b, int r) {
    const size_t N = (size_t)L.N;
    if (r < L.dim) return reinterpret_cast<uint32_t*>(L.tree_a) + ((size_t)b * L.dim + r) * N;
    r -= L.dim;
    if (r < L.dim) return reinterpret_cast<uint32_t*>(L.tree_b) + ((size_t)b * L.dim + r) * N;
    r -= L.dim;
    if (r == 0) return reinterpret_cast<uint32_t*>(L.par_a) + (size_t)b * N;
    if (r == 1) return reinterpret_cast<uint32_t*>(L.par_b) + (size_t)b * N;
    return reinterpret_cast<uint32_t*>(L.radii) + ((size_t)b * 2 + (r - 2)) * N;
}

__global__ void __launch_bounds__(256) fill_kernel(PlanLaunch L) {
    const int rows = 2 * L.dim + 4;
    const bool vec = (L.N & 3) == 0;
    for (int b = blockIdx.y; b < L.B; b += gridDim.y) {
        const int cap = L.caps ? max(1, min(L.caps[b], L.N)) : L.N;
        const int chunks = (cap + kFillChunk - 1) / kFillChunk;
        for (int it = blockIdx.x; it < rows * chunks; it += gridDim.x) {
            const int r = it / chunks, c0 = (it - r * chunks) * kFillChunk;
            const int c1 = min(cap, c0 + kFillChunk);
            uint32_t* row = fill_row(L, b, r);
            const uint32_t w = r >= 2 * L.dim + 2 ? 0x7f7fffffu : ~0u;  // FLT_MAX radii, else all ones
            if (vec) {
                // c0 is a multiple of 4; the last vector may pass cap but stays
                // inside the row (N % 4 == 0), in words nobody reads
                uint4* v = reinterpret_cast<uint4*>(row + c0);
                const int n4 = (c1 - c0 + 3) >> 2;
                for (int k = threadIdx.x; k < n4; k += blockDim.x) v[k] = make_uint4(w, w, w, w);
            } else {
                for (int k = c0 + threadIdx.x; k < c1; k += blockDim.x) row[k] = w;
            }
        }
    }
}

// Roots and counters (prrtc_planner.cu:97-125, 1204-1237).  Tree slots,
// parents and radii of [0, cap_b) were set (NaN / -1 / FLT_MAX) by fill_kernel
// before.
__global__ void init_kernel(PlanLaunch L, int stamp_start) {
    const int b = blockIdx.x, tid = threadIdx.x;
    if (b >= L.B) return;
    const Prob P = prob_ptrs(L, b);
    int G = L.num_goals;
    if (L.goal_counts) G = max(1, min(L.goal_counts[b], L.num_goals));
    G = min(G, P.cap);
    const float* st = L.starts + (size_t)b * L.dim;
    const float* gl = L.goals + (size_t)b * L.num_goals * L.dim;
    for (int d = tid; d < L.dim; d += blockDim.x) P.tree[0][(size_t)d * L.N] = st[d];
    for (int i = tid; i < G * L.dim; i += blockDim.x) {
        const int g = i / L.dim, d = i - g * L.dim;
        P.tree[1][(size_t)d * L.N + g] = gl[g * L.dim + d];
    }
    for (int g = tid; g < G; g += blockDim.x) P.par[1][g] = g;
    if (tid == 0) {
        P.par[0][0] = 0;
        P.sizes[0] = 1; P.sizes[1] = G;
        P.completed[0] = 1; P.completed[1] = G;
        P.iter_count[0] = 0;
        P.conn[0] = -1; P.conn[1] = -1; P.conn[2] = -1;
        P.solved[0] = 0;
        P.ts[0] = stamp_start ? globaltimer() : 0ull;
        P.ts[1] = 0ull;
    }
    if (b == 0 && tid == 0) { L.queue[0] = 0; L.queue[1] = 0; L.queue[2] = 0; }
}

__global__ void finalize_kernel(PlanLaunch L) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= L.B) return;
    const unsigned long long t0 = L.tstamp[2 * b], t1 = L.tstamp[2 * b + 1];
    L.ktime[b] = (t1 > t0 && t0 != 0ull) ? (float)((double)(t1 - t0) * 1e-6) : 0.0f;
    // a device wait ran out somewhere in the launch: problems left open are
    // reported as -2 instead of the "still running" 0
    if (L.queue[1] != 0 && L.solved[b] == 0) L.solved[b] = -2;
}

size_t plan_workspace_bytes(int B, int N, size_t blob_stride) {
    size_t b = 0;
    b += (size_t)B * blob_stride;
    b += ((size_t)B * 2 * N * sizeof(float) + 255) & ~(size_t)255;
    b += ((size_t)B * 2 * sizeof(unsigned long long) + 255) & ~(size_t)255;
    b += 256;
    return b;
}

void plan_carve_workspace(PlanLaunch& L, void* ws, size_t stride) {
    unsigned char* p = static_cast<unsigned char*>(ws);
    L.blobs = p;
    L.blob_stride = stride;
    p += (size_t)L.B * stride;
    L.radii = reinterpret_cast<float*>(p);
    p += ((size_t)L.B * 2 * L.N * sizeof(float) + 255) & ~(size_t)255;
    L.tstamp = reinterpret_cast<unsigned long long*>(p);
    p += ((size_t)L.B * 2 * sizeof(unsigned long long) + 255) & ~(size_t)255;
    L.queue = reinterpret_cast<int32_t*>(p);
}

int device_sm_count() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 1;
}

size_t device_max_smem() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return (size_t)n;
}

// explore_kernel's attributes as last set in one device's CUDA context.
struct ExploreAttrs {
    unsigned long long ctx = 0ull;  // context key (current_context_key)
    int max_dyn = -1;          // largest MaxDynamicSharedMemorySize set
    int carve = INT_MIN;       // carve-out preference set (-1 = none)
    bool have_smem = false;    // the three sizes below are known
    int sm_smem = 0, reserved = 0;
    size_t static_smem = 0;
};
constexpr int kMaxCachedDevices = 256;
static ExploreAttrs g_explore_attr[kMaxCachedDevices];
static std::mutex g_explore_attr_mutex;

// An optional timing event on the stream; inside a stream capture it becomes an
// external event-record node, which records each time the graph runs.
static cudaError_t record_event(cudaEvent_t ev, cudaStream_t st) {
    if (!ev) return cudaSuccess;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(st, &cs);
    if (e != cudaSuccess) return e;
    return cs == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal)
                                               : cudaEventRecord(ev, st);
}

cudaError_t launch_plan(PlanLaunch& L, cudaStream_t st) {
    cudaError_t e;
    {
        // enough fill CTAs for about four per SM in total, at least 16 per problem
        const int gy = std::min(L.B, 65535);
        const int gx = std::max(16, (4 * device_sm_count() + gy - 1) / gy);
        fill_kernel<<<dim3(gx, gy), 256, 0, st>>>(L);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    init_kernel<<<L.B, 128, 0, st>>>(L, L.persistent ? 0 : 1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;

    const size_t cc = (size_t)cc_smem_bytes(L.J, L.S, L.K, L.Q, L.cw);
    const size_t max_smem = device_max_smem();
    const size_t static_smem = sizeof(ExplorerSmem) + 64;
    size_t dyn = cc + (size_t)L.blob_cap;
    if (dyn + static_smem > max_smem) {  // scene too large to stage: read it from global memory
        L.blob_cap = 0;
        dyn = cc;
    }
    // ctas_per_sm > 0: the smallest shared-memory carve-out that holds that many
    // CTAs, so the rest of the SM's unified L1 / shared memory is L1 (the
    // explorers read trees, radii and unstaged scene data through it); measured
    // faster than the largest carve-out's one more resident CTA per SM (-1: no
    // preference).  The kernel's attributes are set only when they change, from
    // a cache per device and CUDA context: querying or setting them while the
    // previous batch's planner still ran measured as a host-side wait for that
    // launch, which serialised back-to-back calls (e2e 134 K against 198 K
    // plans/s with a carve-out set on every call).
    {
        int dev = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        const unsigned long long ctx = current_context_key();
        std::lock_guard<std::mutex> lock(g_explore_attr_mutex);
        ExploreAttrs dflt;
        ExploreAttrs& c = (dev >= 0 && dev < kMaxCachedDevices) ? g_explore_attr[dev] : dflt;
        if (!ctx || c.ctx != ctx) {
            c = ExploreAttrs{};
            c.ctx = ctx;
        }
        if ((int)dyn > c.max_dyn) {
            if ((e = cudaFuncSetAttribute(explore_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn)) !=
                cudaSuccess)
                return e;
            c.max_dyn = (int)dyn;
        }
        int carve = -1;
        if (L.persistent && L.ctas_per_sm > 0) {
            if (!c.have_smem) {
                cudaFuncAttributes fa;
                if ((e = cudaDeviceGetAttribute(&c.sm_smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) !=
                        cudaSuccess ||
                    (e = cudaDeviceGetAttribute(&c.reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev)) !=
                        cudaSuccess ||
                    (e = cudaFuncGetAttributes(&fa, explore_kernel)) != cudaSuccess)
                    return e;
                c.static_smem = fa.sharedSizeBytes;
                c.have_smem = true;
            }
            const size_t need = (size_t)L.ctas_per_sm * (dyn + c.static_smem + (size_t)c.reserved);
            carve = c.sm_smem > 0 ? (int)std::min<size_t>(100, (100 * need + c.sm_smem - 1) / (size_t)c.sm_smem) : -1;
        }
        if (carve != c.carve) {
            if ((e = cudaFuncSetAttribute(explore_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, carve)) !=
                cudaSuccess)
                return e;
            c.carve = carve;
        }
    }
    if (L.persistent) {
        int per_sm = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, explore_kernel, L.threads, dyn)) !=
            cudaSuccess)
            return e;
        per_sm = std::max(per_sm, 1);
        if (L.ctas_per_sm > 0) per_sm = std::min(per_sm, L.ctas_per_sm);
        long long grid = (long long)per_sm * device_sm_count();
        if (L.resident > 0) grid = std::min<long long>(grid, L.resident);
        // no more CTAs than explorer slots: with several batches in flight (one per
        // capacity bucket) a full-GPU grid per launch measured slower, its CTAs
        // piling extra explorers onto a few problems
        grid = std::min<long long>(grid, (long long)L.B * L.E);
        if ((e = record_event(L.explore_events[0], st)) != cudaSuccess) return e;
        explore_kernel<<<(unsigned)std::max<long long>(grid, 1), L.threads, dyn, st>>>(L);
    } else {
        if ((e = record_event(L.explore_events[0], st)) != cudaSuccess) return e;
        explore_kernel<<<dim3(L.E, L.B), L.threads, dyn, st>>>(L);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = record_event(L.explore_events[1], st)) != cudaSuccess) return e;
    finalize_kernel<<<(L.B + 127) / 128, 128, 0, st>>>(L);
    return cudaGetLastError();
}

// ============================================================================ path extraction

// One CTA (32 threads) per problem: lane 0 walks the parent chains
// (prrtc.py:603-640), all lanes copy configurations; cost = sum of segment norms.
__global__ void extract_paths_kernel(int B, int dim, int N, const float* ta, const float* tb, const int32_t* pa,
                                     const int32_t* pb, const int32_t* conn, const int32_t* solved, int max_len,
                                     float* paths, int32_t* lengths, float* costs) {
    const int b = blockIdx.x, lane = threadIdx.x;
    extern __shared__ int chain[];  // max_len entries: node index, negative = tree B (-1 - idx)
    __shared__ int s_len;
    const float* TA = ta + (size_t)b * dim * N;
    const float* TB = tb + (size_t)b * dim * N;
    const int32_t* PA = pa + (size_t)b * N;
    const int32_t* PB = pb + (size_t)b * N;
    if (lane == 0) {
        int len = 0;
        if (solved[b] == 1) {
            const int a = conn[3 * b], c = conn[3 * b + 1];
            if (a >= 0 && c >= 0 && a < N && c < N) {
                int na = 0, curr = a;
                for (int it = 0; it < N; ++it) {  // count tree-A chain
                    ++na;
                    const int p = PA[curr];
                    if (p == curr || p < 0 || p >= N) break;
                    curr = p;
                }
                if (na > max_len) len = -1;
                else {
                    curr = a;
                    for (int i = na - 1; i >= 0; --i) {
                        chain[i] = curr;
                        const int p = PA[curr];
                        if (p == curr || p < 0 || p >= N) break;
                        curr = p;
                    }
                    len = na;
                    curr = c;
                    for (int it = 0; it < N; ++it) {
                        if (len >= max_len) { len = -1; break; }
                        chain[len++] = -1 - curr;
                        const int p = PB[curr];
                        if (p == curr || p < 0 || p >= N) break;
                        curr = p;
                    }
                }
            }
        }
        s_len = len;
    }
    __syncthreads();
    const int len = s_len;
    float* out = paths + (size_t)b * max_len * dim;
    for (int i = lane; i < max(len, 0) * dim; i += blockDim.x) {
        const int k = i / dim, d = i - k * dim;
        const int node = chain[k];
        out[i] = node >= 0 ? TA[(size_t)d * N + node] : TB[(size_t)d * N + (-1 - node)];
    }
    __syncthreads();
    float c = 0.0f;
    for (int k = lane; k + 1 < len; k += blockDim.x) {
        float s2 = 0.0f;
        for (int d = 0; d < dim; ++d) {
            const float df = out[(k + 1) * dim + d] - out[k * dim + d];
            s2 = fmaf(df, df, s2);
        }
        c += sqrtf(s2);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
    if (lane == 0) {
        lengths[b] = len;
        costs[b] = len > 0 ? c : INFINITY;
    }
}

cudaError_t launch_extract_paths(int B, int dim, int N, const float* ta, const float* tb, const int32_t* pa,
                                 const int32_t* pb, const int32_t* conn, const int32_t* solved, int max_len,
                                 float* paths, int32_t* lengths, float* costs, cudaStream_t st) {
    const size_t smem = (size_t)max_len * sizeof(int);
    cudaError_t e;
    if (smem > 48 * 1024) {
        if ((e = cudaFuncSetAttribute(extract_paths_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem)) != cudaSuccess)
            return e;
    }
    extract_paths_kernel<<<B, 32, smem, st>>>(B, dim, N, ta, tb, pa, pb, conn, solved, max_len, paths, lengths,
                                              costs);
    return cudaGetLastError();
}

// Result block: one [B,16] int32 row per problem (columns kBlk*), the scalars
// a caller reads back in one copy.  Column kBlkOffset is the exclusive prefix
// sum of the solved path lengths (one CTA, chunks of 1024 problems scanned
// with warp shuffles), or -1 for a problem whose path is not packed: unsolved,
// longer than the path buffer, or past packed_cap waypoints.
__global__ void result_block_kernel(int B, const ResultSrc R, int32_t* block, long long packed_cap) {
    __shared__ long long warp_sum[32];
    __shared__ long long s_carry;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_carry = 0;
    __syncthreads();
    for (int b0 = 0; b0 < B; b0 += blockDim.x) {
        const int b = b0 + tid;
        int len = 0;
        if (b < B) len = (R.solved[b] == 1 && R.lengths[b] > 0) ? R.lengths[b] : 0;
        long long x = len;  // inclusive scan within the warp
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const long long y = __shfl_up_sync(0xffffffffu, x, off);
            if (lane >= off) x += y;
        }
        if (lane == 31) warp_sum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            const int nwarps = blockDim.x >> 5;
            long long v = lane < nwarps ? warp_sum[lane] : 0;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const long long y = __shfl_up_sync(0xffffffffu, v, off);
                if (lane >= off) v += y;
            }
            if (lane < nwarps) warp_sum[lane] = v;  // inclusive over warps
        }
        __syncthreads();
        const long long carry = s_carry;
        const long long excl = carry + (warp > 0 ? warp_sum[warp - 1] : 0) + x - len;
        if (b < B) {
            int32_t* row = block + (size_t)b * 16;
            row[kBlkSizeA] = R.sizes[2 * b];
            row[kBlkSizeB] = R.sizes[2 * b + 1];
            row[kBlkCompletedA] = R.completed[2 * b];
            row[kBlkCompletedB] = R.completed[2 * b + 1];
            row[kBlkIterations] = R.iterations[b];
            row[kBlkConn + 0] = R.conn[3 * b];
            row[kBlkConn + 1] = R.conn[3 * b + 1];
            row[kBlkConn + 2] = R.conn[3 * b + 2];
            row[kBlkSolved] = R.solved[b];
            row[kBlkKernelMs] = __float_as_int(R.kernel_ms[b]);
            row[kBlkLength] = R.lengths[b];
            row[kBlkCost] = __float_as_int(R.costs[b]);
            row[kBlkOffset] = (len > 0 && excl + len <= packed_cap) ? (int32_t)excl : -1;
            row[13] = row[14] = row[15] = 0;
        }
        __syncthreads();
        if (tid == blockDim.x - 1) s_carry = carry + warp_sum[(blockDim.x >> 5) - 1];
        __syncthreads();
    }
}

// Solved paths copied back to back into packed (the offsets of the result
// block), so that a caller reads every path with one contiguous copy.
__global__ void pack_paths_kernel(int B, int dim, int max_len, const float* paths, const int32_t* block,
                                  float* packed) {
    const int b = blockIdx.x;
    const int32_t* row = block + (size_t)b * 16;
    const int off = row[kBlkOffset], len = row[kBlkLength];
    if (off < 0 || len <= 0) return;
    const float* src = paths + (size_t)b * max_len * dim;
    float* dst = packed + (size_t)off * dim;
    for (int i = threadIdx.x; i < len * dim; i += blockDim.x) dst[i] = src[i];
}

cudaError_t launch_result_block(int B, int dim, int max_len, const ResultSrc& R, int32_t* block,
                                const float* paths, float* packed, long long packed_cap, cudaStream_t st) {
    result_block_kernel<<<1, 1024, 0, st>>>(B, R, block, packed ? packed_cap : 0);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || !packed || packed_cap <= 0) return e;
    pack_paths_kernel<<<B, 64, 0, st>>>(B, dim, max_len, paths, block, packed);
    return cudaGetLastError();
}

}  // namespace prrtc
