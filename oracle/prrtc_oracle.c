/*
 * prrtc_oracle.c -- CPU restatement of the pRRTC hot path (TEST INFRASTRUCTURE).
 * See prrtc_oracle.h for scope and the reference lines each function follows.
 * Build with -ffp-contract=off: the explicit fmaf() calls below are exactly the
 * contractions nvcc applies to the reference's device expressions.
 */
#include "prrtc_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* Sampling                                                                   */
/* ------------------------------------------------------------------------- */

/* prrtc_planner.cu:144-157 -- radical inverse in float, fraction /= base, one
 * fused multiply-add per digit, state post-incremented. */
float orc_halton_next(int base, int* state) {
    float fraction = 1.0f;
    float result = 0.0f;
    int n = *state;
    while (n > 0) {
        fraction = fraction / (float)base;
        result = fmaf(fraction, (float)(n % base), result);
        n /= base;
    }
    *state = *state + 1;
    return result;
}

/* prrtc_planner.cu:747-758 -- explorer 0 keeps the canonical prime order, every
 * other explorer Fisher-Yates shuffles it with an LCG seeded by its index. */
void orc_prime_order(int explorer, int out16[16]) {
    static const int primes0[16] = {3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59};
    int p[16];
    memcpy(p, primes0, sizeof(p));
    if (explorer != 0) {
        uint32_t rng = (uint32_t)explorer * 1664525u + 1013904223u;
        for (int i = 15; i > 0; --i) {
            rng = rng * 1664525u + 1013904223u;
            const int j = (int)(rng % (uint32_t)(i + 1));
            const int t = p[i];
            p[i] = p[j];
            p[j] = t;
        }
    }
    memcpy(out16, p, sizeof(p));
}

/* prrtc_planner.cu:784-788 -- dimension d uses prime_order[d % 16] and its own
 * state; sample = min + val * (max - min) contracted to one fma. */
void orc_halton_sample(const int prime_order[16], int* states, int dim,
                       const float* lo, const float* hi, float* out) {
    for (int d = 0; d < dim; ++d) {
        const float val = orc_halton_next(prime_order[d % 16], &states[d]);
        out[d] = fmaf(val, hi[d] - lo[d], lo[d]);
    }
}

/* ------------------------------------------------------------------------- */
/* Nearest neighbour / extend                                                 */
/* ------------------------------------------------------------------------- */

/* prrtc_planner.cu:845-849 -- dsq accumulated over d in order; the first term
 * is a plain product, every further term one fma (the reference's
 * `dsq += diff*diff` from 0.0f). */
float orc_dist_sq(const float* tree, int max_nodes, int dim, int idx, const float* q) {
    float diff = tree[idx] - q[0];
    float dsq = diff * diff;
    for (int d = 1; d < dim; ++d) {
        diff = tree[(size_t)d * max_nodes + idx] - q[d];
        dsq = fmaf(diff, diff, dsq);
    }
    return dsq;
}

/* Argmin over [0,n) with NaN slots skipped and ties to the lowest index.  The
 * reference's strided scan + tree reduction (841-862) does not guarantee the
 * lowest index on ties; the B200 kernels do, and so does this restatement. */
int orc_nearest(const float* tree, int max_nodes, int dim, int n, const float* q, float* dsq_out) {
    int best = -1;
    float best_d = INFINITY;
    for (int i = 0; i < n; ++i) {
        const float d = orc_dist_sq(tree, max_nodes, dim, i, q);
        if (d < best_d || (best < 0 && d == best_d)) {
            best_d = d;
            best = i;
        }
    }
    if (dsq_out) *dsq_out = best_d;
    return best;
}

/* prrtc_planner.cu:871-875 -- sc = min(1, step/nd) unless nd <= 1e-8;
 * cand = base + (sample - base) * sc contracted to fma(sample-base, sc, base). */
void orc_extend(const float* base, const float* sample, int dim, float nd, float step, float* cand) {
    const float sc = (nd > 1e-8f) ? fminf(1.0f, step / nd) : 1.0f;
    for (int d = 0; d < dim; ++d) cand[d] = fmaf(sample[d] - base[d], sc, base[d]);
}

/* Edge waypoint count.  resolution <= 0: exactly `granularity` (reference:
 * blockDim.x waypoints, 899).  Otherwise max(granularity, ceil(|delta|/res)). */
int orc_edge_waypoints(const float* delta, int dim, int granularity, float resolution) {
    if (!(resolution > 0.0f)) return granularity;
    float s = delta[0] * delta[0];
    for (int d = 1; d < dim; ++d) s = fmaf(delta[d], delta[d], s);
    const float len = sqrtf(s);
    const int n = (int)ceilf(len / resolution);
    return n > granularity ? n : granularity;
}

/* prrtc_planner.cu:899-903 / 571-572 -- t = (k+1)/G, p = base + t*delta (fma). */
void orc_waypoint(const float* base, const float* delta, int dim, int k, int G, float* out) {
    const float t = (float)(k + 1) / (float)G;
    for (int d = 0; d < dim; ++d) out[d] = fmaf(t, delta[d], base[d]);
}

/* ------------------------------------------------------------------------- */
/* Forward kinematics (restated from the geometry: product of exponentials)    */
/* ------------------------------------------------------------------------- */

#define DEFINE_FK(REAL, SUFFIX, SINF, COSF, SQRTF, EPS)                                   \
    static void quat_to_mat_##SUFFIX(const float* q7, REAL R[9]) {                        \
        REAL w = q7[0], x = q7[1], y = q7[2], z = q7[3];                                   \
        const REAL n = SQRTF(w * w + x * x + y * y + z * z);                                \
        if (n > (REAL)0) { w /= n; x /= n; y /= n; z /= n; } else { w = 1; x = y = z = 0; } \
        R[0] = 1 - 2 * (y * y + z * z); R[1] = 2 * (x * y - w * z); R[2] = 2 * (x * z + w * y); \
        R[3] = 2 * (x * y + w * z); R[4] = 1 - 2 * (x * x + z * z); R[5] = 2 * (y * z - w * x); \
        R[6] = 2 * (x * z - w * y); R[7] = 2 * (y * z + w * x); R[8] = 1 - 2 * (x * x + y * y); \
    }                                                                                      \
    /* SE3 exp of the twist (v, w) scaled by `val`: R = I + A K + B K^2,              */   \
    /* t = (I + B K + C K^2) v with K = [w val]x.                                       */   \
    static void se3_exp_##SUFFIX(const float* tw, REAL val, REAL R[9], REAL t[3]) {        \
        const REAL vx = (REAL)tw[0] * val, vy = (REAL)tw[1] * val, vz = (REAL)tw[2] * val;  \
        const REAL wx = (REAL)tw[3] * val, wy = (REAL)tw[4] * val, wz = (REAL)tw[5] * val;  \
        const REAL th2 = wx * wx + wy * wy + wz * wz;                                       \
        const REAL th = SQRTF(th2);                                                         \
        REAL A, B, C;                                                                       \
        if (th < (REAL)EPS) {                                                               \
            A = 1 - th2 / 6; B = (REAL)0.5 - th2 / 24; C = (REAL)(1.0 / 6.0) - th2 / 120;     \
        } else {                                                                            \
            const REAL s = SINF(th), c = COSF(th);                                          \
            A = s / th; B = (1 - c) / th2; C = (th - s) / (th2 * th);                         \
        }                                                                                   \
        /* K = [[0,-wz,wy],[wz,0,-wx],[-wy,wx,0]];  K^2 = w w^T - th2 I */                  \
        const REAL K[9] = {0, -wz, wy, wz, 0, -wx, -wy, wx, 0};                             \
        const REAL K2[9] = {wx * wx - th2, wx * wy, wx * wz, wy * wx, wy * wy - th2, wy * wz, \
                            wz * wx, wz * wy, wz * wz - th2};                              \
        for (int i = 0; i < 9; ++i) R[i] = A * K[i] + B * K2[i];                            \
        R[0] += 1; R[4] += 1; R[8] += 1;                                                    \
        REAL V[9];                                                                          \
        for (int i = 0; i < 9; ++i) V[i] = B * K[i] + C * K2[i];                            \
        V[0] += 1; V[4] += 1; V[8] += 1;                                                    \
        t[0] = V[0] * vx + V[1] * vy + V[2] * vz;                                           \
        t[1] = V[3] * vx + V[4] * vy + V[5] * vz;                                           \
        t[2] = V[6] * vx + V[7] * vy + V[8] * vz;                                           \
    }                                                                                      \
    /* out = a o b for [R|t] frames stored as 12 reals */                                  \
    static void compose_##SUFFIX(const REAL* a, const REAL* b, REAL* out) {                \
        REAL o[12];                                                                         \
        for (int i = 0; i < 3; ++i) {                                                       \
            for (int j = 0; j < 3; ++j)                                                     \
                o[i * 3 + j] = a[i * 3 + 0] * b[0 * 3 + j] + a[i * 3 + 1] * b[1 * 3 + j] +     \
                               a[i * 3 + 2] * b[2 * 3 + j];                                 \
            o[9 + i] = a[i * 3 + 0] * b[9] + a[i * 3 + 1] * b[10] + a[i * 3 + 2] * b[11] +    \
                       a[9 + i];                                                            \
        }                                                                                   \
        memcpy(out, o, sizeof(o));                                                          \
    }                                                                                      \
    static REAL joint_value_##SUFFIX(const OrcScene* sc, int j, const REAL* q) {            \
        if (sc->mimic_act_idx && sc->mimic_act_idx[j] >= 0)                                 \
            return (REAL)sc->mimic_mul[j] * q[sc->mimic_act_idx[j]] + (REAL)sc->mimic_off[j]; \
        if (sc->act_idx[j] >= 0) return q[sc->act_idx[j]];                                  \
        return 0;                                                                           \
    }                                                                                      \
    static void fk_sorted_##SUFFIX(const OrcScene* sc, const REAL* q, REAL* W) {             \
        const int J = sc->n_joints;                                                         \
        for (int j = 0; j < J; ++j) {                                                       \
            REAL P[12], E[12], L[12];                                                       \
            quat_to_mat_##SUFFIX(&sc->parent_tf[j * 7], P);                                  \
            P[9] = sc->parent_tf[j * 7 + 4];                                                \
            P[10] = sc->parent_tf[j * 7 + 5];                                               \
            P[11] = sc->parent_tf[j * 7 + 6];                                               \
            se3_exp_##SUFFIX(&sc->twists[j * 6], joint_value_##SUFFIX(sc, j, q), E, E + 9);  \
            compose_##SUFFIX(P, E, L);                                                      \
            const int p = sc->parent_idx[j];                                                \
            if (p >= 0 && p < j) compose_##SUFFIX(&W[p * 12], L, &W[j * 12]);               \
            else memcpy(&W[j * 12], L, sizeof(L));                                          \
        }                                                                                   \
    }

DEFINE_FK(double, f64, sin, cos, sqrt, 1e-8)
DEFINE_FK(float, f32, sinf, cosf, sqrtf, 1e-4f)

void orc_fk_f64(const OrcScene* sc, const double* q, double* frames) {
    const int J = sc->n_joints;
    double W[ORC_MAX_JOINTS * 12];
    fk_sorted_f64(sc, q, W);
    for (int k = 0; k < J; ++k) {
        const int s = sc->topo_inv ? sc->topo_inv[k] : k;
        memcpy(&frames[k * 12], &W[s * 12], 12 * sizeof(double));
    }
}

void orc_fk_f32(const OrcScene* sc, const float* q, float* frames) {
    const int J = sc->n_joints;
    float W[ORC_MAX_JOINTS * 12];
    fk_sorted_f32(sc, q, W);
    for (int k = 0; k < J; ++k) {
        const int s = sc->topo_inv ? sc->topo_inv[k] : k;
        memcpy(&frames[k * 12], &W[s * 12], 12 * sizeof(float));
    }
}

/* ------------------------------------------------------------------------- */
/* Primitive distances (restated from the geometry; PyRoFFI is unavailable)   */
/* ------------------------------------------------------------------------- */

static void xform(const double* F, const float* local, double out[3]) {
    for (int i = 0; i < 3; ++i)
        out[i] = F[i * 3 + 0] * local[0] + F[i * 3 + 1] * local[1] + F[i * 3 + 2] * local[2] + F[9 + i];
}

/* |s - o| - r - ro */
static double dist_sphere(const double* s, double r, const float* o) {
    const double dx = s[0] - o[0], dy = s[1] - o[1], dz = s[2] - o[2];
    return sqrt(dx * dx + dy * dy + dz * dz) - r - o[3];
}

/* distance from s to segment p1p2 minus r and the capsule radius */
static double dist_capsule(const double* s, double r, const float* c) {
    const double ax = c[3] - c[0], ay = c[4] - c[1], az = c[5] - c[2];
    const double wx = s[0] - c[0], wy = s[1] - c[1], wz = s[2] - c[2];
    const double L2 = ax * ax + ay * ay + az * az;
    double t = L2 > 0 ? (wx * ax + wy * ay + wz * az) / L2 : 0.0;
    t = t < 0 ? 0 : (t > 1 ? 1 : t);
    const double dx = wx - t * ax, dy = wy - t * ay, dz = wz - t * az;
    return sqrt(dx * dx + dy * dy + dz * dz) - r - c[6];
}

/* signed distance to the box (centre c, unit axes a1 a2 a3 as columns of R,
 * half lengths h) minus r */
static double dist_box(const double* s, double r, const float* b) {
    const double px = s[0] - b[0], py = s[1] - b[1], pz = s[2] - b[2];
    double q[3], out2 = 0.0, qmax = -INFINITY;
    for (int k = 0; k < 3; ++k) {
        const float* a = &b[3 + 3 * k];
        const double l = px * a[0] + py * a[1] + pz * a[2];
        q[k] = fabs(l) - b[12 + k];
        if (q[k] > 0) out2 += q[k] * q[k];
        if (q[k] > qmax) qmax = q[k];
    }
    const double inside = qmax < 0 ? qmax : 0.0;
    return sqrt(out2) + inside - r;
}

/* n . (s - p) - r, the normal pointing into free space */
static double dist_halfspace(const double* s, double r, const float* h) {
    return h[0] * (s[0] - h[3]) + h[1] * (s[1] - h[4]) + h[2] * (s[2] - h[5]) - r;
}

/* Smooth margin penalty: d - m/2 inside, -(d-m)^2/(2m) within the margin, 0 beyond.
 * C1-continuous; negative exactly when d < m. */
static double colldist(double d, double m) {
    if (m <= 0) return d < 0 ? d : 0.0;
    if (d < 0) return d - 0.5 * m;
    if (d < m) return -0.5 * (d - m) * (d - m) / m;
    return 0.0;
}

/* ------------------------------------------------------------------------- */
/* Checkers (prrtc_planner.cu:234-531), double precision                      */
/* ------------------------------------------------------------------------- */

static int scene_enabled(const OrcScene* sc) {
    return sc->n_joints > 0 && sc->n_spheres > 0 &&
           (sc->n_ws > 0 || sc->n_wc > 0 || sc->n_wb > 0 || sc->n_wh > 0 || sc->n_self > 0 || sc->n_points > 0);
}

static int sphere_center(const OrcScene* sc, const double* F, int s, double out[3]) {
    const int li = sc->sphere_link_idx[s];
    if (li < 0 || li >= sc->n_joints) return 0;
    xform(&F[li * 12], &sc->sphere_local[s * 3], out);
    return 1;
}

/* one sphere vs every world primitive; returns min distance, early exit when
 * `stop_at_hit` and a distance <= 0 is met (prrtc_planner.cu:391-419) */
static double sphere_vs_world(const OrcScene* sc, const double* c, double r, int stop_at_hit) {
    double m = INFINITY, d;
    for (int i = 0; i < sc->n_ws; ++i) { d = dist_sphere(c, r, &sc->world_spheres[i * 4]); if (d < m) m = d; if (stop_at_hit && d <= 0) return d; }
    for (int i = 0; i < sc->n_wc; ++i) { d = dist_capsule(c, r, &sc->world_capsules[i * 7]); if (d < m) m = d; if (stop_at_hit && d <= 0) return d; }
    for (int i = 0; i < sc->n_wb; ++i) { d = dist_box(c, r, &sc->world_boxes[i * 15]); if (d < m) m = d; if (stop_at_hit && d <= 0) return d; }
    for (int i = 0; i < sc->n_wh; ++i) { d = dist_halfspace(c, r, &sc->world_halfspaces[i * 6]); if (d < m) m = d; if (stop_at_hit && d <= 0) return d; }
    return m;
}

static int self_pair_dist(const OrcScene* sc, const double* F, int p, double* d) {
    const int i = sc->self_pairs[p * 2 + 0], j = sc->self_pairs[p * 2 + 1];
    if (i < 0 || j < 0 || i >= sc->n_spheres || j >= sc->n_spheres) return 0;
    double a[3], b[3];
    if (!sphere_center(sc, F, i, a) || !sphere_center(sc, F, j, b)) return 0;
    const float o[4] = {(float)0, 0, 0, 0};
    (void)o;
    const double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    *d = sqrt(dx * dx + dy * dy + dz * dz) - sc->sphere_radius[i] - sc->sphere_radius[j];
    return 1;
}

/* 234-307: flat early-exit binary check */
static int check_binary(const OrcScene* sc, const double* F) {
    for (int s = 0; s < sc->n_spheres; ++s) {
        double c[3];
        if (!sphere_center(sc, F, s, c)) continue;
        if (sphere_vs_world(sc, c, sc->sphere_radius[s], 1) <= 0) return 1;
    }
    for (int p = 0; p < sc->n_self; ++p) {
        double d;
        if (self_pair_dist(sc, F, p, &d) && d <= 0) return 1;
    }
    return 0;
}

/* 314-387: full sweep, collision iff the summed margin penalty is negative */
static int check_differentiable(const OrcScene* sc, const double* F, double margin) {
    double cost = 0.0;
    for (int s = 0; s < sc->n_spheres; ++s) {
        double c[3];
        if (!sphere_center(sc, F, s, c)) continue;
        const double r = sc->sphere_radius[s];
        for (int i = 0; i < sc->n_ws; ++i) cost += colldist(dist_sphere(c, r, &sc->world_spheres[i * 4]), margin);
        for (int i = 0; i < sc->n_wc; ++i) cost += colldist(dist_capsule(c, r, &sc->world_capsules[i * 7]), margin);
        for (int i = 0; i < sc->n_wb; ++i) cost += colldist(dist_box(c, r, &sc->world_boxes[i * 15]), margin);
        for (int i = 0; i < sc->n_wh; ++i) cost += colldist(dist_halfspace(c, r, &sc->world_halfspaces[i * 6]), margin);
    }
    for (int p = 0; p < sc->n_self; ++p) {
        double d;
        if (self_pair_dist(sc, F, p, &d)) cost += colldist(d, margin);
    }
    return cost < 0.0;
}

/* 426-499: coarse bounding-sphere pre-pass gates the fine world and self work */
static int check_coarse(const OrcScene* sc, const double* F) {
    const int K = sc->n_coarse;
    int dirty[ORC_MAX_LINKS];
    int any = 0;
    for (int k = 0; k < K; ++k) {
        dirty[k] = 0;
        const int li = sc->coarse_link[k];
        if (li < 0 || li >= sc->n_joints) continue;
        double c[3];
        xform(&F[li * 12], &sc->coarse_local[k * 3], c);
        if (sphere_vs_world(sc, c, sc->coarse_radius[k], 1) <= 0) { dirty[k] = 1; any = 1; }
    }
    if (any) {
        for (int k = 0; k < K; ++k) {
            if (!dirty[k]) continue;
            for (int s = sc->fine_offsets[k]; s < sc->fine_offsets[k + 1]; ++s) {
                double c[3];
                if (!sphere_center(sc, F, s, c)) continue;
                if (sphere_vs_world(sc, c, sc->sphere_radius[s], 1) <= 0) return 1;
            }
        }
    }
    for (int p = 0; p < sc->n_coarse_self; ++p) {
        const int ci = sc->coarse_self_pairs[p * 2], cj = sc->coarse_self_pairs[p * 2 + 1];
        if (ci < 0 || cj < 0 || ci >= K || cj >= K) continue;
        const int li = sc->coarse_link[ci], lj = sc->coarse_link[cj];
        if (li < 0 || lj < 0 || li >= sc->n_joints || lj >= sc->n_joints) continue;
        double a[3], b[3];
        xform(&F[li * 12], &sc->coarse_local[ci * 3], a);
        xform(&F[lj * 12], &sc->coarse_local[cj * 3], b);
        const double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
        if (sqrt(dx * dx + dy * dy + dz * dz) - sc->coarse_radius[ci] - sc->coarse_radius[cj] > 0) continue;
        for (int q = sc->self_pair_ranges[p * 2]; q < sc->self_pair_ranges[p * 2 + 1]; ++q) {
            double d;
            if (self_pair_dist(sc, F, q, &d) && d <= 0) return 1;
        }
    }
    return 0;
}

/* smallest |c - p| - r - r_env over the point cloud (brute force) */
static double sphere_vs_points(const OrcScene* sc, const double* c, double r) {
    double m = INFINITY;
    for (int i = 0; i < sc->n_points; ++i) {
        const float* p = &sc->points[i * 3];
        const double dx = c[0] - p[0], dy = c[1] - p[1], dz = c[2] - p[2];
        const double d = sqrt(dx * dx + dy * dy + dz * dz) - r - sc->r_env;
        if (d < m) m = d;
    }
    return m;
}

/* Point-cloud stage: any fine sphere within r_env of a point (inflated by the
 * margin for the differentiable checker, as the device checker does). */
static int check_points(const OrcScene* sc, const double* F, double inflate) {
    for (int s = 0; s < sc->n_spheres; ++s) {
        double c[3];
        if (!sphere_center(sc, F, s, c)) continue;
        if (sphere_vs_points(sc, c, sc->sphere_radius[s] + inflate) <= 0) return 1;
    }
    return 0;
}

static int config_in_collision_d(const OrcScene* sc, const double* q, int mode, float margin) {
    if (!scene_enabled(sc)) return 0;
    if (sc->n_joints <= 0 || sc->n_joints > ORC_MAX_JOINTS) return 0;
    double F[ORC_MAX_JOINTS * 12];
    orc_fk_f64(sc, q, F);
    if (sc->n_points > 0 && check_points(sc, F, mode == 1 ? (double)margin : 0.0)) return 1;
    const int coarse_ok = sc->n_coarse > 0 && sc->n_coarse <= ORC_MAX_LINKS;
    if (mode == 1) return check_differentiable(sc, F, margin);
    if (mode == 2 && coarse_ok) return check_coarse(sc, F);
    /* 741-743: the cooperative checker needs the coarse model and J <= 16;
     * otherwise mode 3 falls through to the flat binary check. */
    if (mode == 3 && coarse_ok && sc->n_joints <= 16) return check_coarse(sc, F);
    return check_binary(sc, F);
}

int orc_config_in_collision(const OrcScene* sc, const float* q, int mode, float margin) {
    double qd[ORC_DIM_MAX];
    for (int d = 0; d < sc->dim && d < ORC_DIM_MAX; ++d) qd[d] = q[d];
    return config_in_collision_d(sc, qd, mode, margin);
}

static double min_distance_d(const OrcScene* sc, const double* q) {
    double F[ORC_MAX_JOINTS * 12];
    if (sc->n_joints <= 0 || sc->n_joints > ORC_MAX_JOINTS) return INFINITY;
    orc_fk_f64(sc, q, F);
    double m = INFINITY;
    for (int s = 0; s < sc->n_spheres; ++s) {
        double c[3];
        if (!sphere_center(sc, F, s, c)) continue;
        double d = sphere_vs_world(sc, c, sc->sphere_radius[s], 0);
        if (d < m) m = d;
        if (sc->n_points > 0) {
            d = sphere_vs_points(sc, c, sc->sphere_radius[s]);
            if (d < m) m = d;
        }
    }
    for (int p = 0; p < sc->n_self; ++p) {
        double d;
        if (self_pair_dist(sc, F, p, &d) && d < m) m = d;
    }
    return m;
}

double orc_min_distance(const OrcScene* sc, const float* q) {
    double qd[ORC_DIM_MAX];
    for (int d = 0; d < sc->dim && d < ORC_DIM_MAX; ++d) qd[d] = q[d];
    return min_distance_d(sc, qd);
}

int orc_edge_in_collision(const OrcScene* sc, const float* base, const float* end,
                          int granularity, float resolution, int mode, float margin) {
    const int dim = sc->dim;
    float delta[ORC_DIM_MAX], w[ORC_DIM_MAX];
    for (int d = 0; d < dim; ++d) delta[d] = end[d] - base[d];
    const int G = orc_edge_waypoints(delta, dim, granularity, resolution);
    for (int k = 0; k < G; ++k) {
        orc_waypoint(base, delta, dim, k, G, w);
        if (orc_config_in_collision(sc, w, mode, margin)) return 1;
    }
    return 0;
}

void orc_check_configs(const OrcScene* sc, const float* configs, int n, int mode, float margin,
                       int32_t* verdict) {
    for (int i = 0; i < n; ++i) verdict[i] = orc_config_in_collision(sc, &configs[(size_t)i * sc->dim], mode, margin);
}

/* ------------------------------------------------------------------------- */
/* Sequential pRRTC (prrtc_planner.cu:675-1066)                               */
/* ------------------------------------------------------------------------- */

typedef struct {
    int prime_order[16];
    int halton[ORC_DIM_MAX];
    int vamp_tree;
    int local_iter;
    int done;
} Explorer;

/* 46-65 (prrtc_radius_shrink_atomic; one update at a time) */
void orc_radius_shrink(float* radii, int idx, float alpha, float r0, float rmin) {
    const float old = radii[idx];
    radii[idx] = (old == FLT_MAX) ? r0 : fmaxf(old * (1.0f - alpha), rmin);
}

/* 67-83 (prrtc_radius_grow_atomic) */
void orc_radius_grow(float* radii, int idx, float alpha) {
    const float old = radii[idx];
    if (old != FLT_MAX) radii[idx] = old * (1.0f + alpha);
}

static void radius_shrink(float* radii, int idx, float alpha, float r0, float rmin) {
    orc_radius_shrink(radii, idx, alpha, r0, rmin);
}

static void radius_grow(float* radii, int idx, float alpha) { orc_radius_grow(radii, idx, alpha); }

/* 790-824 */
int orc_choose_tree(int mode, int local_iter, int bid, int nblocks, int size_a, int size_b, float ratio_thr,
                    int* vamp) {
    const int total = size_a + size_b;
    if (mode == 0 || local_iter == 1) return (bid < (nblocks / 2)) ? 0 : 1;
    if (mode == 1) {
        const int diff = size_a >= size_b ? size_a - size_b : size_b - size_a;
        const float ratio = total > 0 ? (float)size_a / (float)total : 0.5f;
        if (diff < (int)(1.5f * (float)nblocks)) return (bid < (int)((float)nblocks * (1.0f - ratio))) ? 0 : 1;
        return ratio < ratio_thr ? 0 : 1;
    }
    if (mode == 2) {
        const int o_id = 1 - *vamp;
        const int t_sz = *vamp == 0 ? size_a : size_b;
        const int o_sz = o_id == 0 ? size_a : size_b;
        const float r = t_sz > 0 ? fabsf((float)(t_sz - o_sz) / (float)t_sz) : 0.0f;
        if (r < ratio_thr) *vamp = 1 - *vamp;
        return *vamp;
    }
    return size_a <= size_b ? 0 : 1;
}

static int choose_tree(Explorer* ex, int bid, int nblocks, const int sizes[2], int mode, float ratio_thr) {
    return orc_choose_tree(mode, ex->local_iter, bid, nblocks, sizes[0], sizes[1], ratio_thr, &ex->vamp_tree);
}

typedef struct {
    const OrcScene* sc;
    const OrcPlanParams* p;
    const float* lo;
    const float* hi;
    float* cfg[2];
    int* par[2];
    float* rad[2];
    OrcPlanOut* out;
} PlanState;

static int edge_check(PlanState* st, const float* base, const float* delta) {
    const int dim = st->p->dim;
    const int G = orc_edge_waypoints(delta, dim, st->p->granularity, st->p->edge_resolution);
    float w[ORC_DIM_MAX];
    st->out->edge_checks++;
    for (int k = 0; k < G; ++k) {
        orc_waypoint(base, delta, dim, k, G, w);
        st->out->config_checks++;
        if (orc_config_in_collision(st->sc, w, st->p->collision_mode, st->p->collision_margin)) return 1;
    }
    return 0;
}

/* One explorer iteration (770-1065).  Returns 1 when the explorer exits. */
static int explorer_step(PlanState* st, Explorer* ex, int bid) {
    const OrcPlanParams* p = st->p;
    OrcPlanOut* out = st->out;
    const int dim = p->dim, N = p->max_nodes;
    if (out->solved != 0) return 1;
    ex->local_iter++;
    if (ex->local_iter > p->max_iterations) {
        if (out->solved == 0) out->solved = -1;
        if (ex->local_iter > out->iter_count) out->iter_count = ex->local_iter;
        return 1;
    }
    float sample[ORC_DIM_MAX];
    orc_halton_sample(ex->prime_order, ex->halton, dim, st->lo, st->hi, sample);
    const int t = choose_tree(ex, bid, p->num_new_samples, out->tree_sizes, p->balance_mode, p->tree_ratio);
    const int o = 1 - t;
    const int comp_t = out->completed[t] < N ? out->completed[t] : N;
    const int comp_o = out->completed[o] < N ? out->completed[o] : N;
    if (comp_t <= 0 || comp_o <= 0) return 0;

    float dsq;
    const int nn = orc_nearest(st->cfg[t], N, dim, comp_t, sample, &dsq);
    if (nn < 0) return 0;
    const float nd = sqrtf(dsq);
    if (p->dynamic_domain && st->rad[t][nn] < nd) return 0;
    float base[ORC_DIM_MAX], cand[ORC_DIM_MAX], delta[ORC_DIM_MAX];
    for (int d = 0; d < dim; ++d) base[d] = st->cfg[t][(size_t)d * N + nn];
    orc_extend(base, sample, dim, nd, p->step_size, cand);
    for (int d = 0; d < dim; ++d) delta[d] = cand[d] - base[d];
    if (edge_check(st, base, delta)) {
        if (p->dynamic_domain) radius_shrink(st->rad[t], nn, p->dd_alpha, p->dd_radius, p->dd_min_radius);
        return 0;
    }
    /* 925-947 */
    const int idx = out->tree_sizes[t]++;
    if (idx >= N) {
        if (out->solved == 0) out->solved = -1;
        return 1;
    }
    st->par[t][idx] = nn;
    st->rad[t][idx] = FLT_MAX;
    if (p->dynamic_domain) radius_grow(st->rad[t], nn, p->dd_alpha);
    for (int d = 0; d < dim; ++d) st->cfg[t][(size_t)d * N + idx] = cand[d];
    out->completed[t]++;

    /* 949-994 connect */
    const int comp_oc = out->completed[o] < N ? out->completed[o] : N;
    float cdsq;
    const int cnn = orc_nearest(st->cfg[o], N, dim, comp_oc, cand, &cdsq);
    if (cnn < 0) return 0;
    const float cd = sqrtf(cdsq);
    int n_ext = 0;
    if (p->step_size > 1e-8f && cd > 1e-8f) n_ext = (int)ceilf(cd / p->step_size);
    int ext_parent = idx;
    float curr[ORC_DIM_MAX], vec[ORC_DIM_MAX];
    for (int d = 0; d < dim; ++d) {
        curr[d] = cand[d];
        vec[d] = n_ext > 0 ? (st->cfg[o][(size_t)d * N + cnn] - cand[d]) / (float)n_ext : 0.0f;
    }
    int failed = 0;
    for (int e = 0; e < n_ext; ++e) {
        if (edge_check(st, curr, vec)) { failed = 1; break; }
        const int eidx = out->tree_sizes[t]++;
        if (eidx >= N) {
            if (out->solved == 0) out->solved = -1;
            failed = 1;
            break;
        }
        st->par[t][eidx] = ext_parent;
        st->rad[t][eidx] = FLT_MAX;
        ext_parent = eidx;
        for (int d = 0; d < dim; ++d) curr[d] = curr[d] + vec[d];
        for (int d = 0; d < dim; ++d) st->cfg[t][(size_t)d * N + eidx] = curr[d];
        out->completed[t]++;
    }
    /* 1045-1062 */
    if (!failed) {
        if (out->solved == 0) {
            out->solved = 1;
            if (t == 0) { out->connection[0] = ext_parent; out->connection[1] = cnn; }
            else { out->connection[0] = cnn; out->connection[1] = ext_parent; }
            out->connection[2] = t;
        }
        if (ex->local_iter > out->iter_count) out->iter_count = ex->local_iter;
        return 1;
    }
    return out->solved != 0;
}

int orc_prrtc_plan(const OrcScene* sc, const float* start, const float* goals, int n_goals,
                   const float* lo, const float* hi, const OrcPlanParams* p, OrcPlanOut* out) {
    const int dim = p->dim, N = p->max_nodes, E = p->num_new_samples;
    if (dim <= 0 || dim > ORC_DIM_MAX || N < 1 || E < 1 || n_goals < 1 || n_goals > N) return -2;
    const float qnan = NAN;
    for (size_t i = 0; i < (size_t)dim * N; ++i) { out->tree_a[i] = qnan; out->tree_b[i] = qnan; }
    for (int i = 0; i < N; ++i) { out->parents_a[i] = -1; out->parents_b[i] = -1; }
    float* rad_a = (float*)malloc(sizeof(float) * N);
    float* rad_b = (float*)malloc(sizeof(float) * N);
    Explorer* ex = (Explorer*)calloc((size_t)E, sizeof(Explorer));
    for (int i = 0; i < N; ++i) { rad_a[i] = FLT_MAX; rad_b[i] = FLT_MAX; }
    /* 97-125 */
    for (int d = 0; d < dim; ++d) out->tree_a[(size_t)d * N] = start[d];
    out->parents_a[0] = 0;
    for (int g = 0; g < n_goals; ++g) {
        for (int d = 0; d < dim; ++d) out->tree_b[(size_t)d * N + g] = goals[g * dim + d];
        out->parents_b[g] = g;
    }
    out->tree_sizes[0] = 1; out->tree_sizes[1] = n_goals;
    out->completed[0] = 1; out->completed[1] = n_goals;
    out->iter_count = 0;
    out->connection[0] = out->connection[1] = out->connection[2] = -1;
    out->solved = 0;
    out->edge_checks = 0;
    out->config_checks = 0;
    for (int e = 0; e < E; ++e) {
        orc_prime_order(e, ex[e].prime_order);
        for (int d = 0; d < ORC_DIM_MAX; ++d) ex[e].halton[d] = 1;
    }
    PlanState st = {sc, p, lo, hi, {out->tree_a, out->tree_b}, {out->parents_a, out->parents_b},
                    {rad_a, rad_b}, out};
    int live = E;
    while (out->solved == 0 && live > 0) {
        live = 0;
        for (int e = 0; e < E && out->solved == 0; ++e) {
            if (ex[e].done) continue;
            if (explorer_step(&st, &ex[e], e)) ex[e].done = 1;
            else live++;
        }
    }
    free(rad_a);
    free(rad_b);
    free(ex);
    return out->solved;
}

/* prrtc.py:588-640 */
int orc_trace_path(const float* tree_a, const float* tree_b, const int* pa, const int* pb,
                   int max_nodes, int dim, const int connection[3], float* path, int max_len) {
    const int a = connection[0], b = connection[1];
    if (a < 0 || b < 0) {
        if (max_len < 1) return -1;
        for (int d = 0; d < dim; ++d) path[d] = tree_a[(size_t)d * max_nodes];
        return 1;
    }
    int* chain = (int*)malloc(sizeof(int) * (size_t)max_nodes);
    int na = 0, curr = a;
    for (int it = 0; it < max_nodes; ++it) {
        chain[na++] = curr;
        const int par = pa[curr];
        if (par == curr || par < 0) break;
        curr = par;
    }
    int len = 0;
    for (int i = na - 1; i >= 0; --i) {
        if (len >= max_len) { free(chain); return -1; }
        for (int d = 0; d < dim; ++d) path[(size_t)len * dim + d] = tree_a[(size_t)d * max_nodes + chain[i]];
        len++;
    }
    curr = b;
    for (int it = 0; it < max_nodes; ++it) {
        if (len >= max_len) { free(chain); return -1; }
        for (int d = 0; d < dim; ++d) path[(size_t)len * dim + d] = tree_b[(size_t)d * max_nodes + curr];
        len++;
        const int par = pb[curr];
        if (par == curr || par < 0) break;
        curr = par;
    }
    free(chain);
    return len;
}

/* prrtc.py:566 -- sum of segment L2 norms */
float orc_path_cost(const float* path, int len, int dim) {
    float cost = 0.0f;
    for (int i = 0; i + 1 < len; ++i) {
        float s = 0.0f;
        for (int d = 0; d < dim; ++d) {
            const float df = path[(i + 1) * dim + d] - path[i * dim + d];
            s += df * df;
        }
        cost += sqrtf(s);
    }
    return cost;
}

/* ------------------------------------------------------------------------- */
/* Host-driven RRT-Connect (prrtc_robogpu.py:36-298)                          */
/* ------------------------------------------------------------------------- */

static uint64_t splitmix64(uint64_t* s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static double uniform01(uint64_t* s) { return (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0); }

typedef struct {
    float* cfg; /* [max_nodes][dim] */
    int* par;
    int size, cap, dim;
} HostTree;

static int htree_add(HostTree* t, const float* q, int parent) {
    if (t->size >= t->cap) return -1;
    memcpy(&t->cfg[(size_t)t->size * t->dim], q, sizeof(float) * t->dim);
    t->par[t->size] = parent;
    return t->size++;
}

/* first index of the minimum, as np.argmin (prrtc_robogpu.py:82-87) */
static int htree_nearest(const HostTree* t, const float* q) {
    int best = 0;
    float bd = INFINITY;
    for (int i = 0; i < t->size; ++i) {
        float s = 0.0f;
        for (int d = 0; d < t->dim; ++d) {
            const float df = t->cfg[(size_t)i * t->dim + d] - q[d];
            s += df * df;
        }
        if (s < bd) { bd = s; best = i; }
    }
    return best;
}

/* prrtc_robogpu.py:36-44 */
static void steer(const float* from, const float* to, int dim, float step, float* out) {
    float s = 0.0f;
    for (int d = 0; d < dim; ++d) s += (to[d] - from[d]) * (to[d] - from[d]);
    const float dist = sqrtf(s);
    const float scale = fminf(1.0f, step / fmaxf(dist, 1e-8f));
    for (int d = 0; d < dim; ++d) out[d] = from[d] + (to[d] - from[d]) * scale;
}

typedef struct {
    const OrcScene* sc;
    const float* qa;
    const float* qb;
    int n, G, mode;
    float margin;
    int* free_out;
    int64_t checks;
    int lo, hi;
} EdgeJob;

/* prrtc_robogpu.py:47-56 + 183-191: waypoints linspace(0,1,G), endpoints included */
static void* edge_job(void* arg) {
    EdgeJob* j = (EdgeJob*)arg;
    const int dim = j->sc->dim;
    float w[ORC_DIM_MAX];
    for (int e = j->lo; e < j->hi; ++e) {
        int ok = 1;
        for (int k = 0; k < j->G && ok; ++k) {
            const float t = j->G > 1 ? (float)k / (float)(j->G - 1) : 0.0f;
            for (int d = 0; d < dim; ++d)
                w[d] = j->qa[e * dim + d] * (1.0f - t) + j->qb[e * dim + d] * t;
            j->checks++;
            if (orc_config_in_collision(j->sc, w, j->mode, j->margin)) ok = 0;
        }
        j->free_out[e] = ok;
    }
    return NULL;
}

static int64_t edges_free(const OrcScene* sc, const float* qa, const float* qb, int n, int G, int mode,
                          float margin, int n_threads, int* free_out) {
    if (n <= 0) return 0;
    if (n_threads <= 1 || n < 2) {
        EdgeJob j = {sc, qa, qb, n, G, mode, margin, free_out, 0, 0, n};
        edge_job(&j);
        return j.checks;
    }
    if (n_threads > n) n_threads = n;
    if (n_threads > 256) n_threads = 256;
    EdgeJob jobs[256];
    pthread_t th[256];
    for (int i = 0; i < n_threads; ++i) {
        jobs[i] = (EdgeJob){sc, qa, qb, n, G, mode, margin, free_out, 0, n * i / n_threads, n * (i + 1) / n_threads};
        pthread_create(&th[i], NULL, edge_job, &jobs[i]);
    }
    int64_t c = 0;
    for (int i = 0; i < n_threads; ++i) {
        pthread_join(th[i], NULL);
        c += jobs[i].checks;
    }
    return c;
}

static int htree_path(const HostTree* t, int node, int* chain) {
    int n = 0, curr = node;
    for (int it = 0; it < t->size; ++it) {
        chain[n++] = curr;
        const int par = t->par[curr];
        if (par == curr) break;
        curr = par;
    }
    return n;
}

int orc_rrtc_host_plan(const OrcScene* sc, const float* start, const float* goal,
                       const float* lo, const float* hi, int max_iterations, float step_size,
                       int num_new_samples, int granularity, int max_nodes, int connect_max_steps,
                       uint64_t seed, int mode, float margin, int n_threads,
                       float* path_out, int max_path, OrcHostOut* out) {
    const int dim = sc->dim, S = num_new_samples;
    memset(out, 0, sizeof(*out));
    out->cost = INFINITY;
    HostTree ta = {(float*)malloc(sizeof(float) * (size_t)max_nodes * dim), (int*)malloc(sizeof(int) * max_nodes), 0, max_nodes, dim};
    HostTree tb = {(float*)malloc(sizeof(float) * (size_t)max_nodes * dim), (int*)malloc(sizeof(int) * max_nodes), 0, max_nodes, dim};
    htree_add(&ta, start, 0);
    htree_add(&tb, goal, 0);
    float* samples = (float*)malloc(sizeof(float) * S * dim);
    float* qnear = (float*)malloc(sizeof(float) * S * dim);
    float* qnew = (float*)malloc(sizeof(float) * S * dim);
    float* targets = (float*)malloc(sizeof(float) * S * dim);
    float* qfrom = (float*)malloc(sizeof(float) * S * dim);
    float* qstep = (float*)malloc(sizeof(float) * S * dim);
    int* near = (int*)malloc(sizeof(int) * S);
    int* freev = (int*)malloc(sizeof(int) * S);
    int* new_nodes = (int*)malloc(sizeof(int) * S);
    int* other_idx = (int*)malloc(sizeof(int) * S);
    int* live = (int*)malloc(sizeof(int) * S);
    int* li = (int*)malloc(sizeof(int) * S);
    uint64_t rs = seed;
    HostTree *active = &ta, *other = &tb;
    int solved = 0, conn_a = -1, conn_b = -1, it = 0;
    for (it = 1; it <= max_iterations; ++it) {
        for (int s = 0; s < S; ++s)
            for (int d = 0; d < dim; ++d)
                samples[s * dim + d] = (float)((double)lo[d] + ((double)hi[d] - (double)lo[d]) * uniform01(&rs));
        for (int s = 0; s < S; ++s) {
            near[s] = htree_nearest(active, &samples[s * dim]);
            memcpy(&qnear[s * dim], &active->cfg[(size_t)near[s] * dim], sizeof(float) * dim);
            steer(&qnear[s * dim], &samples[s * dim], dim, step_size, &qnew[s * dim]);
        }
        out->config_checks += edges_free(sc, qnear, qnew, S, granularity, mode, margin, n_threads, freev);
        int n_new = 0;
        for (int s = 0; s < S; ++s) {
            if (!freev[s]) continue;
            const int idx = htree_add(active, &qnew[s * dim], near[s]);
            if (idx < 0) break;
            memcpy(&targets[n_new * dim], &qnew[s * dim], sizeof(float) * dim);
            new_nodes[n_new++] = idx;
        }
        if (n_new == 0) {
            HostTree* tmp = active; active = other; other = tmp;
            continue;
        }
        for (int s = 0; s < n_new; ++s) {
            other_idx[s] = htree_nearest(other, &targets[s * dim]);
            live[s] = 1;
        }
        for (int step = 0; step < connect_max_steps && !solved; ++step) {
            int nl = 0;
            for (int s = 0; s < n_new; ++s) if (live[s]) li[nl++] = s;
            if (nl == 0) break;
            for (int k = 0; k < nl; ++k) {
                memcpy(&qfrom[k * dim], &other->cfg[(size_t)other_idx[li[k]] * dim], sizeof(float) * dim);
                steer(&qfrom[k * dim], &targets[li[k] * dim], dim, step_size, &qstep[k * dim]);
            }
            out->config_checks += edges_free(sc, qfrom, qstep, nl, granularity, mode, margin, n_threads, freev);
            for (int k = 0; k < nl; ++k) {
                const int s = li[k];
                if (!freev[k]) { live[s] = 0; continue; }
                const int idx = htree_add(other, &qstep[k * dim], other_idx[s]);
                if (idx < 0) { live[s] = 0; continue; }
                other_idx[s] = idx;
                float dd = 0.0f;
                for (int d = 0; d < dim; ++d) {
                    const float df = qstep[k * dim + d] - targets[s * dim + d];
                    dd += df * df;
                }
                if (sqrtf(dd) <= step_size * 1e-3f + 1e-6f) {
                    live[s] = 0;
                    if (active == &ta) { conn_a = new_nodes[s]; conn_b = idx; }
                    else { conn_a = idx; conn_b = new_nodes[s]; }
                    solved = 1;
                    break;
                }
            }
        }
        if (solved) break;
        HostTree* tmp = active; active = other; other = tmp;
    }
    out->solved = solved;
    out->iterations = it > max_iterations ? max_iterations : it;
    out->size_a = ta.size;
    out->size_b = tb.size;
    out->path_len = 0;
    if (solved) {
        int* chain = (int*)malloc(sizeof(int) * (size_t)(ta.size + tb.size + 2));
        const int na = htree_path(&ta, conn_a, chain);
        int len = 0;
        for (int i = na - 1; i >= 0 && len < max_path; --i, ++len)
            memcpy(&path_out[len * dim], &ta.cfg[(size_t)chain[i] * dim], sizeof(float) * dim);
        const int nb = htree_path(&tb, conn_b, chain);
        for (int i = 0; i < nb && len < max_path; ++i, ++len)
            memcpy(&path_out[len * dim], &tb.cfg[(size_t)chain[i] * dim], sizeof(float) * dim);
        free(chain);
        out->path_len = len;
        out->cost = orc_path_cost(path_out, len, dim);
    }
    free(ta.cfg); free(ta.par); free(tb.cfg); free(tb.par);
    free(samples); free(qnear); free(qnew); free(targets); free(qfrom); free(qstep);
    free(near); free(freev); free(new_nodes); free(other_idx); free(live); free(li);
    return solved;
}

/* ------------------------------------------------------------------------- */
/* Path re-validation and smoothing cost                                      */
/* ------------------------------------------------------------------------- */

int orc_validate_path(const OrcScene* sc, const float* path, int len, float resolution,
                      double* min_dist) {
    const int dim = sc->dim;
    double m = INFINITY;
    int ok = 1;
    double q[ORC_DIM_MAX];
    if (len == 1) {
        for (int d = 0; d < dim; ++d) q[d] = path[d];
        m = min_distance_d(sc, q);
        ok = !(m <= 0.0);
    }
    for (int i = 0; i + 1 < len; ++i) {
        double l2 = 0.0;
        for (int d = 0; d < dim; ++d) {
            const double df = (double)path[(i + 1) * dim + d] - (double)path[i * dim + d];
            l2 += df * df;
        }
        int n = (int)ceil(sqrt(l2) / (double)resolution);
        if (n < 1) n = 1;
        for (int k = (i == 0 ? 0 : 1); k <= n; ++k) {
            const double t = (double)k / (double)n;
            for (int d = 0; d < dim; ++d)
                q[d] = (double)path[i * dim + d] + t * ((double)path[(i + 1) * dim + d] - (double)path[i * dim + d]);
            const double dm = min_distance_d(sc, q);
            if (dm < m) m = dm;
            if (dm <= 0.0) ok = 0;
        }
    }
    if (min_dist) *min_dist = m;
    return ok;
}

static double softplus_b(double x, double beta) {
    const double z = beta * x;
    return (z > 0 ? z + log1p(exp(-z)) : log1p(exp(z))) / beta;
}

double orc_smooth_cost(const OrcScene* sc, const double* wp, int W, float margin, float beta, float w_len) {
    const int dim = sc->dim;
    double total = 0.0;
    double F[ORC_MAX_JOINTS * 12];
    for (int w = 0; w < W; ++w) {
        orc_fk_f64(sc, &wp[w * dim], F);
        for (int s = 0; s < sc->n_spheres; ++s) {
            double c[3];
            if (!sphere_center(sc, F, s, c)) continue;
            const double r = sc->sphere_radius[s];
            for (int i = 0; i < sc->n_ws; ++i) total += softplus_b(margin - dist_sphere(c, r, &sc->world_spheres[i * 4]), beta);
            for (int i = 0; i < sc->n_wc; ++i) total += softplus_b(margin - dist_capsule(c, r, &sc->world_capsules[i * 7]), beta);
            for (int i = 0; i < sc->n_wb; ++i) total += softplus_b(margin - dist_box(c, r, &sc->world_boxes[i * 15]), beta);
            for (int i = 0; i < sc->n_wh; ++i) total += softplus_b(margin - dist_halfspace(c, r, &sc->world_halfspaces[i * 6]), beta);
        }
        for (int p = 0; p < sc->n_self; ++p) {
            double d;
            if (self_pair_dist(sc, F, p, &d)) total += softplus_b(margin - d, beta);
        }
    }
    for (int w = 0; w + 1 < W; ++w) {
        double s = 0.0;
        for (int d = 0; d < dim; ++d) {
            const double df = wp[(w + 1) * dim + d] - wp[w * dim + d];
            s += df * df;
        }
        total += (double)w_len * s;
    }
    return total;
}
