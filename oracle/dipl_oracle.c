/*
 * TEST INFRASTRUCTURE — CHECKER ONLY. Never linked into, or called by, the product library;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * Plain-C restatement of the BVH build-and-trace path, used as the oracle for the CUDA kernels
 * in diplodocus_b200/csrc. Compile with -ffp-contract=off (oracle/Makefile) so every float
 * operation rounds exactly as written, like the reference's own CPU build (CMakeLists.txt:9-11).
 *
 * What each part restates:
 *  - orc_mt: the reference Moller-Trumbore test, Triangle::IntersectRay (src/scene/triangle.cc:10-43),
 *    operation for operation (plain mul/add, IEEE divide, |det| < 1e-6 cull, b1/b2 range tests).
 *  - orc_brute_closest: DummyAccelerationStucture::Intersect
 *    (src/acceleration/dummy_acceleration_structure.cc:21-64): ascending ids, accept t > 1e-6 && t < t_hit,
 *    so exact-t ties go to the lowest id. The same loop runs with the watertight test.
 *  - orc_brute_any: DummyAccelerationStucture::IntersectAny (dummy_acceleration_structure.cc:66-79).
 *  - orc_wt: watertight ray/triangle test of Woop, Benthin and Wald (JCGT 2013), FP32 with the
 *    paper's FP64 recomputation of zero edge functions. Absent from the reference (README.md:156-161 lists
 *    the accelerated path as planned).
 *  - orc_morton30 / orc_emc60: this project's Morton and extended-Morton codes (absent from the
 *    reference; README.md:14-16 names Vinkler et al. 2017 for EMC).
 *  - orc_ploc: this project's PLOC (Meister & Bittner 2017) merge loop with its deterministic
 *    tie rule, restated sequentially so the device topology can be compared bit for bit.
 *  - orc_intersect_f64 / orc_brute_closest_f64: FP64 re-intersection used as the error oracle.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <unistd.h>

/* ------------------------------------------------------------------------------------------ */
/* Minimal parallel-for over [0, n) with pthreads (static contiguous chunks).                   */
/* ------------------------------------------------------------------------------------------ */
typedef void (*orc_range_fn)(void* ctx, int64_t begin, int64_t end);
typedef struct {
    orc_range_fn fn;
    void* ctx;
    int64_t b, e;
} orc_job;

static void* orc_job_run(void* p) {
    orc_job* j = (orc_job*)p;
    j->fn(j->ctx, j->b, j->e);
    return NULL;
}

static int orc_threads = 0;
void orc_set_threads(int n) { orc_threads = n; }

static void orc_parallel_for(int64_t n, orc_range_fn fn, void* ctx) {
    int nt = orc_threads > 0 ? orc_threads : (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nt < 1) nt = 1;
    if (nt > 256) nt = 256;
    if (n < 4 * nt) nt = 1;
    if (nt == 1) {
        fn(ctx, 0, n);
        return;
    }
    pthread_t th[256];
    orc_job jobs[256];
    int64_t chunk = (n + nt - 1) / nt;
    int launched = 0;
    for (int k = 0; k < nt; ++k) {
        int64_t b = k * chunk, e = b + chunk < n ? b + chunk : n;
        if (b >= e) break;
        jobs[k].fn = fn;
        jobs[k].ctx = ctx;
        jobs[k].b = b;
        jobs[k].e = e;
        pthread_create(&th[k], NULL, orc_job_run, &jobs[k]);
        ++launched;
    }
    for (int k = 0; k < launched; ++k) pthread_join(th[k], NULL);
}

#define ORC_EPS 1e-6f                 /* kEpsilon, src/util/util.h:15 */
#define ORC_INF 3.40282346638528859812e+38F /* kInfinity = FLT_MAX, src/util/util.h:16 */

/* ------------------------------------------------------------------------------------------ */
/* Reference Moller-Trumbore (triangle.cc:10-43).                                               */
/* ------------------------------------------------------------------------------------------ */
float orc_mt(const float* a, const float* b, const float* c, const float* o, const float* d, int backface,
             float* b1_out, float* b2_out) {
    float e1x = b[0] - a[0], e1y = b[1] - a[1], e1z = b[2] - a[2];
    float e2x = c[0] - a[0], e2y = c[1] - a[1], e2z = c[2] - a[2];
    /* pvec = Cross(dir, e2) (vec3.h:119-121) */
    float px = d[1] * e2z - d[2] * e2y;
    float py = d[2] * e2x - d[0] * e2z;
    float pz = d[0] * e2y - d[1] * e2x;
    /* det = Dot(e1, pvec) = (x*x + y*y) + z*z (vec3.h:118) */
    float det = e1x * px + e1y * py + e1z * pz;
    if (backface) {
        if (det < ORC_EPS) return ORC_INF;
    } else {
        if (fabsf(det) < ORC_EPS) return ORC_INF;
    }
    float inv = 1.0f / det;
    float tx = o[0] - a[0], ty = o[1] - a[1], tz = o[2] - a[2];
    float b1 = (tx * px + ty * py + tz * pz) * inv;
    if (b1 < 0.0f || b1 > 1.0f) return ORC_INF;
    /* qvec = Cross(tvec, e1) */
    float qx = ty * e1z - tz * e1y;
    float qy = tz * e1x - tx * e1z;
    float qz = tx * e1y - ty * e1x;
    float b2 = (d[0] * qx + d[1] * qy + d[2] * qz) * inv;
    if (b2 < 0.0f || b1 + b2 > 1.0f) return ORC_INF;
    float t = (e2x * qx + e2y * qy + e2z * qz) * inv;
    *b1_out = b1;
    *b2_out = b2;
    return t;
}

/* ------------------------------------------------------------------------------------------ */
/* Watertight test (Woop, Benthin, Wald 2013). Returns t, or ORC_INF on a miss.                 */
/* Backface culling keeps the reference's meaning: a hit needs e1.(d x e2) > 0 (triangle.cc:18). */
/* ------------------------------------------------------------------------------------------ */
float orc_wt(const float* v0, const float* v1, const float* v2, const float* o, const float* d, int backface,
             float* b1_out, float* b2_out) {
    float ax = fabsf(d[0]), ay = fabsf(d[1]), az = fabsf(d[2]);
    int kz = (ax > ay) ? ((ax > az) ? 0 : 2) : ((ay > az) ? 1 : 2);
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    if (d[kz] < 0.0f) { int tmp = kx; kx = ky; ky = tmp; }
    float sx = d[kx] / d[kz];
    float sy = d[ky] / d[kz];
    float sz = 1.0f / d[kz];
    float A[3] = {v0[0] - o[0], v0[1] - o[1], v0[2] - o[2]};
    float B[3] = {v1[0] - o[0], v1[1] - o[1], v1[2] - o[2]};
    float C[3] = {v2[0] - o[0], v2[1] - o[1], v2[2] - o[2]};
    float Ax = A[kx] - sx * A[kz], Ay = A[ky] - sy * A[kz];
    float Bx = B[kx] - sx * B[kz], By = B[ky] - sy * B[kz];
    float Cx = C[kx] - sx * C[kz], Cy = C[ky] - sy * C[kz];
    float U = Cx * By - Cy * Bx;
    float V = Ax * Cy - Ay * Cx;
    float W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
        V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
        W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return ORC_INF;
    float det = U + V + W;
    if (det == 0.0f) return ORC_INF;
    if (backface) {
        /* front face: e1.(d x e2) > 0, which is det > 0 in the sheared frame */
        if (det < 0.0f) return ORC_INF;
    }
    float Az = sz * A[kz], Bz = sz * B[kz], Cz = sz * C[kz];
    float T = U * Az + V * Bz + W * Cz;
    float rcp = 1.0f / det;
    *b1_out = V * rcp;
    *b2_out = W * rcp;
    return T * rcp;
}

/* ------------------------------------------------------------------------------------------ */
/* Brute force closest / any hit.                                                               */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
    const float *tris, *rays;
    int64_t n;
    int leaf_test, backface;
    int32_t* prim;
    float *t, *u, *v;
    uint8_t* occ;
} orc_brute_ctx;

static void brute_closest_range(void* p, int64_t rb, int64_t re) {
    orc_brute_ctx* c = (orc_brute_ctx*)p;
    for (int64_t r = rb; r < re; ++r) {
        const float* ray = c->rays + 8 * r;
        float tmin = ray[3];
        float t_hit = ray[7];
        int32_t best = -1;
        float bu = 0.0f, bv = 0.0f;
        for (int64_t i = 0; i < c->n; ++i) {
            const float* q = c->tris + 9 * i;
            float b1 = 0.0f, b2 = 0.0f;
            float t = c->leaf_test ? orc_wt(q, q + 3, q + 6, ray, ray + 4, c->backface, &b1, &b2)
                                   : orc_mt(q, q + 3, q + 6, ray, ray + 4, c->backface, &b1, &b2);
            /* t == ORC_INF is the tests' miss value; it never hits, also when tmax is +inf */
            if (t > tmin && t < t_hit && t < ORC_INF) {
                t_hit = t;
                best = (int32_t)i;
                bu = b1;
                bv = b2;
            }
        }
        c->prim[r] = best;
        c->t[r] = best >= 0 ? t_hit : INFINITY;
        c->u[r] = best >= 0 ? bu : 0.0f;
        c->v[r] = best >= 0 ? bv : 0.0f;
    }
}

void orc_brute_closest(const float* tris, int64_t n, const float* rays, int64_t nr, int leaf_test, int backface,
                       int32_t* prim, float* t_out, float* u_out, float* v_out) {
    orc_brute_ctx c = {tris, rays, n, leaf_test, backface, prim, t_out, u_out, v_out, NULL};
    orc_parallel_for(nr, brute_closest_range, &c);
}

static void brute_any_range(void* p, int64_t rb, int64_t re) {
    orc_brute_ctx* c = (orc_brute_ctx*)p;
    for (int64_t r = rb; r < re; ++r) {
        const float* ray = c->rays + 8 * r;
        uint8_t hit = 0;
        for (int64_t i = 0; i < c->n && !hit; ++i) {
            const float* q = c->tris + 9 * i;
            float b1, b2;
            float t = c->leaf_test ? orc_wt(q, q + 3, q + 6, ray, ray + 4, c->backface, &b1, &b2)
                                   : orc_mt(q, q + 3, q + 6, ray, ray + 4, c->backface, &b1, &b2);
            if (t > ray[3] && t < ray[7] && t < ORC_INF) hit = 1;
        }
        c->occ[r] = hit;
    }
}

void orc_brute_any(const float* tris, int64_t n, const float* rays, int64_t nr, int leaf_test, int backface,
                   uint8_t* occluded) {
    orc_brute_ctx c = {tris, rays, n, leaf_test, backface, NULL, NULL, NULL, NULL, occluded};
    orc_parallel_for(nr, brute_any_range, &c);
}

/* ------------------------------------------------------------------------------------------ */
/* FP64 oracle: intersection of each ray with a given triangle (Cramer's rule in double), and   */
/* an FP64 closest hit (no epsilon cull; inclusive edges) for classifying disagreements.        */
/* ------------------------------------------------------------------------------------------ */
static int f64_hit(const float* p, const float* ray, double* t, double* u, double* v) {
    double a[3] = {p[0], p[1], p[2]};
    double e1[3] = {(double)p[3] - a[0], (double)p[4] - a[1], (double)p[5] - a[2]};
    double e2[3] = {(double)p[6] - a[0], (double)p[7] - a[1], (double)p[8] - a[2]};
    double d[3] = {ray[4], ray[5], ray[6]};
    double s[3] = {(double)ray[0] - a[0], (double)ray[1] - a[1], (double)ray[2] - a[2]};
    double pv[3] = {d[1] * e2[2] - d[2] * e2[1], d[2] * e2[0] - d[0] * e2[2], d[0] * e2[1] - d[1] * e2[0]};
    double det = e1[0] * pv[0] + e1[1] * pv[1] + e1[2] * pv[2];
    if (det == 0.0) return 0;
    double inv = 1.0 / det;
    double uu = (s[0] * pv[0] + s[1] * pv[1] + s[2] * pv[2]) * inv;
    double q[3] = {s[1] * e1[2] - s[2] * e1[1], s[2] * e1[0] - s[0] * e1[2], s[0] * e1[1] - s[1] * e1[0]};
    double vv = (d[0] * q[0] + d[1] * q[1] + d[2] * q[2]) * inv;
    double tt = (e2[0] * q[0] + e2[1] * q[1] + e2[2] * q[2]) * inv;
    *t = tt;
    *u = uu;
    *v = vv;
    return (uu >= 0.0 && vv >= 0.0 && uu + vv <= 1.0) ? 1 : 0;
}

typedef struct {
    const float *tris, *rays;
    int64_t n;
    const int32_t* prim_in;
    int32_t* prim_out;
    double *t, *u, *v;
} orc_f64_ctx;

static void isect_f64_range(void* p, int64_t rb, int64_t re) {
    orc_f64_ctx* c = (orc_f64_ctx*)p;
    for (int64_t r = rb; r < re; ++r) {
        if (c->prim_in[r] < 0) {
            c->t[r] = INFINITY;
            c->u[r] = c->v[r] = 0.0;
            continue;
        }
        f64_hit(c->tris + 9 * (int64_t)c->prim_in[r], c->rays + 8 * r, &c->t[r], &c->u[r], &c->v[r]);
    }
}

void orc_intersect_f64(const float* tris, const float* rays, int64_t nr, const int32_t* prim, double* t, double* u,
                       double* v) {
    orc_f64_ctx c = {tris, rays, 0, prim, NULL, t, u, v};
    orc_parallel_for(nr, isect_f64_range, &c);
}

static void brute_f64_range(void* p, int64_t rb, int64_t re) {
    orc_f64_ctx* c = (orc_f64_ctx*)p;
    for (int64_t r = rb; r < re; ++r) {
        const float* ray = c->rays + 8 * r;
        double best_t = ray[7];
        int32_t best = -1;
        for (int64_t i = 0; i < c->n; ++i) {
            double t, u, v;
            if (f64_hit(c->tris + 9 * i, ray, &t, &u, &v) && t > (double)ray[3] && t < best_t) {
                best_t = t;
                best = (int32_t)i;
            }
        }
        c->prim_out[r] = best;
        c->t[r] = best >= 0 ? best_t : INFINITY;
    }
}

void orc_brute_closest_f64(const float* tris, int64_t n, const float* rays, int64_t nr, int32_t* prim,
                           double* t_out) {
    orc_f64_ctx c = {tris, rays, n, NULL, prim, t_out, NULL, NULL};
    orc_parallel_for(nr, brute_f64_range, &c);
}

/* ------------------------------------------------------------------------------------------ */
/* Scene bounds, centroids and codes.                                                           */
/* Centroid = (v0 + v1 + v2) / 3 evaluated as ((v0 + v1) + v2) / 3.0f, the reference's          */
/* CalculateTriangleCentroid (src/scene/triangle.h:36).                                          */
/* ------------------------------------------------------------------------------------------ */
static inline void centroid(const float* p, float* c) {
    for (int a = 0; a < 3; ++a) c[a] = ((p[a] + p[3 + a]) + p[6 + a]) / 3.0f;
}

/* A triangle with a NaN or infinite coordinate can never be hit (both leaf tests give t = NaN): it stays
 * out of the scene bounds and its cluster box is empty (lo = +inf, hi = -inf), as on the device. */
static int tri_finite(const float* p) {
    for (int k = 0; k < 9; ++k)
        if (!isfinite(p[k])) return 0;
    return 1;
}

void orc_scene_bounds(const float* tris, int64_t n, float* cmin, float* cmax, float* bmin, float* bmax) {
    for (int a = 0; a < 3; ++a) {
        cmin[a] = bmin[a] = INFINITY;
        cmax[a] = bmax[a] = -INFINITY;
    }
    for (int64_t i = 0; i < n; ++i) {
        const float* p = tris + 9 * i;
        if (!tri_finite(p)) continue;
        float c[3];
        centroid(p, c);
        for (int a = 0; a < 3; ++a) {
            cmin[a] = fminf(cmin[a], c[a]);
            cmax[a] = fmaxf(cmax[a], c[a]);
            for (int k = 0; k < 3; ++k) {
                bmin[a] = fminf(bmin[a], p[3 * k + a]);
                bmax[a] = fmaxf(bmax[a], p[3 * k + a]);
            }
        }
    }
}

static inline uint32_t expand10(uint32_t x) {
    x &= 0x3FFu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

/* 30-bit Morton code of the centroid in the centroid bounds: 10 bits per axis, x highest. */
void orc_morton30(const float* tris, int64_t n, const float* cmin, const float* cmax, uint32_t* codes) {
    float s[3];
    for (int a = 0; a < 3; ++a) {
        float ext = cmax[a] - cmin[a];
        s[a] = ext > 0.0f ? 1024.0f / ext : 0.0f;
    }
    for (int64_t i = 0; i < n; ++i) {
        float c[3];
        centroid(tris + 9 * i, c);
        uint32_t q[3];
        for (int a = 0; a < 3; ++a) {
            float x = (c[a] - cmin[a]) * s[a];
            x = fminf(fmaxf(x, 0.0f), 1023.0f);
            q[a] = (uint32_t)x;
        }
        codes[i] = (expand10(q[0]) << 2) | (expand10(q[1]) << 1) | expand10(q[2]);
    }
}

/* EMC60 bit plan: 60 positions handed out MSB first, each to the dimension (x, y, z, size) with
 * the largest remaining extent (first in that order on ties), which is then halved. Spatial
 * extents are the centroid-bounds extents; the size dimension's extent is the scene-box diagonal. */
void orc_emc60_plan(const float* cmin, const float* cmax, float diag, int* bits, uint64_t* masks) {
    float e[4] = {cmax[0] - cmin[0], cmax[1] - cmin[1], cmax[2] - cmin[2], diag};
    for (int a = 0; a < 4; ++a) {
        bits[a] = 0;
        masks[a] = 0;
        if (!(e[a] > 0.0f)) e[a] = 0.0f;
    }
    for (int pos = 59; pos >= 0; --pos) {
        int best = 0;
        for (int a = 1; a < 4; ++a)
            if (e[a] > e[best]) best = a;
        bits[best] += 1;
        masks[best] |= (uint64_t)1 << pos;
        e[best] *= 0.5f;
    }
}

static inline uint64_t deposit(uint64_t value, uint64_t mask) {
    /* scatter the low bits of value into the set bits of mask, low to high */
    uint64_t out = 0;
    while (mask) {
        uint64_t low = mask & (~mask + 1);
        if (value & 1) out |= low;
        value >>= 1;
        mask &= mask - 1;
    }
    return out;
}

float orc_scene_diag(const float* bmin, const float* bmax) {
    float dx = bmax[0] - bmin[0], dy = bmax[1] - bmin[1], dz = bmax[2] - bmin[2];
    return sqrtf((dx * dx + dy * dy) + dz * dz);
}

void orc_emc60(const float* tris, int64_t n, const float* cmin, const float* cmax, float diag, uint64_t* codes) {
    int bits[4];
    uint64_t masks[4];
    orc_emc60_plan(cmin, cmax, diag, bits, masks);
    float lo[4] = {cmin[0], cmin[1], cmin[2], 0.0f};
    float ext[4] = {cmax[0] - cmin[0], cmax[1] - cmin[1], cmax[2] - cmin[2], diag};
    float s[4];
    uint64_t top[4];
    for (int a = 0; a < 4; ++a) {
        float cells = ldexpf(1.0f, bits[a]);
        s[a] = (ext[a] > 0.0f && bits[a] > 0) ? cells / ext[a] : 0.0f;
        top[a] = bits[a] >= 64 ? ~(uint64_t)0 : (((uint64_t)1 << bits[a]) - 1);
    }
    for (int64_t i = 0; i < n; ++i) {
        const float* p = tris + 9 * i;
        float x[4];
        centroid(p, x);
        float dx = fmaxf(fmaxf(p[0], p[3]), p[6]) - fminf(fminf(p[0], p[3]), p[6]);
        float dy = fmaxf(fmaxf(p[1], p[4]), p[7]) - fminf(fminf(p[1], p[4]), p[7]);
        float dz = fmaxf(fmaxf(p[2], p[5]), p[8]) - fminf(fminf(p[2], p[5]), p[8]);
        x[3] = sqrtf((dx * dx + dy * dy) + dz * dz);
        uint64_t code = 0;
        for (int a = 0; a < 4; ++a) {
            if (bits[a] == 0) continue;
            /* quantise: clamp below at 0 (NaN -> 0), truncate, clamp to the top cell in integers */
            float q = fmaxf((x[a] - lo[a]) * s[a], 0.0f);
            uint64_t qi = q < 1.8e19f ? (uint64_t)q : top[a];
            if (qi > top[a]) qi = top[a];
            code |= deposit(qi, masks[a]);
        }
        codes[i] = code;
    }
}

/* ------------------------------------------------------------------------------------------ */
/* PLOC (Meister & Bittner 2017) as built on the device, restated sequentially.                 */
/*                                                                                              */
/* Clusters start as the triangles in sorted-code order (leaf node id = sorted position).       */
/* Each iteration: NN(i) = argmin over j in [i-r, i+r], j != i, same segment, of the key         */
/* (d(i,j), |i-j|, min(i,j) & 1, j > i), d = dx*dy + dy*dz + dz*dx of the merged box            */
/* (half its surface area), evaluated as fmaf(dx, dy, fmaf(dy, dz, dz*dx)); a NaN distance       */
/* counts as +inf. Mutual pairs (NN(NN(i)) == i) merge: a new node (left = cluster i's node,     */
/* right = cluster j's node) takes the lower position, the higher one is dropped, the rest keep  */
/* their order. Internal node k (creation order: iteration, then position) has id n_leaves + k.  */
/* Stops when one cluster per segment is left.                                                   */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
    float lo[3], hi[3];
    int32_t node, seg;
} orc_cluster;

static inline uint64_t ploc_key(const orc_cluster* a, const orc_cluster* b, int64_t i, int64_t j) {
    float dx = fmaxf(a->hi[0], b->hi[0]) - fminf(a->lo[0], b->lo[0]);
    float dy = fmaxf(a->hi[1], b->hi[1]) - fminf(a->lo[1], b->lo[1]);
    float dz = fmaxf(a->hi[2], b->hi[2]) - fminf(a->lo[2], b->lo[2]);
    float d = fmaf(dx, dy, fmaf(dy, dz, dz * dx));
    uint32_t bits;
    if (d != d) d = INFINITY;
    memcpy(&bits, &d, 4);
    uint64_t gap = (uint64_t)(j > i ? j - i : i - j);
    uint64_t mn = (uint64_t)(j > i ? i : j);
    uint64_t tie = (gap << 2) | ((mn & 1) << 1) | (uint64_t)(j > i ? 1 : 0);
    return ((uint64_t)bits << 32) | tie;
}

/* perm: triangle id at each sorted position; seg: segment id per sorted position (NULL = one).
 * Outputs: children[2k], children[2k+1]; boxes[6k..6k+5] = lo xyz, hi xyz of internal node k.
 * Returns the number of internal nodes, or -1 on bad input. */
int64_t orc_ploc(const float* tris, int64_t n, const int32_t* perm, const int32_t* seg, int64_t nseg, int radius,
                 int32_t* children, float* boxes, int32_t* iterations) {
    if (n <= 0 || radius < 1) return n == 0 ? 0 : -1;
    orc_cluster* cur = (orc_cluster*)malloc(sizeof(orc_cluster) * (size_t)n);
    orc_cluster* nxt = (orc_cluster*)malloc(sizeof(orc_cluster) * (size_t)n);
    int64_t* nn = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        const float* p = tris + 9 * (int64_t)perm[i];
        const int fin = tri_finite(p);
        for (int a = 0; a < 3; ++a) {
            cur[i].lo[a] = fin ? fminf(fminf(p[a], p[3 + a]), p[6 + a]) : INFINITY;
            cur[i].hi[a] = fin ? fmaxf(fmaxf(p[a], p[3 + a]), p[6 + a]) : -INFINITY;
        }
        cur[i].node = (int32_t)i;
        cur[i].seg = seg ? seg[i] : 0;
    }
    int64_t m = n, made = 0;
    int32_t iters = 0;
    while (m > nseg) {
        for (int64_t i = 0; i < m; ++i) {
            uint64_t best = ~(uint64_t)0;
            int64_t bj = -1;
            int64_t jlo = i - radius < 0 ? 0 : i - radius;
            int64_t jhi = i + radius > m - 1 ? m - 1 : i + radius;
            for (int64_t j = jlo; j <= jhi; ++j) {
                if (j == i || cur[j].seg != cur[i].seg) continue;
                uint64_t k = ploc_key(&cur[i], &cur[j], i, j);
                if (k < best) {
                    best = k;
                    bj = j;
                }
            }
            nn[i] = bj;
        }
        int64_t w = 0;
        for (int64_t i = 0; i < m; ++i) {
            int64_t j = nn[i];
            int mutual = (j >= 0 && nn[j] == i);
            if (mutual && i > j) continue; /* merged into the lower position */
            if (mutual) {
                orc_cluster c;
                for (int a = 0; a < 3; ++a) {
                    c.lo[a] = fminf(cur[i].lo[a], cur[j].lo[a]);
                    c.hi[a] = fmaxf(cur[i].hi[a], cur[j].hi[a]);
                }
                children[2 * made] = cur[i].node;
                children[2 * made + 1] = cur[j].node;
                for (int a = 0; a < 3; ++a) {
                    boxes[6 * made + a] = c.lo[a];
                    boxes[6 * made + 3 + a] = c.hi[a];
                }
                c.node = (int32_t)(n + made);
                c.seg = cur[i].seg;
                ++made;
                nxt[w++] = c;
            } else {
                nxt[w++] = cur[i];
            }
        }
        if (w == m) break; /* no progress: cannot happen with a strict total order on pairs */
        orc_cluster* tmp = cur;
        cur = nxt;
        nxt = tmp;
        m = w;
        ++iters;
    }
    if (iterations) *iterations = iters;
    free(cur);
    free(nxt);
    free(nn);
    return made;
}

/* ------------------------------------------------------------------------------------------ */
/* Hierarchical PLOC (after Benthin et al., "H-PLOC", HPG 2024) as built on the device, restated  */
/* sequentially.                                                                                */
/*                                                                                              */
/* The sorted codes define a binary radix tree (LBVH): split s sits between sorted positions s  */
/* and s+1 and has the order key (codes[s] ^ codes[s+1], s ^ (s+1), s), compared                */
/* lexicographically; a split between two segments (meshes) has a key above every other. A node */
/* [l, r] joins its neighbour across the split with the smaller key (Apetrei 2014): split r if   */
/* l == 0 or (r != n-1 and key(r) < key(l-1)), else split l-1; the second of the two children to */
/* arrive at a split goes on with the union of their ranges. Each node holds a list of clusters  */
/* in position order: a leaf holds its triangle; an internal node the left child's list followed */
/* by the right child's, on which PLOC iterations run (the key and mutual-pair rule of orc_ploc, */
/* positions being list indices, radius r) while the list is longer than `threshold`, or longer  */
/* than 1 when the node spans a whole segment (a mesh root: the walk stops there).               */
/*                                                                                              */
/* Node ids are deterministic: internal node ids are n + s for the n - 1 splits s. A list of c   */
/* clusters carries c - 1 unused ids; a node's pool is the left list's unused ids, then n + m    */
/* (its own split m), then the right list's; its merges take ids from the front of the pool in   */
/* creation order (iteration, then position) and the rest go up with its list.                   */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
    uint64_t cx;
    uint32_t ix;
    int64_t s;
    int boundary;
} orc_split_key;

static orc_split_key split_key(const uint64_t* codes, const int32_t* seg, int64_t s) {
    orc_split_key k;
    k.boundary = seg && seg[s] != seg[s + 1];
    k.cx = codes[s] ^ codes[s + 1];
    k.ix = (uint32_t)s ^ (uint32_t)(s + 1);
    k.s = s;
    return k;
}

static int split_less(orc_split_key a, orc_split_key b) {
    if (a.boundary != b.boundary) return a.boundary < b.boundary;
    if (a.cx != b.cx) return a.cx < b.cx;
    if (a.ix != b.ix) return a.ix < b.ix;
    return a.s < b.s;
}

/* PLOC on list L[0..c) in place until c <= target; returns the new count. Merges take ids from pool. */
static int hploc_merge(orc_cluster* L, int c, int target, int radius, const int32_t* pool, int* pool_next,
                       int64_t n, int32_t* children, float* boxes, int32_t* iterations) {
    int nn[64];
    orc_cluster tmp[64];
    while (c > target) {
        for (int i = 0; i < c; ++i) {
            uint64_t best = ~(uint64_t)0;
            int bj = -1;
            int jlo = i - radius < 0 ? 0 : i - radius;
            int jhi = i + radius > c - 1 ? c - 1 : i + radius;
            for (int j = jlo; j <= jhi; ++j) {
                if (j == i) continue;
                uint64_t k = ploc_key(&L[i], &L[j], i, j);
                if (k < best) {
                    best = k;
                    bj = j;
                }
            }
            nn[i] = bj;
        }
        int w = 0;
        for (int i = 0; i < c; ++i) {
            int j = nn[i];
            int mutual = (j >= 0 && nn[j] == i);
            if (mutual && i > j) continue;
            if (mutual) {
                orc_cluster m;
                for (int a = 0; a < 3; ++a) {
                    m.lo[a] = fminf(L[i].lo[a], L[j].lo[a]);
                    m.hi[a] = fmaxf(L[i].hi[a], L[j].hi[a]);
                }
                int32_t id = pool[(*pool_next)++];
                int64_t k = (int64_t)id - n;
                children[2 * k] = L[i].node;
                children[2 * k + 1] = L[j].node;
                for (int a = 0; a < 3; ++a) {
                    boxes[6 * k + a] = m.lo[a];
                    boxes[6 * k + 3 + a] = m.hi[a];
                }
                m.node = id;
                m.seg = L[i].seg;
                tmp[w++] = m;
            } else {
                tmp[w++] = L[i];
            }
        }
        if (iterations) ++*iterations;
        if (w == c) break; /* cannot happen: the pair key is a strict total order */
        memcpy(L, tmp, sizeof(orc_cluster) * (size_t)w);
        c = w;
    }
    return c;
}

/* codes: sorted codes (one per sorted position); perm, seg as in orc_ploc. threshold in [1, 32].
 * children/boxes are indexed by id - n for ids n .. 2n - 2 (minus one per extra segment).
 * Returns the number of internal nodes, or -1 on bad input. */
int64_t orc_hploc_boxes(const float* leaf_boxes, int64_t n, const uint64_t* codes, const int32_t* seg, int radius,
                        int threshold, int32_t* children, float* boxes, int32_t* iterations);

int64_t orc_hploc(const float* tris, int64_t n, const int32_t* perm, const uint64_t* codes, const int32_t* seg,
                  int radius, int threshold, int32_t* children, float* boxes, int32_t* iterations) {
    if (n <= 0) return 0;
    float* lb = (float*)malloc(sizeof(float) * 6 * (size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        const float* p = tris + 9 * (int64_t)perm[i];
        const int fin = tri_finite(p);
        for (int a = 0; a < 3; ++a) {
            lb[6 * i + a] = fin ? fminf(fminf(p[a], p[3 + a]), p[6 + a]) : INFINITY;
            lb[6 * i + 3 + a] = fin ? fmaxf(fmaxf(p[a], p[3 + a]), p[6 + a]) : -INFINITY;
        }
    }
    int64_t r = orc_hploc_boxes(lb, n, codes, seg, radius, threshold, children, boxes, iterations);
    free(lb);
    return r;
}

/* The same over given leaf boxes (6 floats per sorted position: lo xyz, hi xyz), e.g. pre-split references. */
int64_t orc_hploc_boxes(const float* leaf_boxes, int64_t n, const uint64_t* codes, const int32_t* seg, int radius,
                        int threshold, int32_t* children, float* boxes, int32_t* iterations) {
    if (n <= 0) return 0;
    if (radius < 1 || threshold < 1 || threshold > 32) return -1;
    orc_cluster* clus = (orc_cluster*)malloc(sizeof(orc_cluster) * (size_t)n);
    int32_t* fid = (int32_t*)malloc(sizeof(int32_t) * (size_t)n); /* unused ids of the list starting at l */
    int32_t* cnt = (int32_t*)malloc(sizeof(int32_t) * (size_t)n); /* list length of the node starting at l */
    int64_t* other = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 1 ? n - 1 : 1));
    for (int64_t i = 0; i < n; ++i) {
        for (int a = 0; a < 3; ++a) {
            clus[i].lo[a] = leaf_boxes[6 * i + a];
            clus[i].hi[a] = leaf_boxes[6 * i + 3 + a];
        }
        clus[i].node = (int32_t)i;
        clus[i].seg = seg ? seg[i] : 0;
        cnt[i] = 1;
    }
    for (int64_t s = 0; s + 1 < n; ++s) other[s] = -1;
    int64_t made = 0;
    int32_t iters = 0;
    orc_cluster L[64];
    int32_t pool[64];
    for (int64_t i = 0; i < n; ++i) {
        int64_t l = i, r = i;
        for (;;) {
            int segroot = (l == 0 || (seg && seg[l - 1] != seg[l])) && (r == n - 1 || (seg && seg[r] != seg[r + 1]));
            if (segroot) {
                if (l == r) break; /* a one-triangle mesh: its leaf is the root */
                break;
            }
            int64_t split;
            int right_child;
            if (l == 0 || (r != n - 1 && split_less(split_key(codes, seg, r), split_key(codes, seg, l - 1)))) {
                split = r; /* this node is the left child of split r */
                right_child = 0;
            } else {
                split = l - 1;
                right_child = 1;
            }
            if (other[split] < 0) { /* first to arrive: leave the boundary, stop */
                other[split] = right_child ? r : l;
                break;
            }
            int64_t m = split;
            if (right_child) {
                l = other[split];
            } else {
                r = other[split];
            }
            /* combine: left list at [l, l + cl), right list at [m + 1, m + 1 + cr) */
            int cl = cnt[l], cr = cnt[m + 1], c = 0, np = 0;
            for (int k = 0; k < cl; ++k) L[c++] = clus[l + k];
            for (int k = 0; k + 1 < cl; ++k) pool[np++] = fid[l + k];
            pool[np++] = (int32_t)(n + m);
            for (int k = 0; k < cr; ++k) L[c++] = clus[m + 1 + k];
            for (int k = 0; k + 1 < cr; ++k) pool[np++] = fid[m + 1 + k];
            int whole = (l == 0 || (seg && seg[l - 1] != seg[l])) && (r == n - 1 || (seg && seg[r] != seg[r + 1]));
            int used = 0;
            int c_out = hploc_merge(L, c, whole ? 1 : threshold, radius, pool, &used, n, children, boxes, &iters);
            made += used;
            for (int k = 0; k < c_out; ++k) clus[l + k] = L[k];
            for (int k = 0; k + 1 < c_out; ++k) fid[l + k] = pool[used + k];
            cnt[l] = c_out;
        }
    }
    if (iterations) *iterations = iters;
    free(clus);
    free(fid);
    free(cnt);
    free(other);
    return made;
}

/* ------------------------------------------------------------------------------------------ */
/* Re-traversal of the engine's binary layout (as downloaded by dipl_bvh_download_layout), for   */
/* checking its node-visit and triangle-test counters. The traversal is the device's: one step   */
/* is an inner node or a leaf; both child boxes get the conservative slab test (slab distances    */
/* widened by 1e-6 relative, entry beyond the best t + 1e-5 relative pruned), the nearer child is */
/* visited first and the other pushed with its entry t; a leaf tests its triangles with the      */
/* reference Moller-Trumbore (closest-hit rule: t > tmin, smaller t or an equal t at a lower id).  */
/* The device forms the slab distances with an approximate reciprocal of the direction (relative */
/* error below 2^-22) where this uses the IEEE one, so a decision whose two sides lie within     */
/* 1e-6 relative of each other may go either way: such rays are flagged unstable (stable[r] = 0)  */
/* and checks leave them out.                                                                     */
/*                                                                                                */
/* Node: 16 floats: (lx0, hx0, ly0, hy0), (lx1, hx1, ly1, hy1), (lz0, hz0, lz1, hz1), then the two */
/* child references as int bits; a reference < 0 is a leaf ~(first << 3 | count). Leaf triangles: */
/* 12 floats each (v0 xyz, primitive id bits, v1 xyz, 0, v2 xyz, 0).                              */
/* ------------------------------------------------------------------------------------------ */
static int close_rel(float a, float b) {
    if (!isfinite(a) || !isfinite(b)) return 0; /* an infinite side (no hit yet: prune limit +inf) is never close */
    float m = fmaxf(fabsf(a), fabsf(b));
    return fabsf(a - b) <= 1e-6f * m;
}

/* entry t of one box (INFINITY when missed); *unstable |= a decision too close to call */
static float retrace_box(const float* o, const float* inv, float tmin, float lx, float hx, float ly, float hy, float lz,
                         float hz, float t_limit, int* unstable, int* axis, float* numer) {
    float lo[3] = {lx, ly, lz}, hi[3] = {hx, hy, hz};
    float tn = -INFINITY, tf = INFINITY, nn = 0.0f;
    int an = 0;
    for (int a = 0; a < 3; ++a) {
        float d0 = lo[a] - o[a], d1 = hi[a] - o[a];
        float t0 = d0 * inv[a], t1 = d1 * inv[a];
        float n = fminf(t0, t1), f = fmaxf(t0, t1);
        if (a == 0 || n > tn) {
            if (a > 0 && close_rel(n, tn)) *unstable = 1;
            tn = n;
            an = a;
            nn = t0 <= t1 ? d0 : d1;
        } else if (close_rel(n, tn)) {
            *unstable = 1;
        }
        if (a > 0 && close_rel(f, tf)) *unstable = 1;
        tf = a == 0 ? f : fminf(tf, f);
    }
    tn = tn - fabsf(tn) * 1e-6f;
    tf = tf + fabsf(tf) * 1e-6f;
    if (close_rel(tn, tf) || close_rel(tf, tmin) || close_rel(tn, t_limit)) *unstable = 1;
    *axis = an;
    *numer = nn;
    return (tn <= tf && tf >= tmin && tn <= t_limit) ? tn : INFINITY;
}

static float retrace_prune(float best_t) { return best_t + fabsf(best_t) * 1e-5f; }

void orc_retrace_binary(const float* nodes, int64_t num_nodes, const float* tris, int32_t root, const float* rays,
                        int64_t nr, int backface, int64_t* visits, int64_t* tests, uint8_t* stable, int32_t* prim_out,
                        float* t_out) {
    int32_t* sref = (int32_t*)malloc(sizeof(int32_t) * 4096);
    float* st = (float*)malloc(sizeof(float) * 4096);
    for (int64_t r = 0; r < nr; ++r) {
        const float* ray = rays + 8 * r;
        const float* o = ray;
        const float* d = ray + 4;
        float inv[3];
        for (int a = 0; a < 3; ++a) {
            float x = d[a];
            if (fabsf(x) < 1e-20f) x = copysignf(1e-20f, x);
            inv[a] = 1.0f / x;
        }
        float tmin = ray[3], best_t = ray[7];
        int32_t best_prim = -1;
        int found = 0, unstable = 0, sp = 0;
        int64_t v = 0, te = 0;
        int32_t cur = num_nodes > 0 || root < 0 ? root : INT32_MAX;
        const int32_t POP = INT32_MIN, END = INT32_MAX;
        for (int64_t guard = 0; cur != END && guard < 4 * num_nodes + 1024; ++guard) {
            if (cur >= 0) {
                const float* nd = nodes + 16 * (int64_t)cur;
                int32_t ref0, ref1;
                memcpy(&ref0, nd + 12, 4);
                memcpy(&ref1, nd + 13, 4);
                ++v;
                float lim = retrace_prune(best_t);
                int ax0 = 0, ax1 = 0;
                float n0 = 0.0f, n1 = 0.0f;
                float t0 = retrace_box(o, inv, tmin, nd[0], nd[1], nd[2], nd[3], nd[8], nd[9], lim, &unstable, &ax0,
                                       &n0);
                float t1 = retrace_box(o, inv, tmin, nd[4], nd[5], nd[6], nd[7], nd[10], nd[11], lim, &unstable, &ax1,
                                       &n1);
                int h0 = t0 != INFINITY, h1 = t1 != INFINITY;
                if (h0 && h1) {
                    /* two entries from the same slab distance on the same axis are equal under any reciprocal */
                    if (close_rel(t0, t1) && !(ax0 == ax1 && n0 == n1)) unstable = 1;
                    int first0 = t0 <= t1;
                    if (sp >= 4096) { unstable = 1; break; }
                    sref[sp] = first0 ? ref1 : ref0;
                    st[sp] = first0 ? t1 : t0;
                    ++sp;
                    cur = first0 ? ref0 : ref1;
                } else if (h0) {
                    cur = ref0;
                } else if (h1) {
                    cur = ref1;
                } else {
                    cur = POP;
                }
            } else if (cur != POP) {
                int first = (~cur) >> 3, cnt = (~cur) & 7;
                for (int k = 0; k < cnt; ++k) {
                    const float* tp = tris + 12 * (int64_t)(first + k);
                    int32_t pid;
                    memcpy(&pid, tp + 3, 4);
                    float b1 = 0.0f, b2 = 0.0f;
                    float t = orc_mt(tp, tp + 4, tp + 8, o, d, backface, &b1, &b2);
                    ++te;
                    if (t > tmin && t < ORC_INF && (t < best_t || (t == best_t && found && pid < best_prim))) {
                        best_t = t;
                        best_prim = pid;
                        found = 1;
                    }
                }
                cur = POP;
            }
            if (cur == POP) {
                float lim = retrace_prune(best_t);
                cur = END;
                while (sp > 0) {
                    --sp;
                    if (close_rel(st[sp], lim)) unstable = 1;
                    if (st[sp] <= lim) {
                        cur = sref[sp];
                        break;
                    }
                }
            }
        }
        visits[r] = v;
        tests[r] = te;
        stable[r] = (uint8_t)!unstable;
        prim_out[r] = found ? best_prim : -1;
        t_out[r] = found ? best_t : INFINITY;
    }
    free(sref);
    free(st);
}

/* ------------------------------------------------------------------------------------------ */
/* Per-(ray, triangle) re-test: the leaf test of ray r against triangle prim[r] (miss -> t=INF). */
/* ------------------------------------------------------------------------------------------ */
void orc_test_pairs(const float* tris, const float* rays, int64_t nr, const int32_t* prim, int leaf_test,
                    int backface, float* t_out, float* u_out, float* v_out) {
    for (int64_t r = 0; r < nr; ++r) {
        t_out[r] = INFINITY;
        u_out[r] = v_out[r] = 0.0f;
        if (prim[r] < 0) continue;
        const float* q = tris + 9 * (int64_t)prim[r];
        const float* ray = rays + 8 * r;
        float b1 = 0.0f, b2 = 0.0f;
        float t = leaf_test ? orc_wt(q, q + 3, q + 6, ray, ray + 4, backface, &b1, &b2)
                            : orc_mt(q, q + 3, q + 6, ray, ray + 4, backface, &b1, &b2);
        t_out[r] = t;
        u_out[r] = b1;
        v_out[r] = b2;
    }
}

/* ------------------------------------------------------------------------------------------ */
/* GPU frontend restated: pinhole primary rays and cosine-weighted bounce rays, FP32 in the     */
/* device kernels' operation order (IEEE add/mul/div/sqrt only; this file is compiled with      */
/* -ffp-contract=off), so every record must match bit for bit.                                  */
/* Camera basis: the reference renderers' formula (src/renderer/cpu_raytracer.cc:64-70);        */
/* Normalize divides each component by sqrt((x x + y y) + z z) (src/util/vec3.h:111-117).        */
/* ------------------------------------------------------------------------------------------ */
typedef struct { float x, y, z; } orc_v3;
static orc_v3 v3_add(orc_v3 a, orc_v3 b) { orc_v3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static orc_v3 v3_sub(orc_v3 a, orc_v3 b) { orc_v3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static orc_v3 v3_scale(orc_v3 a, float s) { orc_v3 r = {a.x * s, a.y * s, a.z * s}; return r; }
static float v3_dot(orc_v3 a, orc_v3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static orc_v3 v3_cross(orc_v3 a, orc_v3 b) {
    orc_v3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}
static orc_v3 v3_normalize(orc_v3 v) {
    float len = sqrtf(v3_dot(v, v));
    orc_v3 r = {v.x / len, v.y / len, v.z / len};
    return r;
}

/* cam: pos[3], dir[3], up[3], fov, far; rays: width*height records of 8 floats. */
void orc_pinhole_rays(const float* cam, int w, int h, float* rays) {
    orc_v3 pos = {cam[0], cam[1], cam[2]}, dir = {cam[3], cam[4], cam[5]}, up = {cam[6], cam[7], cam[8]};
    float fov = cam[9], far_t = cam[10];
    orc_v3 right = v3_normalize(v3_cross(dir, up));
    float half = fov / 2.0f;
    float gw = (float)(2.0 * tan((double)half));
    float gh = gw * ((float)h / (float)w);
    orc_v3 qw = v3_scale(right, gw / (float)(w - 1));
    orc_v3 nup = {-up.x, -up.y, -up.z};
    orc_v3 qh = v3_scale(nup, gh / (float)(h - 1));
    orc_v3 p00 = v3_add(v3_sub(dir, v3_scale(right, gw / 2.0f)), v3_scale(up, gh / 2.0f));
    for (int64_t i = 0; i < (int64_t)w * h; ++i) {
        float x = (float)(int)(i % w), y = (float)(int)(i / w);
        orc_v3 d = v3_normalize(v3_add(v3_add(p00, v3_scale(qw, x)), v3_scale(qh, y)));
        float* r = rays + 8 * i;
        r[0] = pos.x, r[1] = pos.y, r[2] = pos.z, r[3] = ORC_EPS;
        r[4] = d.x, r[5] = d.y, r[6] = d.z, r[7] = far_t;
    }
}

static uint32_t orc_hash_u32(uint32_t x) { /* HashU32, src/util/util.h:24-32 */
    x ^= x >> 16;
    x *= 0x7FEB352Du;
    x ^= x >> 15;
    x *= 0x846CA68Bu;
    x ^= x >> 16;
    return x;
}
static float orc_u01_key(uint32_t seed, uint32_t stream, uint64_t idx, uint32_t dim) {
    uint32_t k = seed * 0x9E3779B1u + stream * 0x85EBCA6Bu + dim * 0xC2B2AE35u;
    uint32_t lo = (uint32_t)idx, hi = (uint32_t)(idx >> 32);
    uint32_t hh = orc_hash_u32(k ^ orc_hash_u32(lo ^ orc_hash_u32(hi + dim)));
    return (float)(hh >> 8) * (1.0f / 16777216.0f); /* U01FromU32, util.h:34-37 */
}
static float orc_ray_epsilon(orc_v3 p, float t) { /* RayEpsilon, src/scene/ray.h:15-24 */
    float ps = fmaxf(fmaxf(fmaxf(fabsf(p.x), fabsf(p.y)), fabsf(p.z)), 1.0f);
    float ts = fmaxf(t, 1.0f);
    float bias = fmaxf(1e-6f * ps, 1e-7f * ts);
    return fminf(fmaxf(bias, 1e-7f), 1e-3f);
}

/* tris: (N, 3, 3) AoS; rays: n records of 8 floats; prim/t: the hits; out: n bounce rays. */
void orc_bounce_rays(const float* tris, const float* rays, const int32_t* prim, const float* t, int64_t n,
                     uint32_t seed, float* out) {
    for (int64_t i = 0; i < n; ++i) {
        float* q = out + 8 * i;
        if (prim[i] < 0) {
            q[0] = 0.0f, q[1] = 0.0f, q[2] = 0.0f, q[3] = ORC_EPS, q[4] = 0.0f, q[5] = 0.0f, q[6] = 1.0f, q[7] = 0.0f;
            continue;
        }
        const float* r = rays + 8 * i;
        orc_v3 o = {r[0], r[1], r[2]}, din = {r[4], r[5], r[6]};
        const float* tri = tris + 9 * (int64_t)prim[i];
        orc_v3 a = {tri[0], tri[1], tri[2]}, b = {tri[3], tri[4], tri[5]}, c = {tri[6], tri[7], tri[8]};
        orc_v3 ng = v3_cross(v3_sub(b, a), v3_sub(c, a));
        if (!(v3_dot(ng, ng) > 0.0f)) {
            orc_v3 m = {-din.x, -din.y, -din.z};
            ng = m;
        } else {
            ng = v3_normalize(ng);
            if (v3_dot(ng, din) > 0.0f) {
                orc_v3 m = {-ng.x, -ng.y, -ng.z};
                ng = m;
            }
        }
        float dx = 0.0f, dy = 0.0f, r2 = 0.0f;
        for (int k = 0; k < 16; ++k) {
            float x = 2.0f * orc_u01_key(seed, 6u, (uint64_t)i, 2u * (uint32_t)k) - 1.0f;
            float y = 2.0f * orc_u01_key(seed, 6u, (uint64_t)i, 2u * (uint32_t)k + 1u) - 1.0f;
            float qq = x * x + y * y;
            if (qq < 1.0f) {
                dx = x, dy = y, r2 = qq;
                break;
            }
        }
        float dz = sqrtf(1.0f - r2);
        orc_v3 helper = {1.0f, 0.0f, 0.0f};
        if (fabsf(ng.x) > 0.9f) helper.x = 0.0f, helper.y = 1.0f;
        orc_v3 tx = v3_normalize(v3_cross(helper, ng));
        orc_v3 ty = v3_cross(ng, tx);
        orc_v3 d = v3_normalize(v3_add(v3_add(v3_scale(tx, dx), v3_scale(ty, dy)), v3_scale(ng, dz)));
        orc_v3 pos = v3_add(o, v3_scale(din, t[i]));
        float eps = orc_ray_epsilon(pos, t[i]);
        orc_v3 org = v3_add(pos, v3_scale(ng, eps));
        q[0] = org.x, q[1] = org.y, q[2] = org.z, q[3] = ORC_EPS;
        q[4] = d.x, q[5] = d.y, q[6] = d.z, q[7] = ORC_INF;
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Shadow rays of the frontend (dipl_generate_shadow_rays): CpuRaytracer::IsShadowed          */
/* (src/renderer/cpu_raytracer.cc:222-237) around the reference's hit record, with the light     */
/* samples of LocalIlluminationAreaLights (:165-186: RandomAreaLightSample01 :28-40, then       */
/* Triangle::SampleSurface, src/scene/triangle.cc:45-53) and the point lights (:202-218).       */
/* ------------------------------------------------------------------------------------------ */
static float orc_area_light_sample01(uint32_t seed, uint32_t px, uint32_t py, uint32_t light, uint32_t sample,
                                     uint32_t dim) {
    uint32_t key = 0;
    key ^= seed * 0x9e3779b1U;
    key ^= px * 0x165667b1U;
    key ^= py * 0xd3a2646cU;
    key ^= light * 0x85ebca6bU;
    key ^= sample * 0xc2b2ae35U;
    key ^= dim * 0x27d4eb2fU;
    return (float)(orc_hash_u32(key) >> 8) * (1.0f / 16777216.0f);
}

/* Normalize with the reference's cut-off (src/util/vec3.h:111-117). */
static orc_v3 v3_normalize_ref(orc_v3 v) {
    float len = sqrtf(v3_dot(v, v));
    orc_v3 z = {0.0f, 0.0f, 0.0f};
    if (len <= ORC_EPS) return z;
    orc_v3 r = {v.x / len, v.y / len, v.z / len};
    return r;
}

/* out: n * per_hit rays, per_hit = num_area * samples + num_point; area: triangle ids; points: xyz per light. */
void orc_shadow_rays(const float* tris, const float* rays, const int32_t* prim, const float* t, int64_t n, int width,
                     const int32_t* area, int num_area, int samples, const float* points, int num_point, uint32_t seed,
                     float* out) {
    const int per_hit = num_area * samples + num_point;
    for (int64_t i = 0; i < n; ++i) {
        for (int k = 0; k < per_hit; ++k) {
            float* q = out + 8 * (i * per_hit + k);
            q[0] = 0.0f, q[1] = 0.0f, q[2] = 0.0f, q[3] = ORC_EPS, q[4] = 0.0f, q[5] = 0.0f, q[6] = 1.0f, q[7] = 0.0f;
            if (prim[i] < 0) continue;
            orc_v3 light;
            if (k < num_area * samples) {
                int al = k / samples, smp = k - al * samples, lit = 0;
                for (int qq = 0; qq <= al; ++qq)
                    if (area[qq] == prim[i]) lit = 1;
                if (lit) continue;
                uint32_t px = (uint32_t)(i % width), py = (uint32_t)(i / width);
                float r1 = orc_area_light_sample01(seed, px, py, (uint32_t)al, (uint32_t)smp, 0u);
                float r2 = orc_area_light_sample01(seed, px, py, (uint32_t)al, (uint32_t)smp, 1u);
                float u = r1 + r2 > 1.0f ? 1.0f - r1 : r1;
                float w = r1 + r2 > 1.0f ? 1.0f - r2 : r2;
                const float* lt = tris + 9 * (int64_t)area[al];
                orc_v3 a = {lt[0], lt[1], lt[2]}, b = {lt[3], lt[4], lt[5]}, c = {lt[6], lt[7], lt[8]};
                light = v3_add(v3_add(a, v3_scale(v3_sub(b, a), u)), v3_scale(v3_sub(c, a), w));
            } else {
                const float* pl = points + 3 * (k - num_area * samples);
                orc_v3 l = {pl[0], pl[1], pl[2]};
                light = l;
            }
            const float* r = rays + 8 * i;
            orc_v3 o = {r[0], r[1], r[2]}, din = {r[4], r[5], r[6]};
            orc_v3 pos = v3_add(o, v3_scale(din, t[i]));
            float eps = orc_ray_epsilon(pos, t[i]);
            const float* tri = tris + 9 * (int64_t)prim[i];
            orc_v3 a = {tri[0], tri[1], tri[2]}, b = {tri[3], tri[4], tri[5]}, c = {tri[6], tri[7], tri[8]};
            orc_v3 ng = v3_normalize_ref(v3_cross(v3_sub(b, a), v3_sub(c, a)));
            orc_v3 to_light = v3_sub(light, pos);
            float dist = sqrtf(v3_dot(to_light, to_light));
            if (dist < ORC_EPS) continue;
            orc_v3 dir = {to_light.x / dist, to_light.y / dist, to_light.z / dist};
            orc_v3 off = ng;
            if (!(v3_dot(dir, ng) > 0.0f)) off.x = -ng.x, off.y = -ng.y, off.z = -ng.z;
            orc_v3 org = v3_add(pos, v3_scale(off, eps));
            q[0] = org.x, q[1] = org.y, q[2] = org.z, q[3] = ORC_EPS;
            q[4] = dir.x, q[5] = dir.y, q[6] = dir.z, q[7] = dist * (1.0f - eps);
        }
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Pre-splitting of large triangles (the build's split_budget), restated: per mesh, the weights  */
/* q = floor(w 2^32 / D^2) of the triangle boxes (w = (dx dy + dy dz) + dz dx in FP32, D = the     */
/* mesh's vertex-box diagonal), their exact sum Q, the piece counts                                */
/* 1 + min(63, floor(q budget N / (100 Q))), and the pieces: a box of c pieces is split at its    */
/* longest axis' midpoint; each half keeps the polygon of the triangle clipped by the planes of its */
/* halvings (orc_split_half) and that polygon's box clamped to the half (empty: the half itself);   */
/* ceil(c/2) pieces to the lower half first. One mesh (seg = NULL) or meshes of the given sizes in  */
/* input order.                                                                                     */
/* ------------------------------------------------------------------------------------------ */
static uint64_t orc_split_weight(const float* p, float diag) {
    if (!tri_finite(p) || !(diag > 0.0f)) return 0;
    float lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = fminf(fminf(p[a], p[3 + a]), p[6 + a]);
        hi[a] = fmaxf(fmaxf(p[a], p[3 + a]), p[6 + a]);
    }
    float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    float w = (dx * dy + dy * dz) + dz * dx;
    double scale = 4294967296.0 / ((double)diag * (double)diag);
    double q = (double)w * scale;
    return q < 1.8e19 ? (uint64_t)q : (uint64_t)18000000000000000000ull;
}

/* One halving of a piece (the build's split_half): the piece is polygon P (np vertices, the triangle clipped by the
 * planes of the halvings so far) inside box [lo, hi]. The plane x_ax = mid cuts it; the lower (x_ax <= mid) or upper
 * half's polygon Q is P clipped by that plane (Sutherland-Hodgman: vertices on the plane are inside, a crossing point
 * takes mid exactly on axis ax; at most 9 vertices), and its box is Q's box intersected with the half of [lo, hi];
 * an empty Q or box keeps the half. lo and hi are updated in place; returns Q's vertex count. */
#define ORC_POLY_MAX 9
static int orc_split_half(const float (*P)[3], int np, float (*Q)[3], int ax, float mid, int lower, float* lo,
                          float* hi) {
    float bl[3] = {INFINITY, INFINITY, INFINITY}, bh[3] = {-INFINITY, -INFINITY, -INFINITY};
    int nq = 0;
    for (int i = 0; i < np; ++i) {
        const float* p = P[i];
        const float* q = P[i + 1 < np ? i + 1 : 0];
        float pa = p[ax], qa = q[ax];
        int ip = lower ? pa <= mid : pa >= mid, iq = lower ? qa <= mid : qa >= mid;
        if (ip && nq < ORC_POLY_MAX) {
            for (int c = 0; c < 3; ++c) Q[nq][c] = p[c], bl[c] = fminf(bl[c], p[c]), bh[c] = fmaxf(bh[c], p[c]);
            ++nq;
        }
        if (ip != iq && nq < ORC_POLY_MAX) {
            float s = (mid - pa) / (qa - pa);
            for (int c = 0; c < 3; ++c) Q[nq][c] = c == ax ? mid : p[c] + s * (q[c] - p[c]);
            for (int c = 0; c < 3; ++c) bl[c] = fminf(bl[c], Q[nq][c]), bh[c] = fmaxf(bh[c], Q[nq][c]);
            ++nq;
        }
    }
    if (lower) hi[ax] = mid;
    else lo[ax] = mid;
    float nl[3], nh[3];
    int ok = nq > 0;
    for (int c = 0; c < 3; ++c) {
        nl[c] = fmaxf(bl[c], lo[c]);
        nh[c] = fminf(bh[c], hi[c]);
        ok = ok && nl[c] <= nh[c];
    }
    if (ok)
        for (int c = 0; c < 3; ++c) lo[c] = nl[c], hi[c] = nh[c];
    return nq;
}

/* tris: all meshes' triangles in input order; mesh_sizes[nm]. Writes pieces[n] and, when ref_tri != NULL, the
 * references (ref_tri[R], rbox[R][6] = lo xyz, hi xyz). Returns R. */
int64_t orc_presplit(const float* tris, int64_t n, const int64_t* mesh_sizes, int nm, int budget, uint32_t* pieces,
                     int32_t* ref_tri, float* rbox) {
    int64_t first = 0, r = 0;
    for (int k = 0; k < nm; ++k) {
        const float* mt = tris + 9 * first;
        const int64_t nk = mesh_sizes[k];
        float cmin[3], cmax[3], bmin[3], bmax[3];
        orc_scene_bounds(mt, nk, cmin, cmax, bmin, bmax);
        float diag = orc_scene_diag(bmin, bmax);
        uint64_t sum = 0;
        for (int64_t i = 0; i < nk; ++i) sum += orc_split_weight(mt + 9 * i, diag);
        for (int64_t i = 0; i < nk; ++i) {
            uint64_t q = orc_split_weight(mt + 9 * i, diag);
            uint32_t c = 1;
            if (sum != 0 && q != 0) {
                double num = ((double)q * (double)budget) * (double)nk;
                double den = 100.0 * (double)sum;
                double s = floor(num / den);
                c = 1u + (uint32_t)(s < 63.0 ? s : 63.0);
            }
            pieces[first + i] = c;
            const float* p = mt + 9 * i;
            float blo[3], bhi[3];
            for (int a = 0; a < 3; ++a) {
                int fin = tri_finite(p);
                blo[a] = fin ? fminf(fminf(p[a], p[3 + a]), p[6 + a]) : INFINITY;
                bhi[a] = fin ? fmaxf(fmaxf(p[a], p[3 + a]), p[6 + a]) : -INFINITY;
            }
            if (!ref_tri) {
                r += c;
                continue;
            }
            struct {
                float lo[3], hi[3];
                float poly[ORC_POLY_MAX][3];
                int c, np;
            } st[8];
            int sp = 0;
            for (int a = 0; a < 3; ++a) st[0].lo[a] = blo[a], st[0].hi[a] = bhi[a];
            for (int v = 0; v < 3; ++v)
                for (int a = 0; a < 3; ++a) st[0].poly[v][a] = p[3 * v + a];
            st[0].c = (int)c;
            st[0].np = 3;
            sp = 1;
            while (sp > 0) {
                --sp;
                float lo[3], hi[3], poly[ORC_POLY_MAX][3];
                int cc = st[sp].c, np = st[sp].np;
                for (int a = 0; a < 3; ++a) lo[a] = st[sp].lo[a], hi[a] = st[sp].hi[a];
                for (int v = 0; v < np; ++v)
                    for (int a = 0; a < 3; ++a) poly[v][a] = st[sp].poly[v][a];
                if (cc == 1) {
                    ref_tri[r] = (int32_t)(first + i);
                    for (int a = 0; a < 3; ++a) rbox[6 * r + a] = lo[a], rbox[6 * r + 3 + a] = hi[a];
                    ++r;
                    continue;
                }
                float e0 = hi[0] - lo[0], e1 = hi[1] - lo[1], e2 = hi[2] - lo[2];
                int ax = (e0 >= e1 && e0 >= e2) ? 0 : (e1 >= e2 ? 1 : 2);
                float mid = lo[ax] + (hi[ax] - lo[ax]) * 0.5f;
                if (sp + 2 > 8) break;
                /* the upper half is pushed first, so the lower half's pieces come first */
                for (int a = 0; a < 3; ++a) st[sp].lo[a] = lo[a], st[sp].hi[a] = hi[a];
                st[sp].np = orc_split_half((const float (*)[3])poly, np, st[sp].poly, ax, mid, 0, st[sp].lo, st[sp].hi);
                st[sp].c = cc / 2;
                ++sp;
                for (int a = 0; a < 3; ++a) st[sp].lo[a] = lo[a], st[sp].hi[a] = hi[a];
                st[sp].np = orc_split_half((const float (*)[3])poly, np, st[sp].poly, ax, mid, 1, st[sp].lo, st[sp].hi);
                st[sp].c = (cc + 1) / 2;
                ++sp;
            }
        }
        first += nk;
    }
    return r;
}

/* Codes of the references of one mesh (the build's split_refs_kernel): an unsplit triangle's code as orc_morton30 /
 * orc_emc60 compute it; a piece's from its box centre ((lo + hi) * 0.5) and box diagonal. Bounds are the mesh's
 * triangles' (orc_scene_bounds). code_type 0: Morton30, 1: EMC60. */
void orc_ref_codes(const float* tris, int64_t n, const uint32_t* pieces, const int32_t* ref_tri, const float* rbox,
                   int64_t nr, int code_type, uint64_t* codes) {
    float cmin[3], cmax[3], bmin[3], bmax[3];
    orc_scene_bounds(tris, n, cmin, cmax, bmin, bmax);
    float diag = orc_scene_diag(bmin, bmax);
    int bits[4] = {10, 10, 10, 0};
    uint64_t masks[4] = {0, 0, 0, 0};
    float lo4[4] = {cmin[0], cmin[1], cmin[2], 0.0f};
    float ext[4] = {cmax[0] - cmin[0], cmax[1] - cmin[1], cmax[2] - cmin[2], diag};
    float s[4];
    uint64_t top[4];
    if (code_type == 1) orc_emc60_plan(cmin, cmax, diag, bits, masks);
    for (int a = 0; a < 4; ++a) {
        if (code_type == 0) {
            s[a] = a < 3 && ext[a] > 0.0f ? 1024.0f / ext[a] : 0.0f;
            top[a] = 1023;
        } else {
            float cells = ldexpf(1.0f, bits[a]);
            s[a] = (ext[a] > 0.0f && bits[a] > 0) ? cells / ext[a] : 0.0f;
            top[a] = bits[a] >= 64 ? ~(uint64_t)0 : (((uint64_t)1 << bits[a]) - 1);
        }
    }
    for (int64_t r = 0; r < nr; ++r) {
        const int32_t g = ref_tri[r];
        const float* p = tris + 9 * (int64_t)g;
        float x[4], dx, dy, dz;
        if (pieces[g] == 1) {
            centroid(p, x);
            dx = fmaxf(fmaxf(p[0], p[3]), p[6]) - fminf(fminf(p[0], p[3]), p[6]);
            dy = fmaxf(fmaxf(p[1], p[4]), p[7]) - fminf(fminf(p[1], p[4]), p[7]);
            dz = fmaxf(fmaxf(p[2], p[5]), p[8]) - fminf(fminf(p[2], p[5]), p[8]);
        } else {
            const float* b = rbox + 6 * r;
            for (int a = 0; a < 3; ++a) x[a] = (b[a] + b[3 + a]) * 0.5f;
            dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
        }
        if (code_type == 0) {
            uint32_t q[3];
            for (int a = 0; a < 3; ++a) {
                float v = (x[a] - cmin[a]) * s[a];
                v = fminf(fmaxf(v, 0.0f), 1023.0f);
                q[a] = (uint32_t)v;
            }
            codes[r] = (uint64_t)((expand10(q[0]) << 2) | (expand10(q[1]) << 1) | expand10(q[2]));
            continue;
        }
        x[3] = sqrtf((dx * dx + dy * dy) + dz * dz);
        uint64_t code = 0;
        for (int a = 0; a < 4; ++a) {
            if (bits[a] == 0) continue;
            float q = fmaxf((x[a] - lo4[a]) * s[a], 0.0f);
            uint64_t qi = q < 1.8e19f ? (uint64_t)q : top[a];
            if (qi > top[a]) qi = top[a];
            code |= deposit(qi, masks[a]);
        }
        codes[r] = code;
    }
}
