// Ray/triangle tests shared by the trace, any-hit and adjoint kernels.
#pragma once

#include "common.cuh"

namespace dipl {

// The reference Moller-Trumbore test, Triangle::IntersectRay (src/scene/triangle.cc:10-43), operation for
// operation with explicit round-to-nearest intrinsics (no FMA contraction, IEEE reciprocal), so the bits
// of t, b1 and b2 equal the reference CPU build's. Returns t, or kInfinity on a miss (like the reference).
__device__ __forceinline__ float mt_ref(float3 a, float3 b, float3 c, float3 o, float3 d, bool backface, float& b1o,
                                        float& b2o) {
    const float e1x = __fsub_rn(b.x, a.x), e1y = __fsub_rn(b.y, a.y), e1z = __fsub_rn(b.z, a.z);
    const float e2x = __fsub_rn(c.x, a.x), e2y = __fsub_rn(c.y, a.y), e2z = __fsub_rn(c.z, a.z);
    const float px = __fsub_rn(__fmul_rn(d.y, e2z), __fmul_rn(d.z, e2y));
    const float py = __fsub_rn(__fmul_rn(d.z, e2x), __fmul_rn(d.x, e2z));
    const float pz = __fsub_rn(__fmul_rn(d.x, e2y), __fmul_rn(d.y, e2x));
    const float det = __fadd_rn(__fadd_rn(__fmul_rn(e1x, px), __fmul_rn(e1y, py)), __fmul_rn(e1z, pz));
    if (backface) {
        if (det < kEpsilon) return kInfinity;
    } else {
        if (fabsf(det) < kEpsilon) return kInfinity;
    }
    const float inv = __frcp_rn(det);
    const float tx = __fsub_rn(o.x, a.x), ty = __fsub_rn(o.y, a.y), tz = __fsub_rn(o.z, a.z);
    const float b1 = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(tx, px), __fmul_rn(ty, py)), __fmul_rn(tz, pz)), inv);
    if (b1 < 0.0f || b1 > 1.0f) return kInfinity;
    const float qx = __fsub_rn(__fmul_rn(ty, e1z), __fmul_rn(tz, e1y));
    const float qy = __fsub_rn(__fmul_rn(tz, e1x), __fmul_rn(tx, e1z));
    const float qz = __fsub_rn(__fmul_rn(tx, e1y), __fmul_rn(ty, e1x));
    const float b2 = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(d.x, qx), __fmul_rn(d.y, qy)), __fmul_rn(d.z, qz)), inv);
    if (b2 < 0.0f || __fadd_rn(b1, b2) > 1.0f) return kInfinity;
    const float t = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(e2x, qx), __fmul_rn(e2y, qy)), __fmul_rn(e2z, qz)), inv);
    b1o = b1;
    b2o = b2;
    return t;
}

// Per-ray set-up of the watertight test (Woop, Benthin & Wald, JCGT 2013): the axis of largest |d|
// becomes z, the other two keep a right-handed order, and a shear maps the ray onto +z.
struct WtRay {
    int kx, ky, kz;
    float sx, sy, sz;
};

__device__ __forceinline__ float comp(float3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

__device__ __forceinline__ WtRay wt_setup(float3 d) {
    WtRay w;
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    w.kz = (ax > ay) ? ((ax > az) ? 0 : 2) : ((ay > az) ? 1 : 2);
    w.kx = w.kz + 1 == 3 ? 0 : w.kz + 1;
    w.ky = w.kx + 1 == 3 ? 0 : w.kx + 1;
    const float dz = comp(d, w.kz);
    if (dz < 0.0f) {
        int t = w.kx;
        w.kx = w.ky;
        w.ky = t;
    }
    w.sx = __fdiv_rn(comp(d, w.kx), dz);
    w.sy = __fdiv_rn(comp(d, w.ky), dz);
    w.sz = __frcp_rn(dz);
    return w;
}

// Watertight test; FP32 with the paper's FP64 recomputation of zero edge functions. Backface culling
// keeps the reference's meaning (hit only if e1.(d x e2) > 0, i.e. det > 0 here).
__device__ __forceinline__ float wt_test(float3 v0, float3 v1, float3 v2, float3 o, const WtRay& w, bool backface,
                                         float& b1o, float& b2o) {
    const float3 A = make_float3(__fsub_rn(v0.x, o.x), __fsub_rn(v0.y, o.y), __fsub_rn(v0.z, o.z));
    const float3 B = make_float3(__fsub_rn(v1.x, o.x), __fsub_rn(v1.y, o.y), __fsub_rn(v1.z, o.z));
    const float3 C = make_float3(__fsub_rn(v2.x, o.x), __fsub_rn(v2.y, o.y), __fsub_rn(v2.z, o.z));
    const float Akz = comp(A, w.kz), Bkz = comp(B, w.kz), Ckz = comp(C, w.kz);
    const float Ax = __fsub_rn(comp(A, w.kx), __fmul_rn(w.sx, Akz)), Ay = __fsub_rn(comp(A, w.ky), __fmul_rn(w.sy, Akz));
    const float Bx = __fsub_rn(comp(B, w.kx), __fmul_rn(w.sx, Bkz)), By = __fsub_rn(comp(B, w.ky), __fmul_rn(w.sy, Bkz));
    const float Cx = __fsub_rn(comp(C, w.kx), __fmul_rn(w.sx, Ckz)), Cy = __fsub_rn(comp(C, w.ky), __fmul_rn(w.sy, Ckz));
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = __double2float_rn(__dsub_rn(__dmul_rn((double)Cx, (double)By), __dmul_rn((double)Cy, (double)Bx)));
        V = __double2float_rn(__dsub_rn(__dmul_rn((double)Ax, (double)Cy), __dmul_rn((double)Ay, (double)Cx)));
        W = __double2float_rn(__dsub_rn(__dmul_rn((double)Bx, (double)Ay), __dmul_rn((double)By, (double)Ax)));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return kInfinity;
    const float det = __fadd_rn(__fadd_rn(U, V), W);
    if (det == 0.0f) return kInfinity;
    if (backface && det < 0.0f) return kInfinity;
    const float Az = __fmul_rn(w.sz, Akz), Bz = __fmul_rn(w.sz, Bkz), Cz = __fmul_rn(w.sz, Ckz);
    const float T = __fadd_rn(__fadd_rn(__fmul_rn(U, Az), __fmul_rn(V, Bz)), __fmul_rn(W, Cz));
    const float rcp = __frcp_rn(det);
    b1o = __fmul_rn(V, rcp);
    b2o = __fmul_rn(W, rcp);
    return __fmul_rn(T, rcp);
}

// FP64 Cramer's-rule intersection (oracle re-intersection; no epsilon, inclusive edges).
__device__ __forceinline__ bool f64_hit(double3 a, double3 b, double3 c, double3 o, double3 d, double& t, double& u,
                                        double& v) {
    const double e1x = b.x - a.x, e1y = b.y - a.y, e1z = b.z - a.z;
    const double e2x = c.x - a.x, e2y = c.y - a.y, e2z = c.z - a.z;
    const double sx = o.x - a.x, sy = o.y - a.y, sz = o.z - a.z;
    const double px = d.y * e2z - d.z * e2y, py = d.z * e2x - d.x * e2z, pz = d.x * e2y - d.y * e2x;
    const double det = e1x * px + e1y * py + e1z * pz;
    if (det == 0.0) return false;
    const double inv = 1.0 / det;
    u = (sx * px + sy * py + sz * pz) * inv;
    const double qx = sy * e1z - sz * e1y, qy = sz * e1x - sx * e1z, qz = sx * e1y - sy * e1x;
    v = (d.x * qx + d.y * qy + d.z * qz) * inv;
    t = (e2x * qx + e2y * qy + e2z * qz) * inv;
    return u >= 0.0 && v >= 0.0 && u + v <= 1.0;
}

}  // namespace dipl
