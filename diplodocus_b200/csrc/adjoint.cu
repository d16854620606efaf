// Differentiation form: hand-written adjoint of the closest-hit (t, u, v) with respect to the triangle's
// vertices and the ray's origin and direction, plus the FP64 re-intersection used as the error oracle.
//
// With s = o - v0, e1 = v1 - v0, e2 = v2 - v0 and A = [-d | e1 | e2], the hit solves A (t, u, v)^T = s.
// For an upstream gradient g = dL/d(t, u, v), lambda = A^-T g, and
//   dL/do = lambda,  dL/dd = t lambda,  dL/dv1 = -u lambda,  dL/dv2 = -v lambda,  dL/dv0 = -(1 - u - v) lambda.
// A^-T g = [g_t (e1 x e2) + g_u (e2 x -d) + g_v (-d x e1)] / det(A). The hit id is held fixed: visibility is
// discrete, so the derivative is the one of the smooth (t, u, v) of the triangle that was hit.
#include "internal.h"
#include "intersect.cuh"

namespace dipl {
namespace {

__device__ __forceinline__ float3 ld3(const float* p, long long i) {
    return make_float3(__ldg(p + 3 * i), __ldg(p + 3 * i + 1), __ldg(p + 3 * i + 2));
}
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

__global__ void adjoint_kernel(const float* __restrict__ v0, const float* __restrict__ v1, const float* __restrict__ v2,
                               const dipl_ray* __restrict__ rays, const dipl_hit* __restrict__ hits,
                               const float* __restrict__ dtuv, int64_t n, float* dv0, float* dv1, float* dv2,
                               float* __restrict__ dorig, float* __restrict__ ddir) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const dipl_hit h = hits[i];
    float3 lam = make_float3(0.f, 0.f, 0.f), gd = lam;
    if (h.prim >= 0) {
        const dipl_ray r = rays[i];
        const float3 d = make_float3(r.dx, r.dy, r.dz);
        const float3 a = ld3(v0, h.prim), b = ld3(v1, h.prim), c = ld3(v2, h.prim);
        const float3 e1 = sub3(b, a), e2 = sub3(c, a), nd = make_float3(-d.x, -d.y, -d.z);
        const float3 c12 = cross3(e1, e2), c20 = cross3(e2, nd), c01 = cross3(nd, e1);
        const float det = dot3(nd, c12);
        const float gt = dtuv[3 * i], gu = dtuv[3 * i + 1], gv = dtuv[3 * i + 2];
        if (det != 0.0f) {
            const float inv = 1.0f / det;
            lam = make_float3((gt * c12.x + gu * c20.x + gv * c01.x) * inv, (gt * c12.y + gu * c20.y + gv * c01.y) * inv,
                              (gt * c12.z + gu * c20.z + gv * c01.z) * inv);
            gd = make_float3(h.t * lam.x, h.t * lam.y, h.t * lam.z);
            const float w0 = -(1.0f - h.u - h.v);
            float* p0 = dv0 + 3 * (int64_t)h.prim;
            float* p1 = dv1 + 3 * (int64_t)h.prim;
            float* p2 = dv2 + 3 * (int64_t)h.prim;
            atomicAdd(p0, w0 * lam.x), atomicAdd(p0 + 1, w0 * lam.y), atomicAdd(p0 + 2, w0 * lam.z);
            atomicAdd(p1, -h.u * lam.x), atomicAdd(p1 + 1, -h.u * lam.y), atomicAdd(p1 + 2, -h.u * lam.z);
            atomicAdd(p2, -h.v * lam.x), atomicAdd(p2 + 1, -h.v * lam.y), atomicAdd(p2 + 2, -h.v * lam.z);
        }
    }
    if (dorig) dorig[3 * i] = lam.x, dorig[3 * i + 1] = lam.y, dorig[3 * i + 2] = lam.z;
    if (ddir) ddir[3 * i] = gd.x, ddir[3 * i + 1] = gd.y, ddir[3 * i + 2] = gd.z;
}

__global__ void reintersect_kernel(const float* __restrict__ v0, const float* __restrict__ v1,
                                   const float* __restrict__ v2, const dipl_ray* __restrict__ rays,
                                   const dipl_hit* __restrict__ hits, int64_t n, double* __restrict__ tuv) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const dipl_hit h = hits[i];
    double t = __longlong_as_double(0x7FF0000000000000ll), u = 0.0, v = 0.0;
    if (h.prim >= 0) {
        const dipl_ray r = rays[i];
        auto dbl = [](float3 f) { return make_double3(f.x, f.y, f.z); };
        f64_hit(dbl(ld3(v0, h.prim)), dbl(ld3(v1, h.prim)), dbl(ld3(v2, h.prim)), make_double3(r.ox, r.oy, r.oz),
                make_double3(r.dx, r.dy, r.dz), t, u, v);
    }
    tuv[3 * i] = t, tuv[3 * i + 1] = u, tuv[3 * i + 2] = v;
}

}  // namespace

dipl_status trace_adjoint(const float* v0, const float* v1, const float* v2, const dipl_ray* rays,
                          const dipl_hit* hits, const float* dtuv, int64_t n, float* dv0, float* dv1, float* dv2,
                          float* dorig, float* ddir, cudaStream_t s) {
    DIPL_CHECK_ARG(n >= 0, "n must be >= 0");
    if (n == 0) return DIPL_OK;
    DIPL_CHECK_ARG(v0 && v1 && v2 && rays && hits && dtuv && dv0 && dv1 && dv2, "arrays must be non-NULL");
    adjoint_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(v0, v1, v2, rays, hits, dtuv, n, dv0, dv1, dv2, dorig,
                                                                ddir); note_launches();
    DIPL_CUDA(cudaGetLastError());
    return DIPL_OK;
}

dipl_status reintersect_f64(const float* v0, const float* v1, const float* v2, const dipl_ray* rays,
                            const dipl_hit* hits, int64_t n, double* tuv, cudaStream_t s) {
    DIPL_CHECK_ARG(n >= 0, "n must be >= 0");
    if (n == 0) return DIPL_OK;
    DIPL_CHECK_ARG(v0 && v1 && v2 && rays && hits && tuv, "arrays must be non-NULL");
    reintersect_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(v0, v1, v2, rays, hits, n, tuv); note_launches();
    DIPL_CUDA(cudaGetLastError());
    return DIPL_OK;
}

}  // namespace dipl
