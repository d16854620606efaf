// GPU frontend: wavefront ray generation for the renderer path that traces through the engine
// (generate -> dipl_bvh_trace_closest -> bounce -> dipl_bvh_trace_closest), replacing the per-pixel set-up
// of RaytracingBounceKernel (src/gpu/renderer/gpu_renderer_api.cu:43-53) and the next-segment sampling of
// TracePath (src/gpu/renderer/gpu_pathtracer.cu:12), which the reference runs around DummyIntersect.
//
// Both kernels use only IEEE add, mul, div and sqrt in FP32, in a fixed order and without FMA contraction
// (explicit _rn intrinsics), so the host restatement reproduces every record bit for bit.
#include <cmath>

#include "internal.h"

namespace dipl {
namespace {

constexpr int kGenThreads = 256;
constexpr uint32_t kBounceStream = 6;  // hash stream of bounce sampling (distinct from the other uses of a seed)
constexpr int kDiskTries = 16;         // rejection draws for a point of the unit disk (fails with p < 1e-10)

struct V3 {
    float x, y, z;
};

__device__ __forceinline__ V3 v_add(V3 a, V3 b) { return {__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)}; }
__device__ __forceinline__ V3 v_sub(V3 a, V3 b) { return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)}; }
__device__ __forceinline__ V3 v_scale(V3 a, float s) { return {__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)}; }
__device__ __forceinline__ float v_dot(V3 a, V3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
// Cross (src/util/vec3.h:119-121): (a.y b.z - a.z b.y, a.z b.x - a.x b.z, a.x b.y - a.y b.x).
__device__ __forceinline__ V3 v_cross(V3 a, V3 b) {
    return {__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
            __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x))};
}
// v / |v|, |v| = sqrt((x x + y y) + z z), each component divided (Normalize, src/util/vec3.h:111-117).
__device__ __forceinline__ V3 v_normalize(V3 v) {
    const float len = __fsqrt_rn(v_dot(v, v));
    return {__fdiv_rn(v.x, len), __fdiv_rn(v.y, len), __fdiv_rn(v.z, len)};
}

// HashU32 (src/util/util.h:24-32) and the (seed, stream, index, dimension) key of the workload generators.
__device__ __forceinline__ uint32_t hash_u32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7FEB352Du;
    x ^= x >> 15;
    x *= 0x846CA68Bu;
    x ^= x >> 16;
    return x;
}
__device__ __forceinline__ float u01_key(uint32_t seed, uint32_t stream, uint64_t idx, uint32_t dim) {
    const uint32_t k = seed * 0x9E3779B1u + stream * 0x85EBCA6Bu + dim * 0xC2B2AE35u;
    const uint32_t lo = (uint32_t)idx, hi = (uint32_t)(idx >> 32);
    const uint32_t h = hash_u32(k ^ hash_u32(lo ^ hash_u32(hi + dim)));
    return (float)(h >> 8) * (1.0f / 16777216.0f);  // U01FromU32 (util.h:34-37): exact in FP32
}

struct CameraBasis {
    V3 pos, p00, qw, qh;
    float far_t;
};

__global__ void __launch_bounds__(kGenThreads) pinhole_kernel(CameraBasis cb, int width, int64_t n,
                                                              dipl_ray* __restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)kGenThreads + threadIdx.x;
    if (i >= n) return;
    const float x = (float)(int)(i % width), y = (float)(int)(i / width);
    const V3 d = v_normalize(v_add(v_add(cb.p00, v_scale(cb.qw, x)), v_scale(cb.qh, y)));
    float4* o4 = reinterpret_cast<float4*>(out + i);
    o4[0] = make_float4(cb.pos.x, cb.pos.y, cb.pos.z, kEpsilon);
    o4[1] = make_float4(d.x, d.y, d.z, cb.far_t);
}

// RayEpsilon (src/scene/ray.h:15-24).
__device__ __forceinline__ float ray_epsilon(V3 p, float t) {
    const float p_scale = fmaxf(fmaxf(fmaxf(fabsf(p.x), fabsf(p.y)), fabsf(p.z)), 1.0f);
    const float t_scale = fmaxf(t, 1.0f);
    const float bias = fmaxf(__fmul_rn(1e-6f, p_scale), __fmul_rn(1e-7f, t_scale));
    return fminf(fmaxf(bias, 1e-7f), 1e-3f);
}

__global__ void __launch_bounds__(kGenThreads) bounce_kernel(const float* __restrict__ v0, const float* __restrict__ v1,
                                                             const float* __restrict__ v2,
                                                             const dipl_ray* __restrict__ rays,
                                                             const dipl_hit* __restrict__ hits, int64_t n,
                                                             uint32_t seed, dipl_ray* __restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)kGenThreads + threadIdx.x;
    if (i >= n) return;
    const int4 h = __ldg(reinterpret_cast<const int4*>(hits) + i);
    float4* o4 = reinterpret_cast<float4*>(out + i);
    if (h.x < 0) {  // a miss: a ray that can hit nothing (tmin > tmax)
        o4[0] = make_float4(0.0f, 0.0f, 0.0f, kEpsilon);
        o4[1] = make_float4(0.0f, 0.0f, 1.0f, 0.0f);
        return;
    }
    const float4 ra = __ldg(reinterpret_cast<const float4*>(rays + i)), rb = __ldg(reinterpret_cast<const float4*>(rays + i) + 1);
    const V3 o = {ra.x, ra.y, ra.z}, din = {rb.x, rb.y, rb.z};
    const float t = __int_as_float(h.y);
    const int64_t p = h.x;
    const V3 a = {__ldg(v0 + 3 * p), __ldg(v0 + 3 * p + 1), __ldg(v0 + 3 * p + 2)};
    const V3 b = {__ldg(v1 + 3 * p), __ldg(v1 + 3 * p + 1), __ldg(v1 + 3 * p + 2)};
    const V3 c = {__ldg(v2 + 3 * p), __ldg(v2 + 3 * p + 1), __ldg(v2 + 3 * p + 2)};
    V3 ng = v_cross(v_sub(b, a), v_sub(c, a));
    const float len2 = v_dot(ng, ng);
    if (!(len2 > 0.0f)) {
        ng = {-din.x, -din.y, -din.z};  // degenerate triangle: the normal faces the ray
    } else {
        ng = v_normalize(ng);
        if (v_dot(ng, din) > 0.0f) ng = {-ng.x, -ng.y, -ng.z};  // facing the incoming ray
    }
    // a point of the unit disk by rejection, lifted to the hemisphere: cosine-weighted (Malley's method)
    float dx = 0.0f, dy = 0.0f, r2 = 0.0f;
    for (int k = 0; k < kDiskTries; ++k) {
        const float x = __fsub_rn(__fmul_rn(2.0f, u01_key(seed, kBounceStream, (uint64_t)i, 2u * k)), 1.0f);
        const float y = __fsub_rn(__fmul_rn(2.0f, u01_key(seed, kBounceStream, (uint64_t)i, 2u * k + 1u)), 1.0f);
        const float q = __fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y));
        if (q < 1.0f) {
            dx = x, dy = y, r2 = q;
            break;
        }
    }
    const float dz = __fsqrt_rn(__fsub_rn(1.0f, r2));
    const V3 helper = fabsf(ng.x) > 0.9f ? V3{0.0f, 1.0f, 0.0f} : V3{1.0f, 0.0f, 0.0f};
    const V3 tx = v_normalize(v_cross(helper, ng));
    const V3 ty = v_cross(ng, tx);
    const V3 d = v_normalize(v_add(v_add(v_scale(tx, dx), v_scale(ty, dy)), v_scale(ng, dz)));
    const V3 pos = v_add(o, v_scale(din, t));  // Ray::At (src/scene/ray.h:13)
    const float eps = ray_epsilon(pos, t);
    const V3 org = v_add(pos, v_scale(ng, eps));  // d lies on ng's side: OffsetRayOrigin's offset is +ng
    o4[0] = make_float4(org.x, org.y, org.z, kEpsilon);
    o4[1] = make_float4(d.x, d.y, d.z, kInfinity);
}

// Normalize with the reference's cut-off (src/util/vec3.h:111-117): a vector of length <= kEpsilon becomes 0.
__device__ __forceinline__ V3 v_normalize_ref(V3 v) {
    const float len = __fsqrt_rn(v_dot(v, v));
    if (len <= kEpsilon) return {0.0f, 0.0f, 0.0f};
    return {__fdiv_rn(v.x, len), __fdiv_rn(v.y, len), __fdiv_rn(v.z, len)};
}

// RandomAreaLightSample01 (src/renderer/cpu_raytracer.cc:28-40): a key of seed, pixel, light and sample, hashed.
__device__ __forceinline__ float area_light_sample01(uint32_t seed, uint32_t px, uint32_t py, uint32_t light,
                                                     uint32_t sample, uint32_t dim) {
    uint32_t key = 0;
    key ^= seed * 0x9e3779b1U;
    key ^= px * 0x165667b1U;
    key ^= py * 0xd3a2646cU;
    key ^= light * 0x85ebca6bU;
    key ^= sample * 0xc2b2ae35U;
    key ^= dim * 0x27d4eb2fU;
    return (float)(hash_u32(key) >> 8) * (1.0f / 16777216.0f);
}

__device__ __forceinline__ V3 ld_v3(const float* p, int64_t i) { return {__ldg(p + 3 * i), __ldg(p + 3 * i + 1), __ldg(p + 3 * i + 2)}; }

// One shadow ray per (hit, light sample): CpuRaytracer::IsShadowed (src/renderer/cpu_raytracer.cc:222-237) with the
// hit record of the closest-hit trace (position Ray::At(t), RayEpsilon, the triangle's geometric normal) and the
// light sample of LocalIlluminationAreaLights (:165-186; Triangle::SampleSurface, src/scene/triangle.cc:45-53) or
// a point light (:202-218). Rays that cast nothing get tmax = 0 (never occluded).
__global__ void __launch_bounds__(kGenThreads) shadow_kernel(const float* __restrict__ v0, const float* __restrict__ v1,
                                                             const float* __restrict__ v2,
                                                             const dipl_ray* __restrict__ rays,
                                                             const dipl_hit* __restrict__ hits, int64_t n, int width,
                                                             const int32_t* __restrict__ area, int num_area,
                                                             int samples, const float* __restrict__ points,
                                                             int num_point, uint32_t seed, dipl_ray* __restrict__ out) {
    const int per_hit = num_area * samples + num_point;
    const int64_t j = blockIdx.x * (int64_t)kGenThreads + threadIdx.x;
    if (j >= n * per_hit) return;
    const int64_t i = j / per_hit;
    const int k = (int)(j - i * per_hit);
    float4* o4 = reinterpret_cast<float4*>(out + j);
    const float4 none0 = make_float4(0.0f, 0.0f, 0.0f, kEpsilon), none1 = make_float4(0.0f, 0.0f, 1.0f, 0.0f);
    const int4 h = __ldg(reinterpret_cast<const int4*>(hits) + i);
    if (h.x < 0) {
        o4[0] = none0, o4[1] = none1;
        return;
    }
    V3 light;
    if (k < num_area * samples) {
        const int al = k / samples, smp = k - al * samples;
        for (int q = 0; q <= al; ++q)  // the hit is an area light: the reference returns its colour, no more rays
            if (__ldg(area + q) == h.x) {
                o4[0] = none0, o4[1] = none1;
                return;
            }
        const uint32_t px = (uint32_t)(i % width), py = (uint32_t)(i / width);
        const float r1 = area_light_sample01(seed, px, py, (uint32_t)al, (uint32_t)smp, 0u);
        const float r2 = area_light_sample01(seed, px, py, (uint32_t)al, (uint32_t)smp, 1u);
        const bool flip = __fadd_rn(r1, r2) > 1.0f;
        const float u = flip ? __fsub_rn(1.0f, r1) : r1, w = flip ? __fsub_rn(1.0f, r2) : r2;
        const int64_t lt = __ldg(area + al);
        const V3 a = ld_v3(v0, lt), b = ld_v3(v1, lt), c = ld_v3(v2, lt);
        light = v_add(v_add(a, v_scale(v_sub(b, a), u)), v_scale(v_sub(c, a), w));
    } else {
        const int pl = k - num_area * samples;
        light = {__ldg(points + 3 * pl), __ldg(points + 3 * pl + 1), __ldg(points + 3 * pl + 2)};
    }
    const float4 ra = __ldg(reinterpret_cast<const float4*>(rays + i)), rb = __ldg(reinterpret_cast<const float4*>(rays + i) + 1);
    const float t = __int_as_float(h.y);
    const V3 pos = v_add(V3{ra.x, ra.y, ra.z}, v_scale(V3{rb.x, rb.y, rb.z}, t));  // Ray::At
    const float eps = ray_epsilon(pos, t);
    const int64_t p = h.x;
    const V3 ta = ld_v3(v0, p), tb = ld_v3(v1, p), tc = ld_v3(v2, p);
    const V3 ng = v_normalize_ref(v_cross(v_sub(tb, ta), v_sub(tc, ta)));  // RecomputeTriangleGeometricNormal
    const V3 to_light = v_sub(light, pos);
    const float dist = __fsqrt_rn(v_dot(to_light, to_light));  // Length
    if (dist < kEpsilon) {  // on the light's surface: not shadowed
        o4[0] = none0, o4[1] = none1;
        return;
    }
    const V3 dir = {__fdiv_rn(to_light.x, dist), __fdiv_rn(to_light.y, dist), __fdiv_rn(to_light.z, dist)};
    const V3 off = v_dot(dir, ng) > 0.0f ? ng : V3{-ng.x, -ng.y, -ng.z};  // OffsetRayOrigin (:42-47)
    const V3 org = v_add(pos, v_scale(off, eps));
    o4[0] = make_float4(org.x, org.y, org.z, kEpsilon);
    o4[1] = make_float4(dir.x, dir.y, dir.z, __fmul_rn(dist, __fsub_rn(1.0f, eps)));
}

// Camera basis on the host, the reference renderers' formula (cpu_raytracer.cc:64-70) in FP32; 2 tan(fov/2) is
// evaluated once in double precision (tan of the FP32 half angle, rounded to FP32).
CameraBasis camera_basis(const dipl_camera& c, int w, int h) {
    auto add = [](V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; };
    auto sub = [](V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; };
    auto scale = [](V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; };
    auto cross = [](V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; };
    auto normalize = [](V3 v) {
        volatile float s = (v.x * v.x + v.y * v.y) + v.z * v.z;  // no contraction: separate products and sums
        const float len = std::sqrt((float)s);
        return V3{v.x / len, v.y / len, v.z / len};
    };
    const V3 dir = {c.dir[0], c.dir[1], c.dir[2]}, up = {c.up[0], c.up[1], c.up[2]};
    const V3 right = normalize(cross(dir, up));
    const float half = c.fov / 2.0f;
    const float gw = (float)(2.0 * std::tan((double)half));
    const float gh = gw * ((float)h / (float)w);
    const V3 qw = scale(right, gw / (float)(w - 1));
    const V3 qh = scale(V3{-up.x, -up.y, -up.z}, gh / (float)(h - 1));
    const V3 p00 = add(sub(dir, scale(right, gw / 2.0f)), scale(up, gh / 2.0f));
    CameraBasis cb;
    cb.pos = {c.pos[0], c.pos[1], c.pos[2]};
    cb.p00 = p00, cb.qw = qw, cb.qh = qh, cb.far_t = c.far_t;
    return cb;
}

}  // namespace
}  // namespace dipl

using namespace dipl;

extern "C" dipl_status dipl_generate_pinhole_rays(const dipl_camera* camera, int32_t width, int32_t height,
                                                  dipl_ray* d_rays, void* stream) {
    DIPL_CHECK_ARG(camera && width >= 2 && height >= 2, "camera must be non-NULL and width, height >= 2");
    DIPL_CHECK_ARG(d_rays && (reinterpret_cast<uintptr_t>(d_rays) & 15) == 0, "d_rays must be 16-byte aligned");
    const int64_t n = (int64_t)width * height;
    const CameraBasis cb = camera_basis(*camera, width, height);
    pinhole_kernel<<<(unsigned)((n + kGenThreads - 1) / kGenThreads), kGenThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        cb, width, n, d_rays);
    note_launches();
    DIPL_CUDA(cudaGetLastError());
    return DIPL_OK;
}

extern "C" dipl_status dipl_generate_bounce_rays(const float* d_v0, const float* d_v1, const float* d_v2,
                                                 const dipl_ray* d_rays, const dipl_hit* d_hits, int64_t n,
                                                 uint32_t seed, dipl_ray* d_out, void* stream) {
    DIPL_CHECK_ARG(n >= 0, "n must be >= 0");
    if (n == 0) return DIPL_OK;
    DIPL_CHECK_ARG(d_v0 && d_v1 && d_v2 && d_rays && d_hits && d_out, "arrays must be non-NULL");
    DIPL_CHECK_ARG((reinterpret_cast<uintptr_t>(d_rays) & 15) == 0 && (reinterpret_cast<uintptr_t>(d_hits) & 15) == 0 &&
                       (reinterpret_cast<uintptr_t>(d_out) & 15) == 0,
                   "rays, hits and output must be 16-byte aligned");
    DIPL_CHECK_ARG(d_out != d_rays, "d_out may not alias d_rays");
    bounce_kernel<<<(unsigned)((n + kGenThreads - 1) / kGenThreads), kGenThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        d_v0, d_v1, d_v2, d_rays, d_hits, n, seed, d_out);
    note_launches();
    DIPL_CUDA(cudaGetLastError());
    return DIPL_OK;
}

extern "C" dipl_status dipl_generate_shadow_rays(const float* d_v0, const float* d_v1, const float* d_v2,
                                                 const dipl_ray* d_rays, const dipl_hit* d_hits, int64_t n,
                                                 int32_t width, const int32_t* d_area_light_triangles,
                                                 int32_t num_area_lights, int32_t samples, const float* d_point_lights,
                                                 int32_t num_point_lights, uint32_t seed, dipl_ray* d_out,
                                                 void* stream) {
    DIPL_CHECK_ARG(n >= 0 && width >= 1 && num_area_lights >= 0 && num_point_lights >= 0 && samples >= 0,
                   "n, lights and samples must be >= 0 and width >= 1");
    DIPL_CHECK_ARG(num_area_lights == 0 || samples >= 1, "area lights need samples >= 1");
    const int64_t per_hit = (int64_t)num_area_lights * samples + num_point_lights;
    DIPL_CHECK_ARG(per_hit <= (1 << 20), "at most 2^20 shadow rays per hit");
    if (n == 0 || per_hit == 0) return DIPL_OK;
    DIPL_CHECK_ARG(d_v0 && d_v1 && d_v2 && d_rays && d_hits && d_out, "arrays must be non-NULL");
    DIPL_CHECK_ARG(num_area_lights == 0 || d_area_light_triangles, "d_area_light_triangles must be non-NULL");
    DIPL_CHECK_ARG(num_point_lights == 0 || d_point_lights, "d_point_lights must be non-NULL");
    DIPL_CHECK_ARG((reinterpret_cast<uintptr_t>(d_rays) & 15) == 0 && (reinterpret_cast<uintptr_t>(d_hits) & 15) == 0 &&
                       (reinterpret_cast<uintptr_t>(d_out) & 15) == 0,
                   "rays, hits and output must be 16-byte aligned");
    DIPL_CHECK_ARG(d_out != d_rays, "d_out may not alias d_rays");
    const int64_t total = n * per_hit;
    shadow_kernel<<<(unsigned)((total + kGenThreads - 1) / kGenThreads), kGenThreads, 0,
                    static_cast<cudaStream_t>(stream)>>>(d_v0, d_v1, d_v2, d_rays, d_hits, n, width,
                                                         d_area_light_triangles, num_area_lights, samples,
                                                         d_point_lights, num_point_lights, seed, d_out);
    note_launches();
    DIPL_CUDA(cudaGetLastError());
    return DIPL_OK;
}
