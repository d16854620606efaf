// TEST INFRASTRUCTURE — CHECKER ONLY. Never linked into, or called by, the product library.
//
// C ABI around the reference's OWN acceleration structures, compiled from the reference
// sources where they lie (see oracle/Makefile). Used by the parity tests, the golden-vector
// generator and bench.py's CPU-baseline / reference arm.
//
//   SBvh::Build / Intersect           src/acceleration/sbvh.cc:17-145   (CPU binned-SAH BVH)
//   DummyAccelerationStucture::Intersect src/acceleration/dummy_acceleration_structure.cc:21-64
//                                      (brute force, ascending id, strict <: lowest-id ties)
//   Triangle::IntersectRay            src/scene/triangle.cc:10-43       (Moller-Trumbore, eps 1e-6)
//
// Input layout: triangles as float[N][3][3] (v0, v1, v2; xyz), rays as float[R][8]
// (origin xyz, tmin, dir xyz, tmax). The reference Ray has no tmin (it always uses kEpsilon),
// so tmin is ignored here; tmax becomes Ray::t_max.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <span>
#include <stack>
#include <thread>
#include <vector>

#include "util/logger.h"
#define private public  // read SBvh::nodes_ for the SAH cost and bounds checks (layout: sbvh.h:25-36)
#include "acceleration/sbvh.h"
#undef private
#include "acceleration/dummy_acceleration_structure.h"
#include "config/acceleration_structure_config.h"
#include "scene/ray.h"
#include "scene/ray_hit.h"
#include "scene/triangle.h"
#include "stats/stats.h"

using namespace diplodocus;

namespace {

std::vector<Triangle> MakeTriangles(const float* tris, int64_t n) {
    std::vector<Triangle> out(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) {
        const float* p = tris + 9 * i;
        Triangle& t = out[i];
        t.v0.pos = Vec3(p[0], p[1], p[2]);
        t.v1.pos = Vec3(p[3], p[4], p[5]);
        t.v2.pos = Vec3(p[6], p[7], p[8]);
        t.v0.normal = t.v1.normal = t.v2.normal = Vec3(0.0f);
        RecomputeTriangleGeometricNormal(t);
        t.material_id = 0;
        t.has_vertex_normals = false;
    }
    return out;
}

inline Ray MakeRay(const float* r) { return Ray{Vec3(r[0], r[1], r[2]), Vec3(r[4], r[5], r[6]), r[7]}; }

struct SbvhHandle {
    std::vector<Triangle> triangles;
    SBvh bvh;
    AccelerationStructureConfig cfg;
};

template <class F>
void ParallelFor(int64_t n, int nthreads, F&& f) {
    if (nthreads <= 1 || n < 2 * nthreads) {
        f(0, n, 0);
        return;
    }
    std::vector<std::thread> th;
    int64_t chunk = (n + nthreads - 1) / nthreads;
    for (int k = 0; k < nthreads; ++k) {
        int64_t b = k * chunk, e = std::min(n, b + chunk);
        if (b >= e) break;
        th.emplace_back([&, b, e, k] { f(b, e, k); });
    }
    for (auto& t : th) t.join();
}

template <class AS>
void TraceWith(const AS& as, const float* rays, int64_t nrays, int32_t* prim, float* t, float* u, float* v,
               int backface, int nthreads, int64_t* counters) {
    std::vector<Stats> per(static_cast<size_t>(std::max(1, nthreads)));
    ParallelFor(nrays, nthreads, [&](int64_t b, int64_t e, int k) {
        Stats& st = per[k];
        for (int64_t i = b; i < e; ++i) {
            Ray ray = MakeRay(rays + 8 * i);
            RayHit hit;
            if (as.Intersect(st, ray, hit, backface != 0)) {
                prim[i] = hit.triangle_id;
                t[i] = hit.t;
                u[i] = hit.b1;
                v[i] = hit.b2;
            } else {
                prim[i] = -1;
                t[i] = INFINITY;
                u[i] = 0.0f;
                v[i] = 0.0f;
            }
        }
    });
    if (counters) {
        // int counters of the reference (acceleration_stats.h:14-16) summed per thread chunk
        int64_t q = 0, tr = 0, is = 0;
        for (auto& s : per) {
            q += s.accel_stats.query_count;
            tr += s.accel_stats.traversal_count;
            is += s.accel_stats.intersection_count;
        }
        counters[0] = q;
        counters[1] = tr;
        counters[2] = is;
    }
}

double SurfaceArea(const Vec3& lo, const Vec3& hi) {
    double dx = double(hi.x) - lo.x, dy = double(hi.y) - lo.y, dz = double(hi.z) - lo.z;
    return 2.0 * (dx * dy + dy * dz + dz * dx);
}

}  // namespace

extern "C" {

void* ref_sbvh_build(const float* tris, int64_t n, int max_depth, int max_triangles_per_leaf, int bin_count,
                     double* build_ms) {
    if (n <= 0) return nullptr;  // the reference underflows 2n-1 at n = 0 (sbvh.cc:24)
    Logger::init(Logger::LogLevel::Error);
    auto h = std::make_unique<SbvhHandle>();
    h->triangles = MakeTriangles(tris, n);
    h->cfg.acceleration_structure_type = AccelerationStructureType::kSbvh;
    h->cfg.max_depth = max_depth;
    h->cfg.max_triangles_per_leaf = max_triangles_per_leaf;
    h->cfg.bin_count = bin_count;
    Stats st;
    auto t0 = std::chrono::steady_clock::now();
    h->bvh.Build(h->cfg, st, std::span<const Triangle>(h->triangles));
    auto t1 = std::chrono::steady_clock::now();
    if (build_ms) *build_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    return h.release();
}

// Re-run SBvh::Build on an existing handle (same triangles), for timing repeated builds.
double ref_sbvh_rebuild(void* handle) {
    auto* h = static_cast<SbvhHandle*>(handle);
    Stats st;
    auto t0 = std::chrono::steady_clock::now();
    h->bvh.Build(h->cfg, st, std::span<const Triangle>(h->triangles));
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

void ref_sbvh_destroy(void* handle) { delete static_cast<SbvhHandle*>(handle); }

void ref_sbvh_trace(void* handle, const float* rays, int64_t nrays, int32_t* prim, float* t, float* u, float* v,
                    int backface, int nthreads, int64_t* counters) {
    auto* h = static_cast<SbvhHandle*>(handle);
    TraceWith(h->bvh, rays, nrays, prim, t, u, v, backface, nthreads, counters);
}

// SAH cost C = [sum_inner SA(n) + sum_leaf SA(n)*|n|] / SA(root), C_t = C_i = 1, FP64,
// over the reachable SBvh nodes (nodes_[0] is the root; children at t_begin, t_begin+1).
double ref_sbvh_sah_cost(void* handle, int64_t* inner_nodes, int64_t* leaf_nodes) {
    auto* h = static_cast<SbvhHandle*>(handle);
    const auto& nodes = h->bvh.nodes_;
    double root_sa = SurfaceArea(nodes[0].aabb_min, nodes[0].aabb_max);
    double acc = 0.0;
    int64_t ni = 0, nl = 0;
    std::vector<size_t> st{0};
    while (!st.empty()) {
        size_t k = st.back();
        st.pop_back();
        const auto& nd = nodes[k];
        double sa = SurfaceArea(nd.aabb_min, nd.aabb_max);
        if (nd.t_count > 0) {
            acc += sa * nd.t_count;
            ++nl;
        } else {
            acc += sa;
            ++ni;
            st.push_back(nd.t_begin);
            st.push_back(nd.t_begin + 1);
        }
    }
    if (inner_nodes) *inner_nodes = ni;
    if (leaf_nodes) *leaf_nodes = nl;
    return root_sa > 0.0 ? acc / root_sa : 0.0;
}

// Brute-force closest hit: the reference's DummyAccelerationStucture (lowest-id tie rule).
void ref_brute_trace(const float* tris, int64_t n, const float* rays, int64_t nrays, int32_t* prim, float* t,
                     float* u, float* v, int backface, int nthreads) {
    Logger::init(Logger::LogLevel::Error);
    std::vector<Triangle> tv = MakeTriangles(tris, n);
    DummyAccelerationStucture dummy;
    AccelerationStructureConfig cfg;
    Stats st;
    dummy.Build(cfg, st, std::span<const Triangle>(tv));
    TraceWith(dummy, rays, nrays, prim, t, u, v, backface, nthreads, nullptr);
}

// One reference Moller-Trumbore test (triangle.cc:10-43), returning t (kInfinity on a miss).
float ref_intersect_one(const float* tri9, const float* ray8, int backface, float* b1, float* b2) {
    std::vector<Triangle> tv = MakeTriangles(tri9, 1);
    Ray r = MakeRay(ray8);
    return tv[0].IntersectRay(r, *b1, *b2, backface != 0);
}

}  // extern "C"
