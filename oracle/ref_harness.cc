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
//   ObjSceneLoader::Load              src/io/scene/obj_scene_loader.cc:20-205 (OBJ + MTL through the vendored
//                                      tinyobjloader, .meta camera and point lights) -> flat arrays
//   ConsoleStatsExporter::ExportOne   src/io/stats/console_stats_exporter.cc:10-58 (its text on stdout)
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
#include "config/scene_load_config.h"
#include "io/scene/obj_scene_loader.h"
#include "io/stats/console_stats_exporter.h"
#include "scene/scene.h"
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

// The same brute force over large scenes, with the triangles cut into consecutive chunks of `chunk` triangles so
// that one chunk stays in the host's cache while a thread's rays run over it. For each chunk, in ascending order,
// the reference's DummyAccelerationStucture::Intersect runs over the chunk with the ray's t_max lowered to the best
// t found so far. Its loop starts from t_hit = ray.t_max and keeps t > kEpsilon && t < t_hit
// (dummy_acceleration_structure.cc:24-41), so the chunked pass makes exactly the comparisons of one pass over all
// triangles: the same id, t, b1 and b2, exact-t ties kept by the lowest id. Only the loop order differs.
void ref_brute_trace_chunked(const float* tris, int64_t n, const float* rays, int64_t nrays, int32_t* prim, float* t,
                             float* u, float* v, int backface, int nthreads, int64_t chunk) {
    Logger::init(Logger::LogLevel::Error);
    if (chunk <= 0) chunk = 8192;
    std::vector<Triangle> tv = MakeTriangles(tris, n);
    const int64_t nchunks = (n + chunk - 1) / chunk;
    std::vector<DummyAccelerationStucture> parts(static_cast<size_t>(nchunks));
    AccelerationStructureConfig cfg;
    Stats st;
    for (int64_t c = 0; c < nchunks; ++c) {
        const int64_t b = c * chunk, len = std::min(chunk, n - b);
        parts[c].Build(cfg, st, std::span<const Triangle>(tv.data() + b, static_cast<size_t>(len)));
    }
    ParallelFor(nrays, nthreads, [&](int64_t b, int64_t e, int) {
        Stats s;
        std::vector<Ray> rs;
        rs.reserve(static_cast<size_t>(e - b));
        for (int64_t i = b; i < e; ++i) {
            rs.push_back(MakeRay(rays + 8 * i));
            prim[i] = -1;
            t[i] = INFINITY;
            u[i] = 0.0f;
            v[i] = 0.0f;
        }
        for (int64_t c = 0; c < nchunks; ++c) {
            for (int64_t i = b; i < e; ++i) {
                Ray& ray = rs[static_cast<size_t>(i - b)];
                RayHit hit;
                if (parts[c].Intersect(s, ray, hit, backface != 0)) {
                    prim[i] = static_cast<int32_t>(c * chunk + hit.triangle_id);
                    t[i] = hit.t;
                    u[i] = hit.b1;
                    v[i] = hit.b2;
                    ray.t_max = hit.t;  // the next chunk starts from the best t so far
                }
            }
        }
    });
}

// One reference Moller-Trumbore test (triangle.cc:10-43), returning t (kInfinity on a miss).
float ref_intersect_one(const float* tri9, const float* ray8, int backface, float* b1, float* b2) {
    std::vector<Triangle> tv = MakeTriangles(tri9, 1);
    Ray r = MakeRay(ray8);
    return tv[0].IntersectRay(r, *b1, *b2, backface != 0);
}

// ---- scene loading: the reference ObjSceneLoader, its Scene exported as flat arrays -----------------------
struct RefScene {
    Scene scene;
};

// NULL when the reference loader fails (missing or malformed .meta / .obj), like its std::nullopt.
void* ref_obj_scene_load(const char* dirpath, const char* name) {
    Logger::init(Logger::LogLevel::Error);
    SceneLoadConfig cfg;
    cfg.dirpath = dirpath;
    cfg.name = name;
    std::optional<Scene> sc = ObjSceneLoader().Load(cfg);
    if (!sc) return nullptr;
    auto* h = new RefScene{std::move(*sc)};
    return h;
}

void ref_obj_scene_free(void* h) { delete static_cast<RefScene*>(h); }

// counts: triangles, materials, area lights, point lights
void ref_obj_scene_counts(void* h, int64_t* counts) {
    const Scene& s = static_cast<RefScene*>(h)->scene;
    counts[0] = (int64_t)s.Triangles().size();
    counts[1] = (int64_t)s.Materials().size();
    counts[2] = (int64_t)s.AreaLights().size();
    counts[3] = (int64_t)s.PointLights().size();
}

// pos / normals: 9 floats per triangle (v0, v1, v2); geom: 3 floats
void ref_obj_scene_triangles(void* h, float* pos, float* normals, float* geom, int32_t* material_ids,
                             uint8_t* has_normals) {
    const Scene& s = static_cast<RefScene*>(h)->scene;
    size_t i = 0;
    for (const Triangle& t : s.Triangles()) {
        const Vertex* vs[3] = {&t.v0, &t.v1, &t.v2};
        for (int k = 0; k < 3; ++k) {
            pos[9 * i + 3 * k + 0] = vs[k]->pos.x;
            pos[9 * i + 3 * k + 1] = vs[k]->pos.y;
            pos[9 * i + 3 * k + 2] = vs[k]->pos.z;
            normals[9 * i + 3 * k + 0] = t.has_vertex_normals ? vs[k]->normal.x : 0.0f;
            normals[9 * i + 3 * k + 1] = t.has_vertex_normals ? vs[k]->normal.y : 0.0f;
            normals[9 * i + 3 * k + 2] = t.has_vertex_normals ? vs[k]->normal.z : 0.0f;
        }
        geom[3 * i + 0] = t.geom_normal.x;
        geom[3 * i + 1] = t.geom_normal.y;
        geom[3 * i + 2] = t.geom_normal.z;
        material_ids[i] = t.material_id;
        has_normals[i] = t.has_vertex_normals ? 1 : 0;
        ++i;
    }
}

// values: 19 floats per material (ambient, diffuse, specular, transmittance, emission, shininess, ior, r_ior,
// dissolve); names: 64 bytes per material, NUL-terminated (truncated)
void ref_obj_scene_materials(void* h, float* values, char* names) {
    const Scene& s = static_cast<RefScene*>(h)->scene;
    size_t i = 0;
    for (const Material& m : s.Materials()) {
        const Vec3* v3[5] = {&m.ambient, &m.diffuse, &m.specular, &m.transmittance, &m.emission};
        for (int k = 0; k < 5; ++k) {
            values[19 * i + 3 * k + 0] = v3[k]->x;
            values[19 * i + 3 * k + 1] = v3[k]->y;
            values[19 * i + 3 * k + 2] = v3[k]->z;
        }
        values[19 * i + 15] = m.shininess;
        values[19 * i + 16] = m.ior;
        values[19 * i + 17] = m.r_ior;
        values[19 * i + 18] = m.dissolve;
        std::memset(names + 64 * i, 0, 64);
        std::strncpy(names + 64 * i, m.name.c_str(), 63);
        ++i;
    }
}

// the reference leaves AreaLight::power unset: only id, colour and area are exported
void ref_obj_scene_area_lights(void* h, int32_t* triangle_ids, float* colors, float* areas) {
    const Scene& s = static_cast<RefScene*>(h)->scene;
    size_t i = 0;
    for (const AreaLight& a : s.AreaLights()) {
        triangle_ids[i] = a.triangle_id;
        colors[3 * i + 0] = a.color.x;
        colors[3 * i + 1] = a.color.y;
        colors[3 * i + 2] = a.color.z;
        areas[i] = a.surface_area;
        ++i;
    }
}

// cam: pos, dir, up, fov, far (11 floats); lights: pos, color, power (7 floats each)
void ref_obj_scene_camera_lights(void* h, float* cam, float* lights) {
    const Scene& s = static_cast<RefScene*>(h)->scene;
    const Camera& c = s.GetCamera();
    const float cv[11] = {c.pos.x, c.pos.y, c.pos.z, c.dir.x, c.dir.y, c.dir.z, c.up.x, c.up.y, c.up.z, c.fov, c.far};
    std::memcpy(cam, cv, sizeof(cv));
    size_t i = 0;
    for (const PointLight& p : s.PointLights()) {
        const float pv[7] = {p.pos.x, p.pos.y, p.pos.z, p.color.x, p.color.y, p.color.z, p.power};
        std::memcpy(lights + 7 * i, pv, sizeof(pv));
        ++i;
    }
}

// The reference's console statistics text for the given values (written to stdout; the caller captures it).
// rt: raytracing_time, primary, secondary, shadow; accel: build_time, node, inner, leaf, memory, query,
// intersection, traversal (the reference stores the counts as int).
void ref_console_stats(const double* rt, const double* accel) {
    Stats s;
    s.rt_stats.raytracing_time = rt[0];
    s.rt_stats.primary_ray_count = (int)rt[1];
    s.rt_stats.secondary_ray_count = (int)rt[2];
    s.rt_stats.shadow_ray_count = (int)rt[3];
    s.accel_stats.build_time = accel[0];
    s.accel_stats.node_count = (int)accel[1];
    s.accel_stats.inner_node_count = (int)accel[2];
    s.accel_stats.leaf_node_count = (int)accel[3];
    s.accel_stats.memory_consumption = (int)accel[4];
    s.accel_stats.query_count = (int)accel[5];
    s.accel_stats.intersection_count = (int)accel[6];
    s.accel_stats.traversal_count = (int)accel[7];
    ConsoleStatsExporter().ExportOne(StatsExportConfig{}, s);
    std::cout.flush();
}

}  // extern "C"
