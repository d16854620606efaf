// GpuPlocBvh: the reference-side adapter of libdipl_bvh, written against Diplodocus's own headers (C++20).
//
// Drop-in for the reference: add this file as src/gpu/acceleration/gpu_ploc_bvh.h (the directory the reference
// reserves for GPU acceleration structures, src/gpu/acceleration/.gitkeep), link libdipl_bvh, and create it for the
// PLOC types in CreateAccelerationStucture (src/acceleration/acceleration_structure_factory.cc:9-19):
//
//     case AccelerationStructureType::kPloc:
//     case AccelerationStructureType::kPlocEmc:
//     case AccelerationStructureType::kPlocSobb:
//     case AccelerationStructureType::kPlocEmcSobb:
//         return std::make_unique<GpuPlocBvh>();
//
// It implements AccelerationStructure (src/acceleration/acceleration_structure.h:12-19) with SBvh's conventions:
// Build keeps a non-owning span of the triangles (sbvh.h:33), so the Scene must outlive the structure; Intersect
// fills the RayHit as SBvh::Intersect does (sbvh.cc:127-143); the leaf test is the reference-exact one. Intersect and
// IntersectAny trace one ray per call, the CPU renderer's pattern (cpu_raytracer.cc:111-112, 236); IntersectHost and
// IntersectBatch trace whole batches (one launch) for callers that have them. Errors throw std::runtime_error with
// dipl_last_error(), where the reference's CUDA path aborts (CUDA_CHECK, src/gpu/cuda_utils.h:12-18).
#pragma once

#include <cuda_runtime.h>

#include <chrono>
#include <span>
#include <stdexcept>
#include <string>
#include <vector>

#include "acceleration/acceleration_structure.h"
#include "config/acceleration_structure_config.h"
#include "dipl_bvh.h"
#include "scene/ray.h"
#include "scene/ray_hit.h"
#include "scene/triangle.h"
#include "stats/stats.h"

namespace diplodocus {

class GpuPlocBvh : public AccelerationStructure {
   public:
    GpuPlocBvh() = default;
    GpuPlocBvh(const GpuPlocBvh&) = delete;
    GpuPlocBvh& operator=(const GpuPlocBvh&) = delete;
    ~GpuPlocBvh() override { Release(); }

    void Build(const AccelerationStructureConfig& cfg, Stats& stats, std::span<const Triangle> triangles) override {
        const auto t0 = std::chrono::steady_clock::now();
        Release();
        triangles_ = triangles;
        const size_t n = triangles.size();
        std::vector<float> v[3];
        for (auto& a : v) a.resize(3 * n);
        for (size_t i = 0; i < n; ++i) {
            const Vec3* p[3] = {&triangles[i].v0.pos, &triangles[i].v1.pos, &triangles[i].v2.pos};
            for (int k = 0; k < 3; ++k) v[k][3 * i] = p[k]->x, v[k][3 * i + 1] = p[k]->y, v[k][3 * i + 2] = p[k]->z;
        }
        for (int k = 0; k < 3; ++k) {
            Cuda(cudaMalloc(&d_v_[k], sizeof(float) * 3 * (n ? n : 1)), "cudaMalloc");
            Cuda(cudaMemcpy(d_v_[k], v[k].data(), sizeof(float) * 3 * n, cudaMemcpyHostToDevice), "cudaMemcpy");
        }
        dipl_build_desc d;
        dipl_build_desc_init(&d);
        d.d_v0 = d_v_[0], d.d_v1 = d_v_[1], d.d_v2 = d_v_[2];
        d.num_triangles = static_cast<int64_t>(n);
        // BridgeAccelerationConfig (src/gpu/config/gpu_config_bridge.cc:24-60): code and bounding volume by type
        const auto t = cfg.acceleration_structure_type;
        if (t != AccelerationStructureType::kPloc && t != AccelerationStructureType::kPlocEmc &&
            t != AccelerationStructureType::kPlocSobb && t != AccelerationStructureType::kPlocEmcSobb)
            throw std::invalid_argument("GpuPlocBvh builds the PLOC acceleration structure types only");
        d.code_type = (t == AccelerationStructureType::kPlocEmc || t == AccelerationStructureType::kPlocEmcSobb)
                          ? DIPL_CODE_EMC60
                          : DIPL_CODE_MORTON30;
        d.bv_type = (t == AccelerationStructureType::kPlocSobb || t == AccelerationStructureType::kPlocEmcSobb)
                        ? DIPL_BV_SOBB
                        : DIPL_BV_AABB;
        d.max_triangles_per_leaf = cfg.max_triangles_per_leaf;
        d.nn_search_radius = cfg.nn_search_radius;
        d.kdop_size = cfg.kdop_size;
        Status(dipl_bvh_build(&d, &bvh_, nullptr), "dipl_bvh_build");
        dipl_bvh_info info;
        Status(dipl_bvh_get_info(bvh_, &info), "dipl_bvh_get_info");
        stats.accel_stats.inner_node_count = static_cast<int>(info.num_inner_nodes);
        stats.accel_stats.node_count = static_cast<int>(2 * info.num_inner_nodes + 1);
        stats.accel_stats.leaf_node_count = static_cast<int>(info.num_inner_nodes + 1);
        stats.accel_stats.memory_consumption = static_cast<int>(info.node_bytes + info.triangle_bytes);
        stats.accel_stats.build_time =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }

    bool Intersect(Stats& stats, const Ray& ray, RayHit& ray_hit, bool backface_culling) const override {
        bool hit = false;
        IntersectHost(stats, std::span<const Ray>(&ray, 1), std::span<RayHit>(&ray_hit, 1), std::span<bool>(&hit, 1),
                      backface_culling);
        return hit;
    }

    bool IntersectAny(Stats& stats, const Ray& ray, bool backface_culling) const override {
        bool occ = false;
        IntersectAnyHost(stats, std::span<const Ray>(&ray, 1), std::span<bool>(&occ, 1), backface_culling);
        return occ;
    }

    // A batch of host rays: one upload, one launch, one download. hit[i] tells whether ray_hits[i] was filled.
    void IntersectHost(Stats& stats, std::span<const Ray> rays, std::span<RayHit> ray_hits, std::span<bool> hit,
                       bool backface_culling) const {
        const size_t n = rays.size();
        stats.accel_stats.query_count += static_cast<int>(n);
        if (n == 0) return;
        std::vector<dipl_ray> r(n);
        for (size_t i = 0; i < n; ++i) r[i] = ToDipl(rays[i]);
        std::vector<dipl_hit> h(n);
        Reserve(n);
        Cuda(cudaMemcpy(d_rays_, r.data(), sizeof(dipl_ray) * n, cudaMemcpyHostToDevice), "cudaMemcpy");
        Status(dipl_bvh_trace_closest(bvh_, d_rays_, static_cast<int64_t>(n), d_hits_, DIPL_LEAF_REF_MT,
                                      backface_culling ? DIPL_TRACE_BACKFACE_CULLING : 0u, nullptr),
               "dipl_bvh_trace_closest");
        Cuda(cudaMemcpy(h.data(), d_hits_, sizeof(dipl_hit) * n, cudaMemcpyDeviceToHost), "cudaMemcpy");
        Status(dipl_bvh_check_errors(bvh_, nullptr), "dipl_bvh_check_errors");
        for (size_t i = 0; i < n; ++i) {
            hit[i] = h[i].prim >= 0;
            if (hit[i]) Fill(rays[i], h[i], ray_hits[i]);
        }
    }

    void IntersectAnyHost(Stats& stats, std::span<const Ray> rays, std::span<bool> occluded,
                          bool backface_culling) const {
        const size_t n = rays.size();
        stats.accel_stats.query_count += static_cast<int>(n);
        if (n == 0) return;
        std::vector<dipl_ray> r(n);
        for (size_t i = 0; i < n; ++i) r[i] = ToDipl(rays[i]);
        std::vector<uint8_t> o(n);
        Reserve(n);
        Cuda(cudaMemcpy(d_rays_, r.data(), sizeof(dipl_ray) * n, cudaMemcpyHostToDevice), "cudaMemcpy");
        Status(dipl_bvh_trace_any(bvh_, d_rays_, static_cast<int64_t>(n), d_occ_, DIPL_LEAF_REF_MT,
                                  backface_culling ? DIPL_TRACE_BACKFACE_CULLING : 0u, nullptr),
               "dipl_bvh_trace_any");
        Cuda(cudaMemcpy(o.data(), d_occ_, n, cudaMemcpyDeviceToHost), "cudaMemcpy");
        for (size_t i = 0; i < n; ++i) occluded[i] = o[i] != 0;
    }

    // The GPU frontend's batch: device rays in, device hit records out, asynchronously on `stream`.
    void IntersectBatch(const dipl_ray* d_rays, int64_t n, dipl_hit* d_hits, cudaStream_t stream) const {
        Status(dipl_bvh_trace_closest(bvh_, d_rays, n, d_hits, DIPL_LEAF_REF_MT, 0u, stream), "dipl_bvh_trace_closest");
    }

    const dipl_bvh* Handle() const { return bvh_; }

   private:
    // Ray (src/scene/ray.h:7-11) has no tmin: the reference always uses kEpsilon (sbvh.cc:85).
    static dipl_ray ToDipl(const Ray& r) {
        return dipl_ray{r.origin.x, r.origin.y, r.origin.z, kEpsilon, r.dir.x, r.dir.y, r.dir.z, r.t_max};
    }

    // The hit record of SBvh::Intersect (sbvh.cc:127-143) from the engine's (prim, t, b1, b2).
    void Fill(const Ray& ray, const dipl_hit& h, RayHit& out) const {
        const Triangle& tri = triangles_[static_cast<size_t>(h.prim)];
        out.t = h.t;
        out.triangle_id = h.prim;
        out.material_id = tri.material_id;
        out.pos = ray.At(h.t);
        out.b0 = 1.0f - h.u - h.v;
        out.b1 = h.u;
        out.b2 = h.v;
        out.epsilon = RayEpsilon(out.pos, out.t);
        out.geom_normal = tri.geom_normal;
        out.normal = tri.geom_normal;
        if (tri.has_vertex_normals)
            out.normal = Normalize(tri.v0.normal * out.b0 + tri.v1.normal * out.b1 + tri.v2.normal * out.b2);
    }

    void Reserve(size_t n) const {
        if (n <= capacity_) return;
        cudaFree(d_rays_), cudaFree(d_hits_), cudaFree(d_occ_);
        d_rays_ = nullptr, d_hits_ = nullptr, d_occ_ = nullptr, capacity_ = 0;
        Cuda(cudaMalloc(&d_rays_, sizeof(dipl_ray) * n), "cudaMalloc");
        Cuda(cudaMalloc(&d_hits_, sizeof(dipl_hit) * n), "cudaMalloc");
        Cuda(cudaMalloc(&d_occ_, n), "cudaMalloc");
        capacity_ = n;
    }

    static void Cuda(cudaError_t e, const char* what) {
        if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
    }
    static void Status(dipl_status s, const char* what) {
        if (s != DIPL_OK) throw std::runtime_error(std::string(what) + ": " + dipl_last_error());
    }

    void Release() {
        if (bvh_) dipl_bvh_destroy(bvh_);
        bvh_ = nullptr;
        for (auto*& p : d_v_) cudaFree(p), p = nullptr;
        cudaFree(d_rays_), cudaFree(d_hits_), cudaFree(d_occ_);
        d_rays_ = nullptr, d_hits_ = nullptr, d_occ_ = nullptr, capacity_ = 0;
    }

    std::span<const Triangle> triangles_;
    dipl_bvh* bvh_ = nullptr;
    float* d_v_[3] = {nullptr, nullptr, nullptr};
    mutable dipl_ray* d_rays_ = nullptr;
    mutable dipl_hit* d_hits_ = nullptr;
    mutable uint8_t* d_occ_ = nullptr;
    mutable size_t capacity_ = 0;
};

}  // namespace diplodocus
