// TEST INFRASTRUCTURE — CHECKER ONLY. Drives the reference-side adapter (diplodocus_b200/adapter/gpu_ploc_bvh.h),
// compiled against the reference's own headers (oracle/Makefile, target adapter), the way the reference's renderer
// would: Triangles made as its Scene makes them, a GpuPlocBvh from the factory's PLOC case, Build, then per-ray
// Intersect / IntersectAny and the batch paths.
//
//   adapter_check <type> <tris.bin> <rays.bin> <out.bin> <per_ray_count>
//     type: ploc | ploc_emc | ploc_sobb | ploc_emc_sobb
//     tris.bin: float32 [N][3][3]; rays.bin: float32 [R][8] (origin, tmin, dir, tmax; tmin is the reference's
//     kEpsilon and is not read)
//     out.bin: int32 K (= min(R, per_ray_count)), then R batch records and K per-ray records (int32 prim, float t,
//     b1, b2; prim -1 on a miss), then R batch and K per-ray occlusion bytes; then the Stats counters
//     (int32 query_count, inner_node_count)
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <vector>

#include "gpu_ploc_bvh.h"

using namespace diplodocus;

namespace {

std::vector<float> ReadFloats(const char* path) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) throw std::runtime_error(std::string("cannot read ") + path);
    const std::streamsize bytes = f.tellg();
    f.seekg(0);
    std::vector<float> v(static_cast<size_t>(bytes) / sizeof(float));
    f.read(reinterpret_cast<char*>(v.data()), bytes);
    return v;
}

// The factory lines the integration adds to CreateAccelerationStucture (acceleration_structure_factory.cc:9-19).
std::unique_ptr<AccelerationStructure> CreatePloc(const AccelerationStructureConfig& cfg) {
    switch (cfg.acceleration_structure_type) {
        case AccelerationStructureType::kPloc:
        case AccelerationStructureType::kPlocEmc:
        case AccelerationStructureType::kPlocSobb:
        case AccelerationStructureType::kPlocEmcSobb:
            return std::make_unique<GpuPlocBvh>();
        default:
            throw std::invalid_argument("Unkown AccelerationStructureType");
    }
}

struct Rec {
    int32_t prim;
    float t, b1, b2;
};

}  // namespace

int main(int argc, char** argv) {
    if (argc != 6) {
        std::fprintf(stderr, "usage: %s <type> <tris.bin> <rays.bin> <out.bin> <per_ray_count>\n", argv[0]);
        return 2;
    }
    try {
        AccelerationStructureConfig cfg;
        cfg.acceleration_structure_type = ParseEnum<AccelerationStructureType>(argv[1]);
        cfg.nn_search_radius = 16;
        const std::vector<float> tv = ReadFloats(argv[2]);
        const std::vector<float> rv = ReadFloats(argv[3]);
        const size_t n = tv.size() / 9, nr = rv.size() / 8;
        std::vector<Triangle> tris(n);
        for (size_t i = 0; i < n; ++i) {
            const float* p = tv.data() + 9 * i;
            tris[i].v0.pos = Vec3(p[0], p[1], p[2]);
            tris[i].v1.pos = Vec3(p[3], p[4], p[5]);
            tris[i].v2.pos = Vec3(p[6], p[7], p[8]);
            tris[i].v0.normal = tris[i].v1.normal = tris[i].v2.normal = Vec3(0.0f);
            tris[i].material_id = 0;
            tris[i].has_vertex_normals = false;
            RecomputeTriangleGeometricNormal(tris[i]);
        }
        std::vector<Ray> rays(nr);
        for (size_t i = 0; i < nr; ++i) {
            const float* r = rv.data() + 8 * i;
            rays[i] = Ray{Vec3(r[0], r[1], r[2]), Vec3(r[4], r[5], r[6]), r[7]};
        }
        Stats stats;
        std::unique_ptr<AccelerationStructure> as = CreatePloc(cfg);
        as->Build(cfg, stats, std::span<const Triangle>(tris));
        auto* bvh = static_cast<GpuPlocBvh*>(as.get());
        const size_t k = std::min<size_t>(nr, static_cast<size_t>(std::atoi(argv[5])));
        std::vector<RayHit> batch(nr);
        std::unique_ptr<bool[]> hit(new bool[nr]), occ(new bool[nr]);
        bvh->IntersectHost(stats, std::span<const Ray>(rays), std::span<RayHit>(batch), std::span<bool>(hit.get(), nr),
                           false);
        bvh->IntersectAnyHost(stats, std::span<const Ray>(rays), std::span<bool>(occ.get(), nr), false);
        std::vector<Rec> out_batch(nr), out_one(k);
        std::vector<uint8_t> occ_batch(nr), occ_one(k);
        for (size_t i = 0; i < nr; ++i) {
            out_batch[i] = hit[i] ? Rec{batch[i].triangle_id, batch[i].t, batch[i].b1, batch[i].b2}
                                  : Rec{-1, INFINITY, 0.0f, 0.0f};
            occ_batch[i] = occ[i] ? 1 : 0;
        }
        for (size_t i = 0; i < k; ++i) {  // the CPU renderer's per-ray calls through the base interface
            RayHit h;
            out_one[i] = as->Intersect(stats, rays[i], h, false) ? Rec{h.triangle_id, h.t, h.b1, h.b2}
                                                                 : Rec{-1, INFINITY, 0.0f, 0.0f};
            occ_one[i] = as->IntersectAny(stats, rays[i], false) ? 1 : 0;
        }
        std::ofstream f(argv[4], std::ios::binary);
        const int32_t kk = static_cast<int32_t>(k);
        f.write(reinterpret_cast<const char*>(&kk), 4);
        f.write(reinterpret_cast<const char*>(out_batch.data()), sizeof(Rec) * nr);
        f.write(reinterpret_cast<const char*>(out_one.data()), sizeof(Rec) * k);
        f.write(reinterpret_cast<const char*>(occ_batch.data()), nr);
        f.write(reinterpret_cast<const char*>(occ_one.data()), k);
        const int32_t counters[2] = {stats.accel_stats.query_count, stats.accel_stats.inner_node_count};
        f.write(reinterpret_cast<const char*>(counters), sizeof counters);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "adapter_check: %s\n", e.what());
        return 1;
    }
    return 0;
}
