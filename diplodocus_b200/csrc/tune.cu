// Autotuner of the build knobs: clustering (hierarchical or global PLOC), PLOC radius, PLOC block size (global PLOC
// only: the hierarchical clustering's block is fixed) and sort digit width.
//
// For a batch (its total triangle count gives a size bucket, floor(log2 N)), it times real builds of the
// caller's meshes and keeps the fastest setting whose SAH cost stays within 2% of the default radius-16
// tree (the radius trades build time for tree quality; hits are exact with any valid tree, so only time and
// quality are compared). Coordinate search: digit width, then the other clustering (under the same SAH rule: one
// launch over hundreds of meshes can favour the global loop), then block size, then radius, each with the others
// fixed at the best so far. Winners are cached per (code, bounding volume, layout, leaf size, requested clustering,
// bucket) as one JSON object per line in a file, so a bucket is tuned once.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>

#include "internal.h"

namespace dipl {
namespace {

struct Tuned {
    int radius, block, digits;
    double ms, sah;
    int clustering;
};

std::string bucket_key(const dipl_build_desc& d, long long total) {
    int bucket = 0;
    while ((1ll << (bucket + 1)) <= total) ++bucket;
    std::ostringstream os;
    os << (d.code_type == DIPL_CODE_EMC60 ? "emc60" : "morton30") << "/" << (d.bv_type == DIPL_BV_SOBB ? "sobb" : "aabb")
       << "/" << (d.layout == DIPL_LAYOUT_WIDE8_Q8 ? "wide8" : "binary") << "/L" << d.max_triangles_per_leaf << "/"
       << (d.clustering == DIPL_CLUSTER_PLOC ? "ploc" : "hploc") << "/b" << bucket;
    return os.str();
}

bool cache_lookup(const char* path, const std::string& key, Tuned* t) {
    if (!path) return false;
    std::ifstream f(path);
    std::string line;
    bool found = false;
    while (std::getline(f, line)) {
        const std::string pat = "\"key\": \"" + key + "\"";
        if (line.find(pat) == std::string::npos) continue;
        Tuned x{};
        auto num = [&](const char* name, double* v) {
            const std::string k = std::string("\"") + name + "\": ";
            size_t p = line.find(k);
            if (p == std::string::npos) return false;
            *v = std::strtod(line.c_str() + p + k.size(), nullptr);
            return true;
        };
        double r, b, dg, ms, sah, cl;
        if (num("radius", &r) && num("block", &b) && num("digits", &dg) && num("ms", &ms) && num("sah", &sah)) {
            x.radius = (int)r, x.block = (int)b, x.digits = (int)dg, x.ms = ms, x.sah = sah;
            x.clustering = num("clustering", &cl) ? (int)cl : -1;  // entries without it keep the requested one
            *t = x;  // the last entry of a key wins
            found = true;
        }
    }
    return found;
}

void cache_store(const char* path, const std::string& key, const Tuned& t) {
    if (!path) return;
    std::ofstream f(path, std::ios::app);
    f << "{\"key\": \"" << key << "\", \"radius\": " << t.radius << ", \"block\": " << t.block
      << ", \"digits\": " << t.digits << ", \"ms\": " << t.ms << ", \"sah\": " << t.sah
      << ", \"clustering\": " << t.clustering << "}\n";
}

// Mean wall time of `reps` builds (after one warm-up) and the triangle-weighted SAH cost.
dipl_status time_builds(const std::vector<dipl_build_desc>& descs, int reps, cudaStream_t s, double* ms, double* sah) {
    std::vector<dipl_bvh*> out(descs.size(), nullptr);
    double best = 1e300;
    for (int r = 0; r <= reps; ++r) {
        auto t0 = std::chrono::steady_clock::now();
        dipl_status st = build_batched(descs.data(), (int)descs.size(), out.data(), s);
        auto t1 = std::chrono::steady_clock::now();
        if (st != DIPL_OK) return st;
        if (r > 0) best = std::min(best, std::chrono::duration<double, std::milli>(t1 - t0).count());
        if (r == reps) {
            double acc = 0.0, w = 0.0;
            for (auto* h : out) {
                double c = 0.0;
                sah_cost(h, &c, s);
                acc += c * (double)h->num_triangles;
                w += (double)h->num_triangles;
            }
            *sah = w > 0 ? acc / w : 0.0;
        }
        for (auto*& h : out) {
            delete h;
            h = nullptr;
        }
    }
    *ms = best;
    return DIPL_OK;
}

}  // namespace

dipl_status autotune(const dipl_build_desc* descs, int count, const char* cache_path, dipl_build_desc* tuned,
                     int* from_cache, cudaStream_t s) {
    DIPL_CHECK_ARG(descs && tuned && count >= 1, "descs/tuned must be non-NULL and count >= 1");
    long long total = 0;
    for (int i = 0; i < count; ++i) total += descs[i].num_triangles;
    const std::string key = bucket_key(descs[0], total);
    Tuned best{};
    bool cached = cache_lookup(cache_path, key, &best);
    if (from_cache) *from_cache = cached ? 1 : 0;
    if (!cached) {
        std::vector<dipl_build_desc> v(descs, descs + count);
        auto apply = [&](int clustering, int radius, int block, int digits) {
            for (auto& d : v)
                d.clustering = clustering, d.nn_search_radius = radius, d.ploc_block_size = block,
                d.sort_digit_bits = digits;
        };
        double ms = 0, sah = 0;
        const int requested = descs[0].clustering;
        apply(requested, 16, 256, 8);
        dipl_status st = time_builds(v, 2, s, &ms, &sah);
        if (st != DIPL_OK) return st;
        best = Tuned{16, 256, 8, ms, sah, requested};
        const double sah_limit = sah * 1.02;
        for (int digits : {6, 10}) {
            apply(best.clustering, best.radius, best.block, digits);
            if ((st = time_builds(v, 2, s, &ms, &sah)) != DIPL_OK) return st;
            if (ms < best.ms) best.digits = digits, best.ms = ms, best.sah = sah;
        }
        {
            const int other = requested == DIPL_CLUSTER_PLOC ? DIPL_CLUSTER_HPLOC : DIPL_CLUSTER_PLOC;
            apply(other, best.radius, best.block, best.digits);
            if ((st = time_builds(v, 2, s, &ms, &sah)) != DIPL_OK) return st;
            if (ms < best.ms && sah <= sah_limit) best.clustering = other, best.ms = ms, best.sah = sah;
        }
        for (int block : {128, 512}) {
            if (best.clustering != DIPL_CLUSTER_PLOC) break;  // the hierarchical clustering has one block size
            apply(best.clustering, best.radius, block, best.digits);
            if ((st = time_builds(v, 2, s, &ms, &sah)) != DIPL_OK) return st;
            if (ms < best.ms) best.block = block, best.ms = ms, best.sah = sah;
        }
        for (int radius : {8, 12, 24, 32}) {
            apply(best.clustering, radius, best.block, best.digits);
            if ((st = time_builds(v, 2, s, &ms, &sah)) != DIPL_OK) return st;
            if (ms < best.ms && sah <= sah_limit) best.radius = radius, best.ms = ms, best.sah = sah;
        }
        cache_store(cache_path, key, best);
    }
    for (int i = 0; i < count; ++i) {
        tuned[i] = descs[i];
        if (best.clustering >= 0) tuned[i].clustering = best.clustering;
        tuned[i].nn_search_radius = best.radius;
        tuned[i].ploc_block_size = best.block;
        tuned[i].sort_digit_bits = best.digits;
    }
    return DIPL_OK;
}

}  // namespace dipl

extern "C" dipl_status dipl_autotune_build(const dipl_build_desc* descs, int32_t count, const char* cache_path,
                                           dipl_build_desc* tuned, int32_t* from_cache, void* stream) {
    int fc = 0;
    dipl_status st = dipl::autotune(descs, count, cache_path, tuned, &fc, static_cast<cudaStream_t>(stream));
    if (from_cache) *from_cache = fc;
    return st;
}
