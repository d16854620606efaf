// C ABI of libdipl_bvh (include/dipl_bvh.h): argument checks, status mapping, handle management.
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>
#include <string>
#include <unordered_map>

#include "internal.h"

namespace dipl {

static thread_local std::string g_last_error;
static std::atomic<unsigned long long> g_launches{0};

void note_launches(int n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }

void set_last_error(const std::string& msg) { g_last_error = msg; }

dipl_status cuda_status(cudaError_t e, const char* what) {
    std::string msg = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    set_last_error(msg);
    (void)cudaGetLastError();  // clear a sticky-free error so later calls are not misattributed
    return e == cudaErrorMemoryAllocation ? DIPL_ERR_OUT_OF_MEMORY : DIPL_ERR_CUDA;
}

// ---- process-wide limits (dipl_set_limits) -----------------------------------------------------------
static std::atomic<uint64_t> g_mem_limit{0};
static std::atomic<uint32_t> g_clustering_iterations{0};
static std::atomic<uint32_t> g_trace_steps{0};
static std::mutex g_mem_mu;
static uint64_t g_mem_in_use = 0;                    // bytes of live device allocations (under g_mem_mu)
static std::unordered_map<void*, size_t> g_mem_sizes;  // live allocation -> bytes (under g_mem_mu)

uint32_t clustering_iteration_limit() { return g_clustering_iterations.load(std::memory_order_relaxed); }
uint32_t trace_step_limit() { return g_trace_steps.load(std::memory_order_relaxed); }

static DeviceProbe g_pool_configured;  // per device: each device has its own default pool

dipl_status device_alloc(void** ptr, size_t bytes, cudaStream_t stream) {
    {
        std::lock_guard<std::mutex> lock(g_mem_mu);
        const uint64_t limit = g_mem_limit.load(std::memory_order_relaxed);
        if (limit != 0 && g_mem_in_use + bytes > limit) {
            *ptr = nullptr;
            set_last_error("device memory limit of " + std::to_string(limit) + " bytes reached (" +
                           std::to_string(g_mem_in_use) + " in use, " + std::to_string(bytes) + " requested)");
            return DIPL_ERR_OUT_OF_MEMORY;
        }
        g_mem_in_use += bytes;  // reserved before the allocation, so concurrent callers cannot both pass the cap
    }
    probe_per_device(g_pool_configured, [] {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) return 0;
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t threshold = ~0ull;  // keep freed blocks for reuse: builds allocate the same sizes repeatedly
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
        }
        (void)cudaGetLastError();
        return 1;
    });
    cudaError_t e = cudaMallocAsync(ptr, bytes, stream);
    std::lock_guard<std::mutex> lock(g_mem_mu);
    if (e != cudaSuccess) {
        g_mem_in_use -= bytes;
        *ptr = nullptr;
        return cuda_status(e, "cudaMallocAsync");
    }
    g_mem_sizes[*ptr] = bytes;
    return DIPL_OK;
}

void device_free(void* ptr, cudaStream_t stream) {
    if (!ptr) return;
    cudaFreeAsync(ptr, stream);
    std::lock_guard<std::mutex> lock(g_mem_mu);
    auto it = g_mem_sizes.find(ptr);
    if (it != g_mem_sizes.end()) {
        g_mem_in_use -= it->second;
        g_mem_sizes.erase(it);
    }
}

unsigned char* pinned_host_buffer(size_t bytes) {
    struct Buf {
        void* p = nullptr;
        size_t n = 0;
        ~Buf() {
            if (p) cudaFreeHost(p);
        }
    };
    static thread_local Buf buf;
    if (buf.n < bytes) {
        if (buf.p) cudaFreeHost(buf.p);
        buf.p = nullptr;
        buf.n = 0;
        size_t want = std::max<size_t>(bytes, 64 * 1024);
        if (cudaMallocHost(&buf.p, want) != cudaSuccess) {
            buf.p = nullptr;
            return nullptr;
        }
        buf.n = want;
    }
    return static_cast<unsigned char*>(buf.p);
}

dipl_status check_device_error(uint32_t* d_err, cudaStream_t stream, const char* where) {
    uint32_t h = 0;
    DIPL_CUDA(cudaMemcpyAsync(&h, d_err, 4, cudaMemcpyDeviceToHost, stream));
    DIPL_CUDA(cudaStreamSynchronize(stream));
    if (h == 0u) return DIPL_OK;
    DIPL_CUDA(cudaMemsetAsync(d_err, 0, 4, stream));
    std::string msg = std::string(where) + ": device error word 0x" + std::to_string(h);
    set_last_error(msg);
    if (h & kErrTimeout) return DIPL_ERR_TIMEOUT;
    return DIPL_ERR_INTERNAL;
}

dipl_status sah_cost(const dipl_bvh* b, double* cost, cudaStream_t stream) {
    (void)stream;
    if (b->num_triangles == 0) {
        *cost = 0.0;
        return DIPL_OK;
    }
    *cost = b->sah_area > 0.0 ? b->sah_sum / b->sah_area : 0.0;
    return DIPL_OK;
}

}  // namespace dipl

using namespace dipl;

extern "C" {

int32_t dipl_abi_version(void) { return DIPL_ABI_VERSION; }

dipl_status dipl_set_limits(const dipl_limits* limits) {
    if (!limits) {
        set_last_error("dipl_set_limits: limits must be non-NULL");
        return DIPL_ERR_INVALID_ARGUMENT;
    }
    g_mem_limit.store(limits->device_memory_bytes, std::memory_order_relaxed);
    g_clustering_iterations.store(limits->clustering_iterations, std::memory_order_relaxed);
    g_trace_steps.store(limits->trace_steps, std::memory_order_relaxed);
    return DIPL_OK;
}

dipl_status dipl_get_limits(dipl_limits* limits, uint64_t* device_memory_in_use) {
    if (limits) {
        limits->device_memory_bytes = g_mem_limit.load(std::memory_order_relaxed);
        limits->clustering_iterations = g_clustering_iterations.load(std::memory_order_relaxed);
        limits->trace_steps = g_trace_steps.load(std::memory_order_relaxed);
    }
    if (device_memory_in_use) {
        std::lock_guard<std::mutex> lock(g_mem_mu);
        *device_memory_in_use = g_mem_in_use;
    }
    return DIPL_OK;
}

uint64_t dipl_kernel_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

const char* dipl_last_error(void) { return g_last_error.c_str(); }

const char* dipl_status_string(dipl_status s) {
    switch (s) {
        case DIPL_OK: return "DIPL_OK";
        case DIPL_ERR_INVALID_ARGUMENT: return "DIPL_ERR_INVALID_ARGUMENT";
        case DIPL_ERR_CUDA: return "DIPL_ERR_CUDA";
        case DIPL_ERR_OUT_OF_MEMORY: return "DIPL_ERR_OUT_OF_MEMORY";
        case DIPL_ERR_TIMEOUT: return "DIPL_ERR_TIMEOUT";
        case DIPL_ERR_INTERNAL: return "DIPL_ERR_INTERNAL";
        case DIPL_ERR_UNSUPPORTED: return "DIPL_ERR_UNSUPPORTED";
        case DIPL_ERR_IO: return "DIPL_ERR_IO";
    }
    return "DIPL_ERR_UNKNOWN";
}

void dipl_build_desc_init(dipl_build_desc* d) {
    if (!d) return;
    std::memset(d, 0, sizeof(*d));
    d->code_type = DIPL_CODE_MORTON30;
    d->bv_type = DIPL_BV_AABB;
    d->layout = DIPL_LAYOUT_BINARY;
    d->max_triangles_per_leaf = 4;
    d->nn_search_radius = 16;
    d->kdop_size = 32;
    d->ploc_block_size = 0;
    d->sort_digit_bits = 0;
    d->clustering = DIPL_CLUSTER_HPLOC;
    d->split_budget = 0;
}

dipl_status dipl_bvh_build(const dipl_build_desc* desc, dipl_bvh** out, void* stream) {
    if (!desc || !out) {
        set_last_error("dipl_bvh_build: desc/out must be non-NULL");
        return DIPL_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    return build_batched(desc, 1, out, static_cast<cudaStream_t>(stream));
}

dipl_status dipl_bvh_build_batched(const dipl_build_desc* descs, int32_t count, dipl_bvh** out, void* stream) {
    return build_batched(descs, count, out, static_cast<cudaStream_t>(stream));
}

dipl_status dipl_build_plan_create(const dipl_build_desc* descs, int32_t count, dipl_build_plan** out, void* stream) {
    return plan_create(descs, count, out, static_cast<cudaStream_t>(stream));
}

dipl_status dipl_build_plan_launch(dipl_build_plan* plan, void* stream) {
    return plan_launch(plan, static_cast<cudaStream_t>(stream));
}

dipl_status dipl_build_plan_get_bvhs(dipl_build_plan* plan, dipl_bvh** out, void* stream) {
    return plan_get_bvhs(plan, out, static_cast<cudaStream_t>(stream));
}

dipl_status dipl_build_plan_destroy(dipl_build_plan* plan) {
    plan_destroy(plan);
    return DIPL_OK;
}

dipl_status dipl_bvh_trace_closest(const dipl_bvh* bvh, const dipl_ray* d_rays, int64_t n, dipl_hit* d_hits,
                                   int32_t leaf_test, uint32_t flags, void* stream) {
    return trace_closest(bvh, d_rays, n, d_hits, leaf_test, flags, nullptr, static_cast<cudaStream_t>(stream));
}

dipl_status dipl_bvh_trace_closest_counted(const dipl_bvh* bvh, const dipl_ray* d_rays, int64_t n, dipl_hit* d_hits,
                                           int32_t leaf_test, uint32_t flags, uint64_t* d_counters, void* stream) {
    if (!d_counters) {
        set_last_error("dipl_bvh_trace_closest_counted: counters must be non-NULL");
        return DIPL_ERR_INVALID_ARGUMENT;
    }
    return trace_closest(bvh, d_rays, n, d_hits, leaf_test, flags, reinterpret_cast<unsigned long long*>(d_counters),
                         static_cast<cudaStream_t>(stream));
}

dipl_status dipl_bvh_trace_any(const dipl_bvh* bvh, const dipl_ray* d_rays, int64_t n, uint8_t* d_occluded,
                               int32_t leaf_test, uint32_t flags, void* stream) {
    return trace_any(bvh, d_rays, n, d_occluded, leaf_test, flags, static_cast<cudaStream_t>(stream));
}

dipl_status dipl_bvh_sah_cost(const dipl_bvh* bvh, double* cost, void* stream) {
    if (!bvh || !cost) {
        set_last_error("dipl_bvh_sah_cost: bvh/cost must be non-NULL");
        return DIPL_ERR_INVALID_ARGUMENT;
    }
    return sah_cost(bvh, cost, static_cast<cudaStream_t>(stream));
}

dipl_status dipl_bvh_get_info(const dipl_bvh* b, dipl_bvh_info* info) {
    if (!b || !info) {
        set_last_error("dipl_bvh_get_info: bvh/info must be non-NULL");
        return DIPL_ERR_INVALID_ARGUMENT;
    }
    std::memset(info, 0, sizeof(*info));
    info->num_triangles = b->num_triangles;
    info->num_inner_nodes = b->num_nodes;
    info->num_leaves = b->num_refs;
    info->node_bytes = b->num_nodes * b->node_size;
    info->triangle_bytes = b->num_refs * 48;
    info->depth = b->depth;
    info->ploc_iterations = b->ploc_iterations;
    info->code_type = b->code_type;
    info->bv_type = b->bv_type;
    info->layout = b->layout;
    info->max_triangles_per_leaf = b->max_leaf;
    info->nn_search_radius = b->radius;
    info->kdop_size = b->kdop;
    info->clustering = b->clustering;
    return DIPL_OK;
}

dipl_status dipl_bvh_download_topology(const dipl_bvh* b, int32_t* h_perm, int32_t* h_children, float* h_boxes,
                                       void* stream) {
    if (!b) {
        set_last_error("dipl_bvh_download_topology: bvh must be non-NULL");
        return DIPL_ERR_INVALID_ARGUMENT;
    }
    if (b->batched) {
        set_last_error("dipl_bvh_download_topology: handles of a batched build share one topology");
        return DIPL_ERR_UNSUPPORTED;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t n = b->num_refs, k = n > 0 ? n - 1 : 0;
    std::vector<int32_t> ref_tri;
    if (h_perm && n > 0) {
        DIPL_CUDA(cudaMemcpyAsync(h_perm, b->perm, 4 * n, cudaMemcpyDeviceToHost, s));
        if (b->ref_tri) {  // positions hold references: report their triangles
            ref_tri.resize(n);
            DIPL_CUDA(cudaMemcpyAsync(ref_tri.data(), b->ref_tri, 4 * n, cudaMemcpyDeviceToHost, s));
        }
    }
    std::vector<int4> ch(k);
    std::vector<float4> lo(k), hi(k);
    if (k > 0) {
        DIPL_CUDA(cudaMemcpyAsync(ch.data(), b->children, sizeof(int4) * k, cudaMemcpyDeviceToHost, s));
        DIPL_CUDA(cudaMemcpyAsync(lo.data(), b->node_lo, sizeof(float4) * k, cudaMemcpyDeviceToHost, s));
        DIPL_CUDA(cudaMemcpyAsync(hi.data(), b->node_hi, sizeof(float4) * k, cudaMemcpyDeviceToHost, s));
    }
    DIPL_CUDA(cudaStreamSynchronize(s));
    if (!ref_tri.empty())
        for (int64_t i = 0; i < n; ++i) h_perm[i] = ref_tri[h_perm[i]];
    for (int64_t i = 0; i < k; ++i) {
        if (h_children) {
            h_children[2 * i] = ch[i].x;
            h_children[2 * i + 1] = ch[i].y;
        }
        if (h_boxes) {
            float* bx = h_boxes + 6 * i;
            bx[0] = lo[i].x, bx[1] = lo[i].y, bx[2] = lo[i].z;
            bx[3] = hi[i].x, bx[4] = hi[i].y, bx[5] = hi[i].z;
        }
    }
    return DIPL_OK;
}

dipl_status dipl_bvh_download_layout(const dipl_bvh* b, void* h_nodes, void* h_triangles, int32_t* h_root,
                                     void* stream) {
    if (!b) {
        set_last_error("dipl_bvh_download_layout: bvh must be non-NULL");
        return DIPL_ERR_INVALID_ARGUMENT;
    }
    if (b->batched) {
        set_last_error("dipl_bvh_download_layout: handles of a batched build share one layout");
        return DIPL_ERR_UNSUPPORTED;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (h_nodes && b->num_nodes > 0)
        DIPL_CUDA(cudaMemcpyAsync(h_nodes, b->nodes, b->num_nodes * b->node_size, cudaMemcpyDeviceToHost, s));
    if (h_triangles && b->num_refs > 0)
        DIPL_CUDA(cudaMemcpyAsync(h_triangles, b->tris, b->num_refs * 48, cudaMemcpyDeviceToHost, s));
    DIPL_CUDA(cudaStreamSynchronize(s));
    if (h_root) *h_root = b->root;
    return DIPL_OK;
}

dipl_status dipl_bvh_check_errors(const dipl_bvh* b, void* stream) {
    if (!b) {
        set_last_error("dipl_bvh_check_errors: bvh must be non-NULL");
        return DIPL_ERR_INVALID_ARGUMENT;
    }
    return check_device_error(b->d_err, static_cast<cudaStream_t>(stream), "trace");
}

dipl_status dipl_bvh_destroy(dipl_bvh* b) {
    delete b;  // device memory goes back to the pool in stream order when the last handle of a build dies
    return DIPL_OK;
}

dipl_status dipl_compute_codes(const dipl_build_desc* desc, void* d_codes, void* stream) {
    return compute_codes(desc, d_codes, static_cast<cudaStream_t>(stream));
}

dipl_status dipl_radix_sort_pairs(const void* d_keys_in, const uint32_t* d_vals_in, void* d_keys_out,
                                  uint32_t* d_vals_out, int64_t n, int32_t key_bytes, int32_t begin_bit,
                                  int32_t end_bit, int32_t digit_bits, void* stream) {
    if (n < 0 || n >= (1ll << 30) || (key_bytes != 4 && key_bytes != 8) || begin_bit < 0 || end_bit <= begin_bit ||
        end_bit > 8 * key_bytes || !radix_sort_bits_ok(begin_bit, end_bit, digit_bits)) {
        set_last_error("dipl_radix_sort_pairs: bad size, key width, bit range or digit width");
        return DIPL_ERR_INVALID_ARGUMENT;
    }
    if (n == 0) return DIPL_OK;
    if (!d_keys_in || !d_keys_out || !d_vals_out) {
        set_last_error("dipl_radix_sort_pairs: key/value arrays must be non-NULL");
        return DIPL_ERR_INVALID_ARGUMENT;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ScratchArena scratch(s);
    unsigned char *kalt, *sc;
    uint32_t *valt, *err;
    dipl_status st;
    if ((st = scratch.alloc(&kalt, n * key_bytes)) != DIPL_OK || (st = scratch.alloc(&valt, n)) != DIPL_OK ||
        (st = scratch.alloc(&sc, radix_sort_scratch_bytes(n, begin_bit, end_bit, digit_bits))) != DIPL_OK ||
        (st = scratch.alloc(&err, 1)) != DIPL_OK)
        return st;
    DIPL_CUDA(cudaMemsetAsync(err, 0, 4, s));
    st = radix_sort_pairs(d_keys_in, d_vals_in, d_keys_out, d_vals_out, kalt, valt, n, key_bytes, begin_bit, end_bit,
                          digit_bits, sc, s, err);
    if (st != DIPL_OK) return st;
    return check_device_error(err, s, "dipl_radix_sort_pairs");
}

dipl_status dipl_reintersect_f64(const float* d_v0, const float* d_v1, const float* d_v2, const dipl_ray* d_rays,
                                 const dipl_hit* d_hits, int64_t n, double* d_tuv, void* stream) {
    return reintersect_f64(d_v0, d_v1, d_v2, d_rays, d_hits, n, d_tuv, static_cast<cudaStream_t>(stream));
}

dipl_status dipl_trace_adjoint(const float* d_v0, const float* d_v1, const float* d_v2, const dipl_ray* d_rays,
                               const dipl_hit* d_hits, const float* d_dtuv, int64_t n, float* d_dv0, float* d_dv1,
                               float* d_dv2, float* d_dorig, float* d_ddir, void* stream) {
    return trace_adjoint(d_v0, d_v1, d_v2, d_rays, d_hits, d_dtuv, n, d_dv0, d_dv1, d_dv2, d_dorig, d_ddir,
                         static_cast<cudaStream_t>(stream));
}

}  // extern "C"
