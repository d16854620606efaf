// Internal (non-ABI) declarations shared by the engine's translation units.
#pragma once

#include <algorithm>
#include <memory>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace dipl {

// ---- launch-shape probes -----------------------------------------------------------------------
// A launch-shape probe answered once per device: the answer depends on the device's limits (SMs, shared memory,
// schedulable cluster sizes), so each device gets its own, computed under a lock so that concurrent builds on
// other host threads never see a half-made answer.
constexpr int kMaxProbeDevices = 64;
struct DeviceProbe {
    std::mutex mu;
    bool done[kMaxProbeDevices] = {};
    int value[kMaxProbeDevices] = {};
};

template <class F>
int probe_per_device(DeviceProbe& p, F&& probe) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxProbeDevices) {
        (void)cudaGetLastError();
        return probe();  // no cache slot: answer without caching
    }
    std::lock_guard<std::mutex> lock(p.mu);
    if (!p.done[dev]) {
        p.value[dev] = probe();
        p.done[dev] = true;
    }
    return p.value[dev];
}

// ---- sort ----------------------------------------------------------------------------------------
size_t radix_sort_scratch_bytes(int64_t n, int begin_bit, int end_bit, int digit_bits);
bool radix_sort_bits_ok(int begin_bit, int end_bit, int digit_bits);
dipl_status radix_sort_pairs(const void* kin, const uint32_t* vin, void* kout, uint32_t* vout, void* kalt,
                             uint32_t* valt, int64_t n, int key_bytes, int begin_bit, int end_bit, int digit_bits,
                             void* scratch, cudaStream_t stream, uint32_t* d_err);

// ---- scan ----------------------------------------------------------------------------------------
size_t scan_scratch_bytes(int64_t n);
// Exclusive prefix sum of n uint32 values (in and out may alias); optional total written to d_total.
dipl_status exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* d_total, void* scratch,
                               cudaStream_t stream, uint32_t* d_err);

// ---- device memory -------------------------------------------------------------------------------
// Stream-ordered allocation from the device's default pool (kept warm: release threshold raised once).
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
};
dipl_status device_alloc(void** ptr, size_t bytes, cudaStream_t stream);
void device_free(void* ptr, cudaStream_t stream);

// Process-wide limits set by dipl_set_limits (0 = the built-in bound).
uint32_t clustering_iteration_limit();
uint32_t trace_step_limit();

// Scope guard for scratch allocations of one call.
class ScratchArena {
   public:
    explicit ScratchArena(cudaStream_t s) : stream_(s) {}
    ~ScratchArena() {
        for (void* p : ptrs_) device_free(p, stream_);
    }
    template <typename T>
    dipl_status alloc(T** out, size_t count) {
        void* p = nullptr;
        dipl_status st = device_alloc(&p, std::max<size_t>(count * sizeof(T), 16), stream_);
        if (st != DIPL_OK) return st;
        ptrs_.push_back(p);
        *out = static_cast<T*>(p);
        return DIPL_OK;
    }

   private:
    cudaStream_t stream_;
    std::vector<void*> ptrs_;
};

// ---- the BVH handle ------------------------------------------------------------------------------
// Device memory of one build; shared by the handles of a batched build.
struct Storage {
    std::vector<void*> ptrs;
    cudaStream_t stream = nullptr;
    ~Storage() {
        for (void* p : ptrs) device_free(p, stream);
    }
    template <typename T>
    dipl_status alloc(T** out, size_t count) {
        void* p = nullptr;
        dipl_status st = device_alloc(&p, std::max<size_t>(count * sizeof(T), 16), stream);
        if (st != DIPL_OK) return st;
        ptrs.push_back(p);
        *out = static_cast<T*>(p);
        return DIPL_OK;
    }
};

}  // namespace dipl

struct dipl_bvh {
    std::shared_ptr<dipl::Storage> storage;
    int64_t num_triangles = 0;
    int64_t num_nodes = 0;      // nodes of the traced layout that belong to this mesh
    int64_t node_capacity = 0;  // nodes in the (possibly shared) node array: bound of every node index
    int64_t num_leaves = 0;
    int32_t root = 0;           // root reference (node index or leaf reference)
    int32_t depth = 0;
    int32_t ploc_iterations = 0;
    int32_t code_type = 0, bv_type = 0, layout = 0, max_leaf = 4, radius = 16, kdop = 32, clustering = 0;
    // traced arrays (device)
    void* nodes = nullptr;      // BNode / SNode / WNode
    int64_t node_size = 64;     // bytes per node of the traced layout
    float4* tris = nullptr;     // 3 float4 per triangle in leaf order (v0.w = primitive id bits)
    // clustering result (device), for downloads
    int32_t* perm = nullptr;    // triangle id per sorted position (of this mesh, local ids)
    int4* children = nullptr;   // internal node k: left/right node ids (global ids of the batch), height
    float4* node_lo = nullptr;  // internal node k: lo xyz, count (int bits)
    float4* node_hi = nullptr;  // internal node k: hi xyz, first sorted position (int bits)
    int64_t leaf_base = 0;      // first leaf id of this mesh in the batch numbering
    int64_t inner_base = 0;     // first internal node index of this mesh
    int64_t batch_leaves = 0;   // leaves of the whole batch (internal node id = batch_leaves + k)
    int64_t num_refs = 0;       // clustering leaves of this mesh: its triangles, or triangles and pieces
    bool batched = false;       // one of several meshes built together (they share the arrays)
    const int* ref_tri = nullptr;  // per leaf of the batch: its triangle (global index); NULL without pre-splitting
    double sah_area = 0.0;      // surface area of the root box
    double sah_sum = 0.0;       // sum over inner SA + leaf SA * count (FP64, device-summed)
    // device error word shared by the build and later traces
    uint32_t* d_err = nullptr;
};

namespace dipl {

// ---- build / trace entry points used by api.cu ---------------------------------------------------
dipl_status build_batched(const dipl_build_desc* descs, int count, dipl_bvh** out, cudaStream_t stream);
dipl_status plan_create(const dipl_build_desc* descs, int count, dipl_build_plan** out, cudaStream_t stream);
dipl_status plan_launch(dipl_build_plan* plan, cudaStream_t stream);
dipl_status plan_get_bvhs(dipl_build_plan* plan, dipl_bvh** out, cudaStream_t stream);
void plan_destroy(dipl_build_plan* plan);
dipl_status compute_codes(const dipl_build_desc* desc, void* d_codes, cudaStream_t stream);
dipl_status trace_closest(const dipl_bvh* bvh, const dipl_ray* rays, int64_t n, dipl_hit* hits, int leaf_test,
                          uint32_t flags, unsigned long long* counters, cudaStream_t stream);
dipl_status trace_any(const dipl_bvh* bvh, const dipl_ray* rays, int64_t n, uint8_t* occluded, int leaf_test,
                      uint32_t flags, cudaStream_t stream);
dipl_status sah_cost(const dipl_bvh* bvh, double* cost, cudaStream_t stream);
// Coherent ray order of large traces (trace.cu): with DIPL_TRACE_COHERENT_ORDER, batches of kReorderMinRays rays
// or more are traced in the order of a key of the origin cell and the direction octant, sorted on the device;
// records still go to each ray's index.
constexpr int64_t kReorderMinRays = int64_t(1) << 20;
inline bool reorder_rays(int64_t n, uint32_t flags) {
    return n >= kReorderMinRays && (flags & DIPL_TRACE_COHERENT_ORDER) != 0u;
}
// Device memory of one reordered trace: keys, the order and the sort's scratch (released in stream order).
struct RayOrder {
    void* mem = nullptr;
    uint32_t* order = nullptr;  // the ray index to trace at each position of the work order
};
dipl_status make_ray_order(const dipl_ray* rays, int64_t n, uint32_t* d_err, cudaStream_t s, RayOrder& ro);

// Traversal of the SOBB and 8-wide quantised layouts.
dipl_status trace_closest_ext(const dipl_bvh* bvh, const dipl_ray* rays, int64_t n, dipl_hit* hits, int leaf_test,
                              uint32_t flags, unsigned long long* counters, cudaStream_t stream);
dipl_status trace_any_ext(const dipl_bvh* bvh, const dipl_ray* rays, int64_t n, uint8_t* occluded, int leaf_test,
                          uint32_t flags, cudaStream_t stream);
dipl_status reintersect_f64(const float* v0, const float* v1, const float* v2, const dipl_ray* rays,
                            const dipl_hit* hits, int64_t n, double* tuv, cudaStream_t stream);
dipl_status trace_adjoint(const float* v0, const float* v1, const float* v2, const dipl_ray* rays,
                          const dipl_hit* hits, const float* dtuv, int64_t n, float* dv0, float* dv1, float* dv2,
                          float* dorig, float* ddir, cudaStream_t stream);

// Precision form (wide.cu): 8-wide quantised layout built from the binary clustering, and its traversal.
dipl_status build_wide(const int4* child, const float4* node_lo, const float4* node_hi, const int* leaf_start_of,
                       const float4* btris, int N, int L, const std::vector<int>& root_ids,
                       const std::vector<int>& root_counts, Storage& storage, cudaStream_t s, uint32_t* d_err,
                       WNode** out_nodes, float4** out_tris, int64_t* out_num_nodes, std::vector<int>& out_root_refs,
                       std::vector<int>& out_levels);
dipl_status trace_wide(const dipl_bvh* b, const dipl_ray* rays, int64_t n, dipl_hit* hits, uint8_t* occ, int leaf_test,
                       uint32_t flags, unsigned long long* counters, bool any, cudaStream_t s);

// SOBB form (sobb.cu): skewed oriented child boxes refitted over the binary layout, and their traversal.
struct SobbScratch {
    void* kdop = nullptr;  // k-DOP per node id
    float* mag = nullptr;  // coordinate magnitude per node id
    unsigned* arrivals = nullptr;
    int triples = 0;
};
// Pre-split builds: per slot of the leaf triangle array its sorted position, the sorted order of the references
// and every reference's box (all NULL without pre-splitting).
struct SobbRefs {
    const int* slot_pos = nullptr;
    const uint32_t* perm = nullptr;
    const float4* rbox = nullptr;
};
dipl_status sobb_prepare(long long N, long long K, Storage& work, Storage& out, SobbScratch* sc, SNode** snodes);
dipl_status sobb_enqueue(const int4* child, const float4* node_lo, const float4* node_hi, const int* parent,
                         const int* leaf_start_of, const int* owner_leaf, const float4* btris, const BNode* bnodes,
                         const uint32_t* rev_index, int N, int K, int L, int kdop_size, const SobbScratch& sc,
                         const SobbRefs& refs, SNode* snodes, cudaStream_t s, uint32_t* d_err);
dipl_status trace_sobb(const dipl_bvh* b, const dipl_ray* rays, int64_t n, dipl_hit* hits, uint8_t* occ, int leaf_test,
                       uint32_t flags, unsigned long long* counters, bool any, cudaStream_t s);

// Process-wide count of kernels this library has launched (for launch-count reporting).
void note_launches(int n = 1);

// Grow-only pinned host staging buffer of the calling thread.
unsigned char* pinned_host_buffer(size_t bytes);

// Reads and clears a device error word (synchronises the stream) and maps it to a status.
dipl_status check_device_error(uint32_t* d_err, cudaStream_t stream, const char* where);

}  // namespace dipl
