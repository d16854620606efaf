// Closest-hit and any-hit traversal of the binary FP32 BVH: one thread per ray, near-child-first descent
// with a per-thread stack of (reference, entry t), conservative slab tests.
//
// Replaces SBvh::Intersect / IntersectAny (src/acceleration/sbvh.cc:60-191) and the device brute force
// DummyIntersect / DummyIntersectAny (src/gpu/renderer/gpu_renderer_util.h:29-94).
//
// Closest-hit rule: among triangles with tmin < t < tmax, the smallest t, ties to the lowest primitive id.
// That is exactly what the reference brute force returns (ascending ids, strict <,
// dummy_acceleration_structure.cc:21-64). To keep it under any traversal order the box tests are
// conservative: slab distances widen by 1e-6 relative (their own rounding, with the approximate reciprocal
// of the direction, stays below 5e-7), boxes are padded
// by 2^-20 of their coordinate magnitude at build time, and a node is pruned only when it starts beyond
// the best t by more than 1e-5 relative, so a node can never be skipped for rounding of its own box.
#include "internal.h"
#include "intersect.cuh"

namespace dipl {
namespace {

constexpr int kTraceThreads = 128;
// Resident blocks per SM the kernel is compiled for: 9 x 128 threads at <= 56 registers. Builds with more
// registers and 8 blocks per SM measured up to 1.5x slower on the 16M-triangle soup.
constexpr int kTraceMinBlocks = 9;
constexpr float kSlabWiden = 1e-6f;
constexpr float kPruneSlack = 1e-5f;

struct RayState {
    float3 o, d, inv;
    float tmin, tmax;
};

__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// One 32-byte read-only load (p must be 32-byte aligned): a 64-byte node in two loads instead of four.
__device__ __forceinline__ void ldg_v8(const void* p, float4& x, float4& y) {
    asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(x.x), "=f"(x.y), "=f"(x.z), "=f"(x.w), "=f"(y.x), "=f"(y.y), "=f"(y.z), "=f"(y.w)
        : "l"(p));
}

__device__ __forceinline__ RayState load_ray(const dipl_ray* rays, int64_t i) {
    const float4* r4 = reinterpret_cast<const float4*>(rays) + 2 * i;
    const float4 a = __ldg(r4), b = __ldg(r4 + 1);
    RayState r;
    r.o = make_float3(a.x, a.y, a.z);
    r.d = make_float3(b.x, b.y, b.z);
    r.tmin = a.w;
    r.tmax = b.w;
    // Directions below 1e-20 in magnitude are treated as +-1e-20 so that 1/d stays finite and a ray lying
    // on a slab plane is still inside it (0 * inf would be NaN). 1/d only feeds the slab tests, which widen
    // their interval by 1e-6 relative: the hardware reciprocal (relative error below 2^-22) is well inside
    // that margin.
    auto safe = [](float x) { return fabsf(x) < 1e-20f ? copysignf(1e-20f, x) : x; };
    r.inv = make_float3(rcp_approx(safe(r.d.x)), rcp_approx(safe(r.d.y)), rcp_approx(safe(r.d.z)));
    return r;
}

// Conservative ray/box interval; returns entry t (or +inf when the box is missed or out of range).
__device__ __forceinline__ float box_entry(const RayState& r, float lx, float hx, float ly, float hy, float lz, float hz,
                                           float t_limit) {
    const float tx0 = __fmul_rn(__fsub_rn(lx, r.o.x), r.inv.x), tx1 = __fmul_rn(__fsub_rn(hx, r.o.x), r.inv.x);
    const float ty0 = __fmul_rn(__fsub_rn(ly, r.o.y), r.inv.y), ty1 = __fmul_rn(__fsub_rn(hy, r.o.y), r.inv.y);
    const float tz0 = __fmul_rn(__fsub_rn(lz, r.o.z), r.inv.z), tz1 = __fmul_rn(__fsub_rn(hz, r.o.z), r.inv.z);
    float tn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fminf(tz0, tz1));
    float tf = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fmaxf(tz0, tz1));
    tn = tn - fabsf(tn) * kSlabWiden;
    tf = tf + fabsf(tf) * kSlabWiden;
    const bool hit = tn <= tf && tf >= r.tmin && tn <= t_limit;
    return hit ? tn : __int_as_float(0x7F800000);
}

__device__ __forceinline__ float prune_limit(float best_t) { return best_t + fabsf(best_t) * kPruneSlack; }

// Traversal stack of (node reference, entry t). Entries [0, SHORT) live in shared memory, one column per
// thread (entry k of thread j at sh[k * kTraceThreads + j], so a warp's accesses never share a bank), the rest
// in local memory.
template <int STACK, int SHORT>
struct Stack {
    int2* sh;
    int ref[STACK - SHORT];
    float t[STACK - SHORT];
    int sp = 0;
    __device__ __forceinline__ void push(int r, float tt) {
        if (sp < SHORT) {
            sh[sp * kTraceThreads] = make_int2(r, __float_as_int(tt));
        } else {
            ref[sp - SHORT] = r;
            t[sp - SHORT] = tt;
        }
        ++sp;
    }
    __device__ __forceinline__ int2 get(int k) const {
        return k < SHORT ? sh[k * kTraceThreads] : make_int2(ref[k - SHORT], __float_as_int(t[k - SHORT]));
    }
};

// Leaf test dispatch: ref_mt or watertight.
template <int LEAF>
__device__ __forceinline__ float leaf_test(float3 a, float3 b, float3 c, const RayState& r, const WtRay& w,
                                           bool backface, float& b1, float& b2) {
    if (LEAF == DIPL_LEAF_REF_MT) return mt_ref(a, b, c, r.o, r.d, backface, b1, b2);
    return wt_test(a, b, c, r.o, w, backface, b1, b2);
}

// Persistent traversal: each warp owns a contiguous chunk of rays and advances every lane by one node or
// one leaf per step; a lane whose ray finished takes the next ray of the chunk at the following step, so
// lanes do not idle behind the warp's longest ray (most rays of a batch may finish at the root while a few
// descend to the leaves).
template <int LEAF, bool ANY, bool COUNT, int STACK, int SHORT>
__global__ void __launch_bounds__(kTraceThreads, kTraceMinBlocks) trace_kernel(const BNode* __restrict__ nodes,
                                                              const float4* __restrict__ tris, int root,
                                                              int num_nodes, const dipl_ray* __restrict__ rays,
                                                              int64_t n, int64_t chunk, dipl_hit* __restrict__ hits,
                                                              uint8_t* __restrict__ occluded, uint32_t flags,
                                                              unsigned long long* __restrict__ counters,
                                                              uint32_t* __restrict__ err) {
    __shared__ int2 sh_stack[SHORT > 0 ? SHORT * kTraceThreads : 1];
    const int lane = threadIdx.x & 31;
    const int64_t warp_id = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t beg = warp_id * chunk;
    const int64_t end = min(n, beg + chunk);
    const bool backface = (flags & DIPL_TRACE_BACKFACE_CULLING) != 0u;
    const uint32_t lt_mask = lanemask_lt();
    const uint32_t step_limit = 2u * (uint32_t)max(num_nodes, 0) + 64u;
    int64_t next = beg;  // next ray of the chunk (warp-uniform)
    int64_t my = -1;     // this lane's ray, -1 when idle
    RayState r{};
    WtRay w{};
    float best_t = 0.0f, best_u = 0.0f, best_v = 0.0f;
    int best_prim = -1;
    bool found = false;
    int cur = 0;
    uint32_t steps = 0;
    Stack<STACK, SHORT> st;
    st.sh = sh_stack + threadIdx.x;
    unsigned visits = 0, tests = 0;
    bool bad = false;
    for (;;) {
        // ---- refill idle lanes from the chunk --------------------------------------------------------
        const bool idle = my < 0;
        const uint32_t idle_mask = __ballot_sync(0xffffffffu, idle);
        if (idle_mask) {
            if (idle) {
                const int64_t cand = next + __popc(idle_mask & lt_mask);
                if (cand < end) {
                    my = cand;
                    r = load_ray(rays, my);
                    if (LEAF == DIPL_LEAF_WATERTIGHT) w = wt_setup(r.d);
                    best_t = r.tmax, best_u = 0.0f, best_v = 0.0f, best_prim = -1, found = false;
                    cur = num_nodes >= 0 ? root : 0x7FFFFFFF;
                    st.sp = 0;
                    steps = 0;
                }
            }
            next = min(end, next + (int64_t)__popc(idle_mask));
        }
        if (__all_sync(0xffffffffu, my < 0)) break;
        if (my < 0) continue;

        // ---- one step: an inner node or a leaf --------------------------------------------------------
        bool finished = false;
        if (cur == 0x7FFFFFFF) {
            finished = true;  // empty BVH
        } else if (++steps > step_limit || (cur >= 0 && cur >= num_nodes)) {
            bad = true;       // only a corrupted tree gets here
            finished = true;
        } else if (cur >= 0) {
            const float4* np = reinterpret_cast<const float4*>(nodes + cur);
            float4 a, b, c, df;
            ldg_v8(np, a, b);
            ldg_v8(np + 2, c, df);
            const int2 d = make_int2(__float_as_int(df.x), __float_as_int(df.y));
            if (COUNT) ++visits;
            const float lim = prune_limit(best_t);
            const float t0 = box_entry(r, a.x, a.y, a.z, a.w, c.x, c.y, lim);
            const float t1 = box_entry(r, b.x, b.y, b.z, b.w, c.z, c.w, lim);
            const bool h0 = t0 != __int_as_float(0x7F800000), h1 = t1 != __int_as_float(0x7F800000);
            if (h0 && h1) {
                const bool first0 = t0 <= t1;
                if (st.sp >= STACK) {
                    bad = true;
                    finished = true;
                } else {
                    st.push(first0 ? d.y : d.x, first0 ? t1 : t0);
                    cur = first0 ? d.x : d.y;
                }
            } else if (h0) {
                cur = d.x;
            } else if (h1) {
                cur = d.y;
            } else {
                cur = -0x7FFFFFFF - 1;  // pop below
            }
        } else if (cur != -0x7FFFFFFF - 1) {
            const int first = leaf_first(cur), cnt = leaf_count(cur);
            for (int k = 0; k < cnt; ++k) {
                const float4* tp = tris + 3 * (int64_t)(first + k);
                const float4 p0 = __ldg(tp), p1 = __ldg(tp + 1), p2 = __ldg(tp + 2);
                const int prim = __float_as_int(p0.w);
                float b1 = 0.0f, b2 = 0.0f;
                const float t = leaf_test<LEAF>(make_float3(p0.x, p0.y, p0.z), make_float3(p1.x, p1.y, p1.z),
                                                make_float3(p2.x, p2.y, p2.z), r, w, backface, b1, b2);
                if (COUNT) ++tests;
                // t == kInfinity is the tests' miss value (also when tmax is +inf)
                if (ANY) {
                    if (t > r.tmin && t < r.tmax && t < kInfinity) {
                        found = true;
                        break;
                    }
                } else if (t > r.tmin && t < kInfinity &&
                           (t < best_t || (t == best_t && found && prim < best_prim))) {
                    best_t = t;
                    best_prim = prim;
                    best_u = b1;
                    best_v = b2;
                    found = true;
                }
            }
            if (ANY && found) finished = true;
            else cur = -0x7FFFFFFF - 1;  // pop below
        }
        if (!finished && cur == -0x7FFFFFFF - 1) {
            // pop the next entry that can still hold a better hit
            const float lim = prune_limit(best_t);
            cur = 0x7FFFFFFF;
            while (st.sp > 0) {
                --st.sp;
                const int2 e = st.get(st.sp);
                if (__int_as_float(e.y) <= lim) {
                    cur = e.x;
                    break;
                }
            }
            if (cur == 0x7FFFFFFF) finished = true;
        }
        if (finished) {
            if (ANY) {
                occluded[my] = found ? 1 : 0;
            } else {
                int4 out;
                out.x = found ? best_prim : -1;
                out.y = __float_as_int(found ? best_t : __int_as_float(0x7F800000));
                out.z = __float_as_int(found ? best_u : 0.0f);
                out.w = __float_as_int(found ? best_v : 0.0f);
                reinterpret_cast<int4*>(hits)[my] = out;
            }
            my = -1;
        }
    }
    if (bad) atomicOr(err, kErrStack);
    if (COUNT) {
        const unsigned v = __reduce_add_sync(0xffffffffu, visits);
        const unsigned t = __reduce_add_sync(0xffffffffu, tests);
        if (lane == 0) {
            atomicAdd(&counters[0], (unsigned long long)v);
            atomicAdd(&counters[1], (unsigned long long)t);
        }
    }
}

template <typename K>
int persistent_grid(K kernel) {
    static int grid = 0;  // per instantiation
    if (grid == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kTraceThreads, 0);
        grid = std::max(1, sms * std::max(1, per_sm));
    }
    return grid;
}

template <int LEAF, bool ANY, bool COUNT, int STACK, int SHORT>
dipl_status launch_trace(const dipl_bvh* b, const dipl_ray* rays, int64_t n, dipl_hit* hits, uint8_t* occ,
                         uint32_t flags, unsigned long long* counters, cudaStream_t s) {
    auto kernel = trace_kernel<LEAF, ANY, COUNT, STACK, SHORT>;
    const int max_grid = persistent_grid(kernel);
    const int64_t warps_needed = (n + 31) / 32;
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(max_grid, (warps_needed * 32 + kTraceThreads - 1) /
                                                                               kTraceThreads));
    const int64_t warps = grid * (kTraceThreads / 32);
    const int64_t chunk = (n + warps - 1) / warps;
    const int num_nodes = b->num_triangles == 0 ? -1 : (int)b->node_capacity;
    if ((reinterpret_cast<uintptr_t>(b->nodes) & 63) != 0) {
        set_last_error("trace: node array is not 64-byte aligned");
        return DIPL_ERR_INTERNAL;
    }
    kernel<<<(unsigned)grid, kTraceThreads, 0, s>>>(static_cast<const BNode*>(b->nodes), b->tris, b->root, num_nodes,
                                                   rays, n, chunk, hits, occ, flags, counters, b->d_err);
    note_launches();
    DIPL_CUDA(cudaGetLastError());
    return DIPL_OK;
}

template <int LEAF, bool ANY, bool COUNT>
dipl_status launch_trace_stack(const dipl_bvh* b, const dipl_ray* rays, int64_t n, dipl_hit* hits, uint8_t* occ,
                               uint32_t flags, unsigned long long* counters, cudaStream_t s) {
    // Deep trees keep the top 16 stack entries in shared memory (4-5% faster on the 1M-triangle sphere, whose
    // grazing rays push deep); shallower ones leave that memory to L1 for nodes (the 16M soup is ~1.5% slower
    // with it).
    if (b->depth < 64) return launch_trace<LEAF, ANY, COUNT, 64, 0>(b, rays, n, hits, occ, flags, counters, s);
    if (b->depth < 128) return launch_trace<LEAF, ANY, COUNT, 128, 16>(b, rays, n, hits, occ, flags, counters, s);
    return launch_trace<LEAF, ANY, COUNT, 512, 16>(b, rays, n, hits, occ, flags, counters, s);
}

}  // namespace

dipl_status trace_closest(const dipl_bvh* b, const dipl_ray* rays, int64_t n, dipl_hit* hits, int leaf_test,
                          uint32_t flags, unsigned long long* counters, cudaStream_t s) {
    DIPL_CHECK_ARG(b && n >= 0, "bvh must be non-NULL and n >= 0");
    DIPL_CHECK_ARG(n == 0 || (rays && hits), "rays/hits must be non-NULL");
    DIPL_CHECK_ARG(leaf_test == DIPL_LEAF_REF_MT || leaf_test == DIPL_LEAF_WATERTIGHT, "bad leaf_test");
    DIPL_CHECK_ARG((reinterpret_cast<uintptr_t>(rays) & 15) == 0 && (reinterpret_cast<uintptr_t>(hits) & 15) == 0,
                   "rays and hits must be 16-byte aligned");
    if (n == 0) return DIPL_OK;
    if (b->layout != DIPL_LAYOUT_BINARY || b->bv_type != DIPL_BV_AABB) return trace_closest_ext(b, rays, n, hits, leaf_test, flags, counters, s);
    const bool cnt = counters != nullptr;
    if (leaf_test == DIPL_LEAF_REF_MT)
        return cnt ? launch_trace_stack<DIPL_LEAF_REF_MT, false, true>(b, rays, n, hits, nullptr, flags, counters, s)
                   : launch_trace_stack<DIPL_LEAF_REF_MT, false, false>(b, rays, n, hits, nullptr, flags, nullptr, s);
    return cnt ? launch_trace_stack<DIPL_LEAF_WATERTIGHT, false, true>(b, rays, n, hits, nullptr, flags, counters, s)
               : launch_trace_stack<DIPL_LEAF_WATERTIGHT, false, false>(b, rays, n, hits, nullptr, flags, nullptr, s);
}

dipl_status trace_any(const dipl_bvh* b, const dipl_ray* rays, int64_t n, uint8_t* occ, int leaf_test, uint32_t flags,
                      cudaStream_t s) {
    DIPL_CHECK_ARG(b && n >= 0, "bvh must be non-NULL and n >= 0");
    DIPL_CHECK_ARG(n == 0 || (rays && occ), "rays/occluded must be non-NULL");
    DIPL_CHECK_ARG(leaf_test == DIPL_LEAF_REF_MT || leaf_test == DIPL_LEAF_WATERTIGHT, "bad leaf_test");
    DIPL_CHECK_ARG((reinterpret_cast<uintptr_t>(rays) & 15) == 0, "rays must be 16-byte aligned");
    if (n == 0) return DIPL_OK;
    if (b->layout != DIPL_LAYOUT_BINARY || b->bv_type != DIPL_BV_AABB) return trace_any_ext(b, rays, n, occ, leaf_test, flags, s);
    if (leaf_test == DIPL_LEAF_REF_MT)
        return launch_trace_stack<DIPL_LEAF_REF_MT, true, false>(b, rays, n, nullptr, occ, flags, nullptr, s);
    return launch_trace_stack<DIPL_LEAF_WATERTIGHT, true, false>(b, rays, n, nullptr, occ, flags, nullptr, s);
}

}  // namespace dipl
