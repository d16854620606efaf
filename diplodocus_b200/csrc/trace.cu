// Closest-hit and any-hit traversal of the binary FP32 BVH: one thread per ray, near-child-first descent
// with a per-thread stack of (reference, entry t), conservative slab tests.
//
// Replaces SBvh::Intersect / IntersectAny (src/acceleration/sbvh.cc:60-191) and the device brute force
// DummyIntersect / DummyIntersectAny (src/gpu/renderer/gpu_renderer_util.h:29-94).
//
// Closest-hit rule: among triangles with tmin < t < tmax, the smallest t, ties to the lowest primitive id.
// That is exactly what the reference brute force returns (ascending ids, strict <,
// dummy_acceleration_structure.cc:21-64). To keep it under any traversal order the box tests are
// conservative: slab distances widen by 1e-6 relative (their own rounding is below 2e-7), boxes are padded
// by 2^-20 of their coordinate magnitude at build time, and a node is pruned only when it starts beyond
// the best t by more than 1e-5 relative, so a node can never be skipped for rounding of its own box.
#include "internal.h"
#include "intersect.cuh"

namespace dipl {
namespace {

constexpr int kTraceThreads = 128;
constexpr float kSlabWiden = 1e-6f;
constexpr float kPruneSlack = 1e-5f;

struct RayState {
    float3 o, d, inv;
    float tmin, tmax;
};

__device__ __forceinline__ RayState load_ray(const dipl_ray* rays, int64_t i) {
    const float4* r4 = reinterpret_cast<const float4*>(rays) + 2 * i;
    const float4 a = __ldg(r4), b = __ldg(r4 + 1);
    RayState r;
    r.o = make_float3(a.x, a.y, a.z);
    r.d = make_float3(b.x, b.y, b.z);
    r.tmin = a.w;
    r.tmax = b.w;
    // Directions below 1e-20 in magnitude are treated as +-1e-20 so that 1/d stays finite and a ray lying
    // on a slab plane is still inside it (0 * inf would be NaN).
    auto safe = [](float x) { return fabsf(x) < 1e-20f ? copysignf(1e-20f, x) : x; };
    r.inv = make_float3(__frcp_rn(safe(r.d.x)), __frcp_rn(safe(r.d.y)), __frcp_rn(safe(r.d.z)));
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

template <int STACK>
struct Stack {
    int ref[STACK];
    float t[STACK];
    int sp = 0;
};

// Leaf test dispatch: ref_mt or watertight.
template <int LEAF>
__device__ __forceinline__ float leaf_test(float3 a, float3 b, float3 c, const RayState& r, const WtRay& w,
                                           bool backface, float& b1, float& b2) {
    if (LEAF == DIPL_LEAF_REF_MT) return mt_ref(a, b, c, r.o, r.d, backface, b1, b2);
    return wt_test(a, b, c, r.o, w, backface, b1, b2);
}

template <int LEAF, bool ANY, bool COUNT, int STACK>
__device__ __forceinline__ void trace_one(const BNode* __restrict__ nodes, const float4* __restrict__ tris, int root,
                                          int num_nodes, const dipl_ray* __restrict__ rays, int64_t i,
                                          dipl_hit* __restrict__ hits, uint8_t* __restrict__ occluded, uint32_t flags,
                                          uint32_t* __restrict__ err, unsigned& visits, unsigned& tests) {
    const RayState r = load_ray(rays, i);
    const bool backface = (flags & DIPL_TRACE_BACKFACE_CULLING) != 0u;
    WtRay w{};
    if (LEAF == DIPL_LEAF_WATERTIGHT) w = wt_setup(r.d);
    float best_t = r.tmax, best_u = 0.0f, best_v = 0.0f;
    int best_prim = -1;
    bool found = false;
    Stack<STACK> st;
    int cur = (num_nodes >= 0) ? root : 0x7FFFFFFF;  // num_nodes < 0 marks an empty BVH
    bool bad = false;
    // Each node is entered at most once per ray; the limit only guards against a corrupted tree.
    const uint32_t step_limit = 2u * (uint32_t)max(num_nodes, 0) + 64u;
    uint32_t steps = 0;
    while (cur != 0x7FFFFFFF) {
        if (++steps > step_limit) {
            bad = true;
            break;
        }
        if (cur >= 0) {
            if (cur >= num_nodes) {
                bad = true;
                break;
            }
            const float4* np = reinterpret_cast<const float4*>(nodes + cur);
            const float4 a = __ldg(np), b = __ldg(np + 1), c = __ldg(np + 2);
            const int4 d = __ldg(reinterpret_cast<const int4*>(np + 3));
            if (COUNT) ++visits;
            const float lim = prune_limit(best_t);
            const float t0 = box_entry(r, a.x, a.y, a.z, a.w, c.x, c.y, lim);
            const float t1 = box_entry(r, b.x, b.y, b.z, b.w, c.z, c.w, lim);
            const bool h0 = t0 != __int_as_float(0x7F800000), h1 = t1 != __int_as_float(0x7F800000);
            if (h0 && h1) {
                const bool first0 = t0 <= t1;
                if (st.sp >= STACK) {
                    bad = true;
                    break;
                }
                st.ref[st.sp] = first0 ? d.y : d.x;
                st.t[st.sp] = first0 ? t1 : t0;
                ++st.sp;
                cur = first0 ? d.x : d.y;
                continue;
            }
            if (h0) {
                cur = d.x;
                continue;
            }
            if (h1) {
                cur = d.y;
                continue;
            }
        } else {
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
                } else if (t > r.tmin && t < kInfinity && (t < best_t || (t == best_t && found && prim < best_prim))) {
                    best_t = t;
                    best_prim = prim;
                    best_u = b1;
                    best_v = b2;
                    found = true;
                }
            }
            if (ANY && found) break;
        }
        // pop the next entry that can still hold a better hit
        cur = 0x7FFFFFFF;
        const float lim = prune_limit(best_t);
        while (st.sp > 0) {
            --st.sp;
            if (st.t[st.sp] <= lim) {
                cur = st.ref[st.sp];
                break;
            }
        }
    }
    if (bad) atomicOr(err, kErrStack);
    if (ANY) {
        occluded[i] = found ? 1 : 0;
    } else {
        int4 out;
        out.x = found ? best_prim : -1;
        out.y = __float_as_int(found ? best_t : __int_as_float(0x7F800000));
        out.z = __float_as_int(found ? best_u : 0.0f);
        out.w = __float_as_int(found ? best_v : 0.0f);
        reinterpret_cast<int4*>(hits)[i] = out;
    }
}

template <int LEAF, bool ANY, bool COUNT, int STACK>
__global__ void __launch_bounds__(kTraceThreads) trace_kernel(const BNode* __restrict__ nodes,
                                                              const float4* __restrict__ tris, int root,
                                                              int num_nodes, const dipl_ray* __restrict__ rays,
                                                              int64_t n, dipl_hit* __restrict__ hits,
                                                              uint8_t* __restrict__ occluded, uint32_t flags,
                                                              unsigned long long* __restrict__ counters,
                                                              uint32_t* __restrict__ err) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    unsigned visits = 0, tests = 0;
    if (i < n) trace_one<LEAF, ANY, COUNT, STACK>(nodes, tris, root, num_nodes, rays, i, hits, occluded, flags, err,
                                                   visits, tests);
    if (COUNT) {
        // every lane of the (full) warp reaches this point
        const unsigned v = __reduce_add_sync(0xffffffffu, visits);
        const unsigned t = __reduce_add_sync(0xffffffffu, tests);
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&counters[0], (unsigned long long)v);
            atomicAdd(&counters[1], (unsigned long long)t);
        }
    }
}

template <int LEAF, bool ANY, bool COUNT>
dipl_status launch_trace_stack(const dipl_bvh* b, const dipl_ray* rays, int64_t n, dipl_hit* hits, uint8_t* occ,
                               uint32_t flags, unsigned long long* counters, cudaStream_t s) {
    const unsigned grid = (unsigned)((n + kTraceThreads - 1) / kTraceThreads);
    const int num_nodes = b->num_triangles == 0 ? -1 : (int)b->node_capacity;
    const BNode* nodes = static_cast<const BNode*>(b->nodes);
    if (b->depth < 64)
        trace_kernel<LEAF, ANY, COUNT, 64><<<grid, kTraceThreads, 0, s>>>(nodes, b->tris, b->root, num_nodes, rays, n,
                                                                          hits, occ, flags, counters, b->d_err);
    else if (b->depth < 128)
        trace_kernel<LEAF, ANY, COUNT, 128><<<grid, kTraceThreads, 0, s>>>(nodes, b->tris, b->root, num_nodes, rays,
                                                                           n, hits, occ, flags, counters, b->d_err);
    else
        trace_kernel<LEAF, ANY, COUNT, 512><<<grid, kTraceThreads, 0, s>>>(nodes, b->tris, b->root, num_nodes, rays,
                                                                           n, hits, occ, flags, counters, b->d_err); note_launches();
    DIPL_CUDA(cudaGetLastError());
    return DIPL_OK;
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
