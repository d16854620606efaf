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
#include <limits>

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

// Long rays of a warp that has no rays left to take move to tail_kernel: once at most kTailLanes lanes of the warp
// are still tracing, a lane whose ray has taken kTailSteps steps or more writes the ray's state (ray index, next
// node, best hit so far, stack) to a slot and takes no more work; tail_kernel then traverses each such ray with a
// whole warp. Without it the warp keeps issuing one-lane steps until its longest ray ends (the 1M sphere's
// grazing rays take up to ~430 steps). With all 32 lanes busy (the soup) nothing is offloaded: the warp is
// already fully used. Measured (4M rays on the 1M sphere / 1M rays on the 16M soup, identical hits): 0.633 ->
// 0.497 ms / 52.97 -> 51.85 ms; offloading at 8-32 steps sends rays whose remaining work is too short for a
// warp (sphere 0.73-0.84 ms), and offloading from full warps slows the soup (55.2 ms).
constexpr int kTailSteps = 64;
constexpr int kTailLanes = 8;  // ... and only when at most this many lanes of the warp are still tracing
constexpr int kTailHeaderInts = 12;  // ray (2), cur, sp, best t/u/v, prim, found, pad
constexpr size_t kTailBytes = 64u << 20;  // slot storage per trace call, at most
// Batches smaller than this trace without the offload: their warps run out of rays early, the rays of
// such batches are mostly short (a 512x512 frame of the small scene), and the offload's allocation, clearing
// and extra launch cost more there (0.243 against 0.279-0.289 ms per frame of two traces).
constexpr int64_t kTailMinRays = 1 << 19;

struct TailQueue {
    int* slots;          // slot_ints ints each: header, then sp (ref, t) pairs
    unsigned* count;     // [0]: slots written (may exceed cap), [1]: slots taken by tail_kernel
    int cap;             // slots available
    int slot_ints;
    int min_steps;       // 0: no offload
    int max_lanes;
    uint32_t step_limit; // steps one ray may take (both kernels), beyond which it is given up and flagged
};

// Float bits in an order that compares like the floats (for warp minima).
__device__ __forceinline__ unsigned ordered_bits(float f) {
    const unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float from_ordered_bits(unsigned k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

// Leaf test dispatch: ref_mt or watertight.
template <int LEAF>
__device__ __forceinline__ float leaf_test(float3 a, float3 b, float3 c, const RayState& r, const WtRay& w,
                                           bool backface, float& b1, float& b2) {
    if (LEAF == DIPL_LEAF_REF_MT) return mt_ref(a, b, c, r.o, r.d, backface, b1, b2);
    return wt_test(a, b, c, r.o, w, backface, b1, b2);
}

// Traversal: every lane advances its ray by one inner node or one leaf triangle per step. With a persistent grid
// (rays in the given order) a lane whose ray finished takes its warp's next ray at the following step, so lanes do
// not idle behind the warp's longest ray (most rays of a batch may finish at the root while a few descend to the
// leaves); with one lane per ray (the coherent order) each warp traces its 32 rays and hands long ones on.
template <int LEAF, bool ANY, bool COUNT, int STACK, int SHORT>
__global__ void __launch_bounds__(kTraceThreads, kTraceMinBlocks) trace_kernel(const BNode* __restrict__ nodes,
                                                              const float4* __restrict__ tris, int root,
                                                              int num_nodes, const dipl_ray* __restrict__ rays,
                                                              int64_t n, dipl_hit* __restrict__ hits,
                                                              uint8_t* __restrict__ occluded, uint32_t flags,
                                                              unsigned long long* __restrict__ counters,
                                                              uint32_t* __restrict__ err, TailQueue tq,
                                                              const uint32_t* __restrict__ order) {
    __shared__ int2 sh_stack[SHORT > 0 ? SHORT * kTraceThreads : 1];
    const int lane = threadIdx.x & 31;
    const int64_t warp_id = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    // The k-th ray a warp takes is at position ((k / 32) * warps + warp) * 32 + k % 32 of the work order, so all
    // warps walk the order together and the rays in flight are one window of it (a coherent order then keeps the
    // whole GPU in one region of the tree; one chunk per warp measured 181 against 163 ms on the pre-split soup).
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t end = n;
    auto position = [&](int64_t k) -> int64_t { return (((k >> 5) * warps + warp_id) << 5) + (k & 31); };
    const bool backface = (flags & DIPL_TRACE_BACKFACE_CULLING) != 0u;
    const uint32_t lt_mask = lanemask_lt();
    const uint32_t step_limit = tq.step_limit;
    int64_t next = 0;    // rays this warp has taken (warp-uniform)
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
    bool may_offload = tq.min_steps > 0;
    for (;;) {
        // ---- refill idle lanes ---------------------------------------------------------------------
        const bool idle = my < 0;
        const uint32_t idle_mask = __ballot_sync(0xffffffffu, idle);
        if (idle_mask) {
            if (idle) {
                const int64_t cand = position(next + __popc(idle_mask & lt_mask));
                if (cand < end) {
                    my = order ? (int64_t)__ldg(order + cand) : cand;  // the ray's own index (hits go there)
                    r = load_ray(rays, my);
                    if (LEAF == DIPL_LEAF_WATERTIGHT) w = wt_setup(r.d);
                    best_t = r.tmax, best_u = 0.0f, best_v = 0.0f, best_prim = -1, found = false;
                    cur = num_nodes >= 0 ? root : 0x7FFFFFFF;
                    st.sp = 0;
                    steps = 0;
                }
            }
            if (position(next) < end) next += __popc(idle_mask);
        }
        const uint32_t active_mask = __ballot_sync(0xffffffffu, my >= 0);
        if (!active_mask) break;
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
            // one triangle per step: a lane at a leaf never holds the warp for the leaf's other triangles (the
            // rest of the leaf stays in cur as the reference of its remaining triangles)
            const int first = leaf_first(cur), cnt = leaf_count(cur);
            const float4* tp = tris + 3 * (int64_t)first;
            const float4 p0 = __ldg(tp), p1 = __ldg(tp + 1), p2 = __ldg(tp + 2);
            const int prim = __float_as_int(p0.w);
            float b1 = 0.0f, b2 = 0.0f;
            const float t = leaf_test<LEAF>(make_float3(p0.x, p0.y, p0.z), make_float3(p1.x, p1.y, p1.z),
                                            make_float3(p2.x, p2.y, p2.z), r, w, backface, b1, b2);
            if (COUNT) ++tests;
            // t == kInfinity is the tests' miss value (also when tmax is +inf)
            if (ANY) {
                if (t > r.tmin && t < r.tmax && t < kInfinity) found = true;
            } else if (t > r.tmin && t < kInfinity && (t < best_t || (t == best_t && found && prim < best_prim))) {
                best_t = t;
                best_prim = prim;
                best_u = b1;
                best_v = b2;
                found = true;
            }
            if (ANY && found) finished = true;
            else if (cnt > 1) cur = make_leaf_ref(first + 1, cnt - 1);
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
        } else if (may_offload && position(next) >= end && steps >= (uint32_t)tq.min_steps &&
                   __popc(active_mask) <= tq.max_lanes) {
            // the warp has no rays left and this ray is still going: hand it to tail_kernel if a slot is free
            const unsigned slot = atomicAdd(&tq.count[0], 1u);
            if (slot < (unsigned)tq.cap) {
                int* w = tq.slots + (size_t)slot * tq.slot_ints;
                w[0] = (int)(uint32_t)(uint64_t)my;
                w[1] = (int)(uint32_t)((uint64_t)my >> 32);
                w[2] = cur;
                w[3] = st.sp;
                w[4] = __float_as_int(best_t);
                w[5] = __float_as_int(best_u);
                w[6] = __float_as_int(best_v);
                w[7] = best_prim;
                w[8] = found ? 1 : 0;
                for (int k = 0; k < st.sp; ++k) reinterpret_cast<int2*>(w + kTailHeaderInts)[k] = st.get(k);
                my = -1;
            }
            may_offload = false;  // one try per lane
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

// One warp per offloaded ray. Its pending work (the node it was at and its stack entries) is dealt round-robin to
// the lanes; each lane traverses near-child first with its own stack, lanes without work take the bottom entry
// (the largest pending subtree) of a lane holding two or more, and every step prunes against the best t of the
// whole warp (warp minimum, the same conservative slack as the main kernel). Each lane accepts leaf hits by the
// closest-hit rule against its own best; the warp then keeps the smallest (t, primitive id) over its lanes and
// the hit carried over from the main kernel, so the record is the one a single thread would produce.
template <int LEAF, bool ANY, bool COUNT, int STACK>
__global__ void __launch_bounds__(kTraceThreads) tail_kernel(const BNode* __restrict__ nodes,
                                                             const float4* __restrict__ tris, int num_nodes,
                                                             const dipl_ray* __restrict__ rays,
                                                             dipl_hit* __restrict__ hits, uint8_t* __restrict__ occluded,
                                                             uint32_t flags, unsigned long long* __restrict__ counters,
                                                             uint32_t* __restrict__ err, TailQueue tq) {
    constexpr int kNone = -0x7FFFFFFF - 1;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const uint32_t lt_mask = lanemask_lt();
    const bool backface = (flags & DIPL_TRACE_BACKFACE_CULLING) != 0u;
    const uint32_t step_limit = tq.step_limit;
    const unsigned total = min(*reinterpret_cast<volatile unsigned*>(&tq.count[0]), (unsigned)tq.cap);
    if (total == 0) return;  // nothing was handed on: the whole grid leaves at once
    unsigned visits = 0, tests = 0;
    bool bad = false;
    int sref[STACK];
    float stt[STACK];
    for (;;) {
        // slots claimed one at a time: a warp that drew a short ray takes the next (a fixed warp stride
        // measured slower on the 1M sphere, 0.525 against 0.50 ms)
        unsigned slot = 0;
        if (lane == 0) slot = atomicAdd(&tq.count[1], 1u);
        slot = __shfl_sync(full, slot, 0);
        if (slot >= total) break;
        const int* w = tq.slots + (size_t)slot * tq.slot_ints;
        const int64_t my = (int64_t)(((uint64_t)(uint32_t)w[1] << 32) | (uint32_t)w[0]);
        const int sp0 = min(w[3], STACK);
        const RayState r = load_ray(rays, my);
        WtRay wt{};
        if (LEAF == DIPL_LEAF_WATERTIGHT) wt = wt_setup(r.d);
        float best_t = r.tmax, best_u = 0.0f, best_v = 0.0f;
        int best_prim = -1;
        bool found = false;
        if (lane == 0 && w[8]) {
            best_t = __int_as_float(w[4]), best_u = __int_as_float(w[5]), best_v = __int_as_float(w[6]);
            best_prim = w[7];
            found = true;
        }
        // deal the pending items: stack entries 0..sp0-1, then the node the ray was at (always visited)
        int bot = 0, sp = 0, cur = kNone;
        for (int k = lane; k <= sp0; k += 32) {
            int ref;
            float t;
            if (k < sp0) {
                const int2 e = reinterpret_cast<const int2*>(w + kTailHeaderInts)[k];
                ref = e.x, t = __int_as_float(e.y);
            } else {
                ref = w[2], t = -__int_as_float(0x7F800000);
            }
            sref[sp] = ref, stt[sp] = t, ++sp;
        }
        uint32_t steps = 0;
        for (;;) {
            const float gbest = from_ordered_bits(__reduce_min_sync(full, ordered_bits(best_t)));
            const float lim = prune_limit(gbest);
            while (cur == kNone && sp > bot) {
                --sp;
                if (stt[sp] <= lim) cur = sref[sp];
            }
            if (sp == bot) sp = bot = 0;
            const bool hungry = cur == kNone;
            const uint32_t hm = __ballot_sync(full, hungry);
            if (hm == full) break;
            if (hm) {
                const uint32_t dm = __ballot_sync(full, sp - bot >= 2);
                const int nh = __popc(hm), nd = __popc(dm);
                const bool donate = ((dm >> lane) & 1u) && __popc(dm & lt_mask) < nh;
                int gref = kNone;
                float gt = 0.0f;
                if (donate) {
                    gref = sref[bot], gt = stt[bot];
                    ++bot;
                }
                const int rank = __popc(hm & lt_mask);
                const bool receive = hungry && rank < nd;
                const int src = receive ? (int)__fns(dm, 0, rank + 1) : lane;
                const int rref = __shfl_sync(full, gref, src);
                const float rt = __shfl_sync(full, gt, src);
                if (receive && rref != kNone && rt <= lim) cur = rref;
            }
            if (cur != kNone) {
                if (++steps > step_limit || (cur >= 0 && cur >= num_nodes)) {
                    bad = true;
                    cur = kNone;
                    sp = bot = 0;
                } else if (cur >= 0) {
                    const float4* np = reinterpret_cast<const float4*>(nodes + cur);
                    float4 a, b, c, df;
                    ldg_v8(np, a, b);
                    ldg_v8(np + 2, c, df);
                    if (COUNT) ++visits;
                    const float t0 = box_entry(r, a.x, a.y, a.z, a.w, c.x, c.y, lim);
                    const float t1 = box_entry(r, b.x, b.y, b.z, b.w, c.z, c.w, lim);
                    const bool h0 = t0 != __int_as_float(0x7F800000), h1 = t1 != __int_as_float(0x7F800000);
                    const int c0 = __float_as_int(df.x), c1 = __float_as_int(df.y);
                    if (h0 && h1) {
                        const bool first0 = t0 <= t1;
                        if (sp >= STACK) {
                            bad = true;
                            cur = kNone;
                        } else {
                            sref[sp] = first0 ? c1 : c0, stt[sp] = first0 ? t1 : t0, ++sp;
                            cur = first0 ? c0 : c1;
                        }
                    } else {
                        cur = h0 ? c0 : (h1 ? c1 : kNone);
                    }
                } else {
                    const int first = leaf_first(cur), cnt = leaf_count(cur);
                    for (int k = 0; k < cnt; ++k) {
                        const float4* tp = tris + 3 * (int64_t)(first + k);
                        const float4 p0 = __ldg(tp), p1 = __ldg(tp + 1), p2 = __ldg(tp + 2);
                        const int prim = __float_as_int(p0.w);
                        float b1 = 0.0f, b2 = 0.0f;
                        const float t = leaf_test<LEAF>(make_float3(p0.x, p0.y, p0.z), make_float3(p1.x, p1.y, p1.z),
                                                        make_float3(p2.x, p2.y, p2.z), r, wt, backface, b1, b2);
                        if (COUNT) ++tests;
                        if (ANY) {
                            if (t > r.tmin && t < r.tmax && t < kInfinity) found = true;
                        } else if (t > r.tmin && t < kInfinity &&
                                   (t < best_t || (t == best_t && found && prim < best_prim))) {
                            best_t = t, best_prim = prim, best_u = b1, best_v = b2, found = true;
                        }
                    }
                    cur = kNone;
                }
            }
            if (ANY && __any_sync(full, found)) break;
        }
        // the smallest (t, primitive id) of the warp
        if (ANY) {
            const bool any = __any_sync(full, found);
            if (lane == 0) occluded[my] = any ? 1 : 0;
        } else {
            const unsigned tk = found ? ordered_bits(best_t) : 0xFFFFFFFFu;
            const unsigned tmin = __reduce_min_sync(full, tk);
            const bool cand = found && tk == tmin;
            const unsigned pmin = __reduce_min_sync(full, cand ? (unsigned)best_prim : 0xFFFFFFFFu);
            const uint32_t win = __ballot_sync(full, cand && (unsigned)best_prim == pmin);
            const int wl = win ? __ffs(win) - 1 : 0;
            const float ft = __shfl_sync(full, best_t, wl), fu = __shfl_sync(full, best_u, wl),
                        fv = __shfl_sync(full, best_v, wl);
            const int fp = __shfl_sync(full, best_prim, wl);
            if (lane == 0) {
                int4 out;
                out.x = win ? fp : -1;
                out.y = __float_as_int(win ? ft : __int_as_float(0x7F800000));
                out.z = __float_as_int(win ? fu : 0.0f);
                out.w = __float_as_int(win ? fv : 0.0f);
                reinterpret_cast<int4*>(hits)[my] = out;
            }
        }
    }
    if (bad) atomicOr(err, kErrStack);
    if (COUNT) {
        const unsigned v = __reduce_add_sync(full, visits);
        const unsigned t = __reduce_add_sync(full, tests);
        if (lane == 0) {
            atomicAdd(&counters[0], (unsigned long long)v);
            atomicAdd(&counters[1], (unsigned long long)t);
        }
    }
}

// ---- ray order ----------------------------------------------------------------------------------------
// On request, batches of at least kReorderMinRays rays are traced in the order of a 30-bit key: the direction's octant
// above a 9-bit-per-axis Morton code of the origin within the batch's origin bounds. A warp's 32 rays then
// start in one small region and head the same way, so its lanes fetch the same nodes and branch alike.
// Records still go to each ray's own index; only the order of work changes, never a result.
constexpr int kReorderBits = 30;

__global__ void __launch_bounds__(256) ray_bounds_kernel(const dipl_ray* __restrict__ rays, int64_t n,
                                                         int* __restrict__ box) {
    float lo[3] = {__int_as_float(0x7F800000), __int_as_float(0x7F800000), __int_as_float(0x7F800000)};
    float hi[3] = {__int_as_float(0xFF800000), __int_as_float(0xFF800000), __int_as_float(0xFF800000)};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float4 o = __ldg(reinterpret_cast<const float4*>(rays) + 2 * i);
        const float v[3] = {o.x, o.y, o.z};
        for (int a = 0; a < 3; ++a)
            if (isfinite(v[a])) lo[a] = fminf(lo[a], v[a]), hi[a] = fmaxf(hi[a], v[a]);
    }
    for (int a = 0; a < 3; ++a) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(box + a, float_to_ordered(lo[a]));
            atomicMax(box + 3 + a, float_to_ordered(hi[a]));
        }
    }
}

__global__ void ray_box_init_kernel(int* box) {
    if (threadIdx.x < 6)
        box[threadIdx.x] = float_to_ordered(__int_as_float(threadIdx.x < 3 ? 0x7F800000 : 0xFF800000));
}

__device__ __forceinline__ uint32_t spread3_9(uint32_t x) {  // 9 bits to every third bit
    x &= 0x1FFu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

__global__ void __launch_bounds__(256) ray_keys_kernel(const dipl_ray* __restrict__ rays, int64_t n,
                                                       const int* __restrict__ box, uint32_t* __restrict__ keys) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 o = __ldg(reinterpret_cast<const float4*>(rays) + 2 * i);
    const float4 d = __ldg(reinterpret_cast<const float4*>(rays) + 2 * i + 1);
    const float v[3] = {o.x, o.y, o.z};
    uint32_t cell[3];
    for (int a = 0; a < 3; ++a) {
        const float lo = ordered_to_float(__ldg(box + a)), hi = ordered_to_float(__ldg(box + 3 + a));
        const float ext = hi - lo;
        const float q = ext > 0.0f ? (v[a] - lo) * (512.0f / ext) : 0.0f;
        cell[a] = (uint32_t)fminf(fmaxf(q, 0.0f), 511.0f);  // NaN -> 0
    }
    const uint32_t oct = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
    keys[i] = (oct << 27) | (spread3_9(cell[0]) << 2) | (spread3_9(cell[1]) << 1) | spread3_9(cell[2]);
}

// Blocks of a persistent trace launch: every resident block on every SM (per kernel instantiation and device).
template <typename K>
int persistent_grid(K kernel) {
    static DeviceProbe probe;  // per instantiation
    return probe_per_device(probe, [kernel] {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kTraceThreads, 0);
        (void)cudaGetLastError();
        return std::max(1, sms * std::max(1, per_sm));
    });
}

template <int LEAF, bool ANY, bool COUNT, int STACK, int SHORT>
dipl_status launch_trace(const dipl_bvh* b, const dipl_ray* rays, int64_t n, dipl_hit* hits, uint8_t* occ,
                         uint32_t flags, unsigned long long* counters, cudaStream_t s) {
    auto kernel = trace_kernel<LEAF, ANY, COUNT, STACK, SHORT>;
    // Rays in the coherent order get one lane each (a grid over the whole batch, blocks launched in order): the
    // GPU then works through the sorted order as one moving window and the lanes of a warp start neighbouring rays
    // together; long rays still move to tail_kernel. Measured on the pre-split 16M soup with 16M sorted rays: 137.7
    // ms (Morton30 126.7 ms) against 160.7 ms (147.8 ms) with persistent warps refilling lanes. Rays in the given
    // order keep the persistent grid, where a lane takes its warp's next ray when its own ends (the 1M sphere's
    // grazing rays would otherwise hold their warps).
    const int max_grid = reorder_rays(n, flags) ? std::numeric_limits<int>::max() : persistent_grid(kernel);
    const int64_t warps_needed = (n + 31) / 32;
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(max_grid, (warps_needed * 32 + kTraceThreads - 1) /
                                                                               kTraceThreads));
    const int num_nodes = b->num_triangles == 0 ? -1 : (int)b->node_capacity;
    if ((reinterpret_cast<uintptr_t>(b->nodes) & 63) != 0) {
        set_last_error("trace: node array is not 64-byte aligned");
        return DIPL_ERR_INTERNAL;
    }
    // a ray takes at most one step per inner node and one per leaf triangle
    const uint32_t steps_cap = trace_step_limit() ? trace_step_limit()
                                                  : (uint32_t)std::min<int64_t>(0xFFFFFFFFll, 2ll * std::max(num_nodes, 0) +
                                                                                                b->num_refs + 64);
    TailQueue tq{nullptr, nullptr, 0, kTailHeaderInts + 2 * STACK, n >= kTailMinRays ? kTailSteps : 0, kTailLanes,
                 steps_cap};
    void* tail_mem = nullptr;
    if (tq.min_steps > 0) {
        const size_t slot_bytes = sizeof(int) * (size_t)tq.slot_ints;
        tq.cap = (int)std::max<int64_t>(1, std::min<int64_t>(n, (int64_t)(kTailBytes / slot_bytes)));
        const size_t bytes = (size_t)tq.cap * slot_bytes;
        dipl_status st = device_alloc(&tail_mem, bytes + 16, s);
        if (st != DIPL_OK) return st;
        tq.slots = static_cast<int*>(tail_mem);
        tq.count = reinterpret_cast<unsigned*>(static_cast<char*>(tail_mem) + bytes);
        const cudaError_t e = cudaMemsetAsync(tq.count, 0, 2 * sizeof(unsigned), s);
        if (e != cudaSuccess) {
            device_free(tail_mem, s);
            return cuda_status(e, "cudaMemsetAsync");
        }
    }
    RayOrder ro;
    if (reorder_rays(n, flags)) {
        dipl_status st = make_ray_order(rays, n, b->d_err, s, ro);
        if (st != DIPL_OK) {
            if (ro.mem) device_free(ro.mem, s);
            device_free(tail_mem, s);
            return st;
        }
    }
    kernel<<<(unsigned)grid, kTraceThreads, 0, s>>>(static_cast<const BNode*>(b->nodes), b->tris, b->root, num_nodes,
                                                   rays, n, hits, occ, flags, counters, b->d_err, tq,
                                                   ro.order);
    note_launches();
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && tq.min_steps > 0) {
        auto tk = tail_kernel<LEAF, ANY, COUNT, STACK>;
        tk<<<(unsigned)persistent_grid(tk), kTraceThreads, 0, s>>>(static_cast<const BNode*>(b->nodes), b->tris,
                                                                   num_nodes, rays, hits, occ, flags, counters,
                                                                   b->d_err, tq);
        note_launches();
        e = cudaGetLastError();
    }
    device_free(tail_mem, s);
    if (ro.mem) device_free(ro.mem, s);
    DIPL_CUDA(e);
    return DIPL_OK;
}

template <int LEAF, bool ANY, bool COUNT>
dipl_status launch_trace_stack(const dipl_bvh* b, const dipl_ray* rays, int64_t n, dipl_hit* hits, uint8_t* occ,
                               uint32_t flags, unsigned long long* counters, cudaStream_t s) {
    // The top 16 stack entries live in shared memory (16 KB per 128-thread block), the rest in local memory.
    // Measured with the one-triangle step (pre-split 16M soup, EMC60 / Morton30, 16M rays; 1M sphere, 4M rays):
    // coherent order 137.8 -> 127.2 ms / 126.7 -> 116.6 ms, given order 212.9 -> 216.2 ms / 159.8 -> 140.4 ms,
    // sphere 0.545 -> 0.501 ms; 8 entries in shared memory gained nothing.
    if (b->depth < 64) return launch_trace<LEAF, ANY, COUNT, 64, 16>(b, rays, n, hits, occ, flags, counters, s);
    if (b->depth < 128) return launch_trace<LEAF, ANY, COUNT, 128, 16>(b, rays, n, hits, occ, flags, counters, s);
    return launch_trace<LEAF, ANY, COUNT, 512, 16>(b, rays, n, hits, occ, flags, counters, s);
}

}  // namespace

dipl_status make_ray_order(const dipl_ray* rays, int64_t n, uint32_t* d_err, cudaStream_t s, RayOrder& ro) {
    const size_t sort_bytes = radix_sort_scratch_bytes(n, 0, kReorderBits, 8);
    const size_t key_bytes = sizeof(uint32_t) * (size_t)n;
    const size_t bytes = 256 + 5 * key_bytes + sort_bytes;
    dipl_status st = device_alloc(&ro.mem, bytes, s);
    if (st != DIPL_OK) return st;
    unsigned char* base = static_cast<unsigned char*>(ro.mem);
    int* box = reinterpret_cast<int*>(base);
    uint32_t* keys = reinterpret_cast<uint32_t*>(base + 256);
    uint32_t* keys_sorted = keys + n;
    uint32_t* keys_alt = keys_sorted + n;
    ro.order = keys_alt + n;
    uint32_t* order_alt = ro.order + n;
    unsigned char* scratch = reinterpret_cast<unsigned char*>(order_alt + n);
    ray_box_init_kernel<<<1, 32, 0, s>>>(box);
    note_launches();
    const int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
    ray_bounds_kernel<<<grid, 256, 0, s>>>(rays, n, box);
    note_launches();
    ray_keys_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(rays, n, box, keys);
    note_launches();
    DIPL_CUDA(cudaGetLastError());
    return radix_sort_pairs(keys, nullptr, keys_sorted, ro.order, keys_alt, order_alt, n, 4, 0, kReorderBits, 8,
                            scratch, s, d_err);
}


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
