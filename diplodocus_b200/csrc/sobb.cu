// SOBB form: skewed oriented bounding boxes (after Kacerik et al., "SOBB: Skewed Oriented Bounding Boxes
// for Ray Tracing", 2025) refitted over the finished PLOC topology.
//
// Each child box is the intersection of three slabs along directions taken from a fixed table of up to 16
// directions (kdop_size / 2 of them: the axes, the 4 corner diagonals, the 6 edge diagonals, 3 more). The
// refit computes every node's k-DOP (the interval of projections on all table directions) bottom-up with
// one thread per leaf (the second thread to reach a parent continues upwards), then each child keeps the
// direction triple whose parallelepiped has the least surface area,
//   SA(a, b, c) = 2 (w_a w_b + w_b w_c + w_c w_a) / |det(n_a, n_b, n_c)|,  w = interval width.
// With the axes only (kdop_size 6) this is the AABB. Intervals are padded by 2^-20 of the subtree's
// coordinate magnitude (more than the rounding of an FP32 projection), and the traversal widens each slab by
// a bound on the rounding of the ray's own projection, so no hit of an exact test can be lost.
#include <cmath>
#include <mutex>

#include "internal.h"
#include "intersect.cuh"

namespace dipl {

namespace {

constexpr int kDirs = 16;

// Direction table (unnormalised components are fine: the same float values are used to build and to trace).
__constant__ float c_dir[kDirs][3] = {
    {1.f, 0.f, 0.f}, {0.f, 1.f, 0.f}, {0.f, 0.f, 1.f},
    {0.57735026f, 0.57735026f, 0.57735026f}, {0.57735026f, 0.57735026f, -0.57735026f},
    {0.57735026f, -0.57735026f, 0.57735026f}, {-0.57735026f, 0.57735026f, 0.57735026f},
    {0.70710677f, 0.70710677f, 0.f}, {0.70710677f, -0.70710677f, 0.f}, {0.70710677f, 0.f, 0.70710677f},
    {0.70710677f, 0.f, -0.70710677f}, {0.f, 0.70710677f, 0.70710677f}, {0.f, 0.70710677f, -0.70710677f},
    {0.f, 0.52573111f, 0.85065081f}, {0.52573111f, 0.85065081f, 0.f}, {0.85065081f, 0.f, 0.52573111f},
};

// 1/|det(n_a, n_b, n_c)| at a*256 + b*16 + c for a < b < c with |det| > 0.2, else 0; filled by the host once.
__constant__ float c_inv3[kDirs * kDirs * kDirs];

struct Kdop {
    float lo[kDirs], hi[kDirs];
};

__device__ __forceinline__ float proj(int i, float x, float y, float z) {
    return __fmaf_rn(c_dir[i][0], x, __fmaf_rn(c_dir[i][1], y, __fmul_rn(c_dir[i][2], z)));
}

struct SobbIn {
    const int4* child;
    const float4* node_lo;
    const float4* node_hi;
    const int* parent;
    const int* leaf_start_of;
    const float4* btris;
    int N;
    int L;
    int dirs;
};

__device__ __forceinline__ int scount(const SobbIn& S, int id) {
    return id < S.N ? 1 : __float_as_int(S.node_lo[id - S.N].w);
}

__device__ __forceinline__ unsigned atomic_add_acq_rel(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Stores / loads a k-DOP as 8 float4 (the whole struct stays in registers: every index is a constant).
__device__ __forceinline__ void store_kdop(Kdop* dst, const Kdop& k) {
    float4* d = reinterpret_cast<float4*>(dst);
#pragma unroll
    for (int i = 0; i < kDirs / 4; ++i) {
        d[i] = make_float4(k.lo[4 * i], k.lo[4 * i + 1], k.lo[4 * i + 2], k.lo[4 * i + 3]);
        d[kDirs / 4 + i] = make_float4(k.hi[4 * i], k.hi[4 * i + 1], k.hi[4 * i + 2], k.hi[4 * i + 3]);
    }
}

// Up the tree from node x with its k-DOP k and magnitude m already stored: the second arriver at a parent merges
// the sibling's k-DOP and continues.
__device__ __forceinline__ void kdop_ascend(const SobbIn& S, int x, Kdop& k, float m, Kdop* __restrict__ kdop,
                                            float* __restrict__ mag, unsigned* __restrict__ arrivals) {
    for (int guard = 0; guard < 4096; ++guard) {
        const int par = S.parent[x];
        if (par < 0) return;
        // release: our k-DOP is visible before the count moves; acquire: so is the sibling's when we are second
        if (atomic_add_acq_rel(&arrivals[par - S.N], 1u) == 0u) return;  // the sibling is not done yet
        const int4 c = S.child[par - S.N];
        const int sib = c.x == x ? c.y : c.x;
        // the sibling's k-DOP was written by another SM: read through L2 (no stale L1 lines)
        const float4* b = reinterpret_cast<const float4*>(kdop + sib);
#pragma unroll
        for (int i = 0; i < kDirs / 4; ++i) {
            const float4 bl = __ldcg(b + i), bh = __ldcg(b + kDirs / 4 + i);
            k.lo[4 * i] = fminf(k.lo[4 * i], bl.x), k.lo[4 * i + 1] = fminf(k.lo[4 * i + 1], bl.y);
            k.lo[4 * i + 2] = fminf(k.lo[4 * i + 2], bl.z), k.lo[4 * i + 3] = fminf(k.lo[4 * i + 3], bl.w);
            k.hi[4 * i] = fmaxf(k.hi[4 * i], bh.x), k.hi[4 * i + 1] = fmaxf(k.hi[4 * i + 1], bh.y);
            k.hi[4 * i + 2] = fmaxf(k.hi[4 * i + 2], bh.z), k.hi[4 * i + 3] = fmaxf(k.hi[4 * i + 3], bh.w);
        }
        m = fmaxf(m, __ldcg(mag + sib));
        store_kdop(kdop + par, k);
        mag[par] = m;
        x = par;
    }
}

__device__ __forceinline__ void empty_kdop(Kdop& k) {
#pragma unroll
    for (int i = 0; i < kDirs; ++i) k.lo[i] = __int_as_float(0x7F800000), k.hi[i] = __int_as_float(0xFF800000);
}

// k-DOP of a final leaf from its triangles, then up the tree: the second arriver at a parent merges. All 16
// table directions are always projected (a smaller kdop_size only restricts which triples the node kernel
// considers), so the k-DOP never leaves registers. In a pre-split build a reference bounds only the part of its
// triangle inside the reference's box, so each slot's triangle k-DOP is first intersected with the k-DOP of its
// reference's box (each interval of the intersection holds the projections of every point of the triangle inside
// the box; an interval that rounding leaves empty keeps the triangle's), then merged into the leaf's.
__global__ void __launch_bounds__(256) kdop_refit_kernel(SobbIn S, const int* __restrict__ owner_leaf,
                                                         SobbRefs refs, Kdop* __restrict__ kdop,
                                                         float* __restrict__ mag, unsigned* __restrict__ arrivals,
                                                         const uint32_t* err) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= S.N || *err != 0u) return;
    int x = owner_leaf[p];
    if (x < 0) return;
    const int cnt = scount(S, x);
    const int start = S.leaf_start_of[x];
    const float4* t = S.btris + 3 * (long long)start;
    Kdop k;
    float m = 0.0f;
    empty_kdop(k);
    for (int tr = 0; tr < cnt; ++tr) {
        const float4 q0 = __ldg(t + 3 * tr), q1 = __ldg(t + 3 * tr + 1), q2 = __ldg(t + 3 * tr + 2);
        // a triangle with a non-finite coordinate is never hit: it adds nothing
        if (!(isfinite(q0.x) && isfinite(q0.y) && isfinite(q0.z) && isfinite(q1.x) && isfinite(q1.y) &&
              isfinite(q1.z) && isfinite(q2.x) && isfinite(q2.y) && isfinite(q2.z)))
            continue;
        m = fmaxf(m, fmaxf(fmaxf(fmaxf(fabsf(q0.x), fabsf(q0.y)), fmaxf(fabsf(q0.z), fabsf(q1.x))),
                           fmaxf(fmaxf(fabsf(q1.y), fabsf(q1.z)), fmaxf(fmaxf(fabsf(q2.x), fabsf(q2.y)), fabsf(q2.z)))));
        float4 lo = make_float4(0.f, 0.f, 0.f, 0.f), hi = lo;
        if (refs.slot_pos) {
            const long long r = refs.perm[refs.slot_pos[start + tr]];
            lo = __ldg(refs.rbox + 2 * r), hi = __ldg(refs.rbox + 2 * r + 1);
        }
#pragma unroll
        for (int i = 0; i < kDirs; ++i) {
            const float d0 = proj(i, q0.x, q0.y, q0.z), d1 = proj(i, q1.x, q1.y, q1.z), d2 = proj(i, q2.x, q2.y, q2.z);
            float tl = fminf(fminf(d0, d1), d2), th = fmaxf(fmaxf(d0, d1), d2);
            if (refs.slot_pos) {
                const float bl = proj(i, c_dir[i][0] >= 0.0f ? lo.x : hi.x, c_dir[i][1] >= 0.0f ? lo.y : hi.y,
                                      c_dir[i][2] >= 0.0f ? lo.z : hi.z);
                const float bh = proj(i, c_dir[i][0] >= 0.0f ? hi.x : lo.x, c_dir[i][1] >= 0.0f ? hi.y : lo.y,
                                      c_dir[i][2] >= 0.0f ? hi.z : lo.z);
                const float nl = fmaxf(tl, bl), nh = fminf(th, bh);
                if (nl <= nh) tl = nl, th = nh;
            }
            k.lo[i] = fminf(k.lo[i], tl);
            k.hi[i] = fmaxf(k.hi[i], th);
        }
    }
    store_kdop(kdop + x, k);
    mag[x] = m;
    kdop_ascend(S, x, k, m, kdop, mag, arrivals);
}

// One warp per inner node of the final layout, one half-warp per child; lane l of a half holds the child's
// interval on direction l. Only the 8 directions of least width take part (ranked in the half by width,
// ties to the lower index): their C(8,3) = 56 triples are spread over the 16 lanes, each looks up 1/|det|
// in a dense 16^3 table (0 = not admissible: |det| <= 0.2, or a direction beyond kdop_size / 2), and a
// 16-lane minimum over (area, a*256 + b*16 + c) keeps the least area, ties to the lexicographically first
// triple. Any triple bounds the child (every slab holds all its geometry), so the choice only steers
// traversal cost; the axes are the fallback when no candidate triple is admissible.
constexpr int kSobbNodeThreads = 256;

// The 56 index triples i < j < k of 0..7, packed i | j << 3 | k << 6.
__constant__ unsigned short c_combo8[56] = {
#define DIPL_C8(i, j, k) (unsigned short)((i) | ((j) << 3) | ((k) << 6))
    DIPL_C8(0, 1, 2), DIPL_C8(0, 1, 3), DIPL_C8(0, 1, 4), DIPL_C8(0, 1, 5), DIPL_C8(0, 1, 6), DIPL_C8(0, 1, 7),
    DIPL_C8(0, 2, 3), DIPL_C8(0, 2, 4), DIPL_C8(0, 2, 5), DIPL_C8(0, 2, 6), DIPL_C8(0, 2, 7), DIPL_C8(0, 3, 4),
    DIPL_C8(0, 3, 5), DIPL_C8(0, 3, 6), DIPL_C8(0, 3, 7), DIPL_C8(0, 4, 5), DIPL_C8(0, 4, 6), DIPL_C8(0, 4, 7),
    DIPL_C8(0, 5, 6), DIPL_C8(0, 5, 7), DIPL_C8(0, 6, 7), DIPL_C8(1, 2, 3), DIPL_C8(1, 2, 4), DIPL_C8(1, 2, 5),
    DIPL_C8(1, 2, 6), DIPL_C8(1, 2, 7), DIPL_C8(1, 3, 4), DIPL_C8(1, 3, 5), DIPL_C8(1, 3, 6), DIPL_C8(1, 3, 7),
    DIPL_C8(1, 4, 5), DIPL_C8(1, 4, 6), DIPL_C8(1, 4, 7), DIPL_C8(1, 5, 6), DIPL_C8(1, 5, 7), DIPL_C8(1, 6, 7),
    DIPL_C8(2, 3, 4), DIPL_C8(2, 3, 5), DIPL_C8(2, 3, 6), DIPL_C8(2, 3, 7), DIPL_C8(2, 4, 5), DIPL_C8(2, 4, 6),
    DIPL_C8(2, 4, 7), DIPL_C8(2, 5, 6), DIPL_C8(2, 5, 7), DIPL_C8(2, 6, 7), DIPL_C8(3, 4, 5), DIPL_C8(3, 4, 6),
    DIPL_C8(3, 4, 7), DIPL_C8(3, 5, 6), DIPL_C8(3, 5, 7), DIPL_C8(3, 6, 7), DIPL_C8(4, 5, 6), DIPL_C8(4, 5, 7),
    DIPL_C8(4, 6, 7), DIPL_C8(5, 6, 7),
#undef DIPL_C8
};

__global__ void __launch_bounds__(kSobbNodeThreads) sobb_node_kernel(
    SobbIn S, const BNode* __restrict__ bnodes, const uint32_t* __restrict__ rev_index, int num_inner,
    const Kdop* __restrict__ kdop, const float* __restrict__ mag, SNode* __restrict__ snodes, const uint32_t* err) {
    __shared__ float s_inv[kDirs * kDirs * kDirs];
    __shared__ unsigned short s_combo[56];
    for (int t = threadIdx.x; t < kDirs * kDirs * kDirs; t += kSobbNodeThreads)
        s_inv[t] = ((t & 15) < S.dirs) ? c_inv3[t] : 0.0f;  // a < b < c: c < dirs admits the triple
    for (int t = threadIdx.x; t < 56; t += kSobbNodeThreads) s_combo[t] = c_combo8[t];
    __syncthreads();
    if (*err != 0u) return;
    const int lane = threadIdx.x & 31, l = lane & 15, half = lane >> 4;
    const int warps = (int)(gridDim.x * (kSobbNodeThreads / 32));
    // the node loop is warp-uniform and every loop below has a fixed trip count: all shuffles see 32 lanes
    for (int k = (int)((blockIdx.x * kSobbNodeThreads + threadIdx.x) >> 5); k < num_inner; k += warps) {
        if (__float_as_int(S.node_lo[k].w) < S.L) continue;  // not an inner node of the layout
        const int4 c = S.child[k];
        const int id = half ? c.y : c.x;
        const float* kd = reinterpret_cast<const float*>(kdop + id);
        const float lo = kd[l], hi = kd[kDirs + l];
        float w = hi - lo;
        if (!(w == w) || l >= S.dirs) w = __int_as_float(0x7F800000);  // NaN or unused direction: widest
        // rank of this direction by width within the half (ties to the lower index)
        int rank = 0;
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const float wm = __shfl_sync(0xffffffffu, w, m, 16);
            rank += (wm < w || (wm == w && m < l)) ? 1 : 0;
        }
        const uint32_t sel = (__ballot_sync(0xffffffffu, rank < 8) >> (16 * half)) & 0xFFFFu;
        // lane p < 8 of the half: the p-th selected direction in index order
        uint32_t mm = sel;
        for (int q = 0; q < (l & 7); ++q) mm &= mm - 1u;
        const int dir_p = __ffs(mm) - 1;
        const float w_p = __shfl_sync(0xffffffffu, w, dir_p & 15, 16);
        float best = __int_as_float(0x7F800000);
        uint32_t bkey = 0xFFFFFFFFu;
#pragma unroll
        for (int c0 = 0; c0 < 64; c0 += 16) {
            const int t = c0 + l;
            const uint32_t cb = t < 56 ? s_combo[t] : 0u;
            const int i = cb & 7, j = (cb >> 3) & 7, q = (cb >> 6) & 7;
            const float wa = __shfl_sync(0xffffffffu, w_p, i, 16), wb = __shfl_sync(0xffffffffu, w_p, j, 16),
                        wc = __shfl_sync(0xffffffffu, w_p, q, 16);
            const int a = __shfl_sync(0xffffffffu, dir_p, i, 16), b = __shfl_sync(0xffffffffu, dir_p, j, 16),
                      cc = __shfl_sync(0xffffffffu, dir_p, q, 16);
            const uint32_t key = (uint32_t)(a * 256 + b * 16 + cc);
            const float inv = t < 56 ? s_inv[key & 4095u] : 0.0f;
            if (inv > 0.0f) {
                const float sa = (wa * wb + wb * wc + wc * wa) * inv;
                if (sa < best || (sa == best && key < bkey)) {
                    best = sa;
                    bkey = key;
                }
            }
        }
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) {
            const float ob = __shfl_xor_sync(0xffffffffu, best, o, 16);
            const uint32_t ok = __shfl_xor_sync(0xffffffffu, bkey, o, 16);
            if (ob < best || (ob == best && ok < bkey)) {
                best = ob;
                bkey = ok;
            }
        }
        if (bkey == 0xFFFFFFFFu) bkey = (0u << 8) | (1u << 4) | 2u;  // the axes
        const int ax0 = (int)(bkey >> 8), ax1 = (int)((bkey >> 4) & 15u), ax2 = (int)(bkey & 15u);
        const uint32_t abc = (uint32_t)ax0 | ((uint32_t)ax1 << 8) | ((uint32_t)ax2 << 16);
        const float pad = mag[id] * 9.5367431640625e-07f + 1e-30f;
        const float lo0 = __shfl_sync(0xffffffffu, lo, ax0, 16) - pad, hi0 = __shfl_sync(0xffffffffu, hi, ax0, 16) + pad;
        const float lo1 = __shfl_sync(0xffffffffu, lo, ax1, 16) - pad, hi1 = __shfl_sync(0xffffffffu, hi, ax1, 16) + pad;
        const float lo2 = __shfl_sync(0xffffffffu, lo, ax2, 16) - pad, hi2 = __shfl_sync(0xffffffffu, hi, ax2, 16) + pad;
        // child 1's values to lane 0
        const float r0 = __shfl_down_sync(0xffffffffu, lo0, 16), r1 = __shfl_down_sync(0xffffffffu, hi0, 16);
        const float r2 = __shfl_down_sync(0xffffffffu, lo1, 16), r3 = __shfl_down_sync(0xffffffffu, hi1, 16);
        const float r4 = __shfl_down_sync(0xffffffffu, lo2, 16), r5 = __shfl_down_sync(0xffffffffu, hi2, 16);
        const int rax = __shfl_down_sync(0xffffffffu, (int)abc, 16);
        if (lane == 0) {
            const int f = (int)rev_index[num_inner - 1 - k];
            SNode nd;
            nd.a = make_float4(lo0, hi0, lo1, hi1);
            nd.b = make_float4(lo2, hi2, r0, r1);
            nd.c = make_float4(r2, r3, r4, r5);
            const int4 refs = bnodes[f].d;  // the same references as the binary layout
            nd.d = make_int4(refs.x, refs.y, (int)abc, rax);
            snodes[f] = nd;
        }
    }
}

// ------------------------------------------------------------------------------------------------
// Traversal: the ray's projections on the table directions are computed once per ray into shared memory.
// ------------------------------------------------------------------------------------------------
constexpr int kSThreads = 128;
constexpr float kSSlabWiden = 1e-6f;
constexpr float kSPruneSlack = 1e-5f;

template <int LEAF>
__device__ __forceinline__ float sleaf_test(float3 a, float3 b, float3 c, float3 o, float3 d, const WtRay& w,
                                            bool backface, float& b1, float& b2) {
    if (LEAF == DIPL_LEAF_REF_MT) return mt_ref(a, b, c, o, d, backface, b1, b2);
    return wt_test(a, b, c, o, w, backface, b1, b2);
}

// The ray's record per table direction, in its shared-memory column: projected origin, reciprocal projected
// direction, and the two widening terms (the rounding of the projected origin as a distance along the ray,
// absolute, and of the projected direction as a relative error of every distance on this slab, large for grazing
// slabs), so a slab costs one shared load.
__device__ __forceinline__ void sobb_ray_setup(float4 (*s_ray)[kSThreads], int tid, int dirs, float3 o, float3 d) {
    const float omag = fabsf(o.x) + fabsf(o.y) + fabsf(o.z);
    const float dmag = fabsf(d.x) + fabsf(d.y) + fabsf(d.z);
    for (int k = 0; k < dirs; ++k) {
        const float dk = proj(k, d.x, d.y, d.z);
        const float inv = __frcp_rn(fabsf(dk) < 1e-20f ? copysignf(1e-20f, dk) : dk);
        s_ray[k][tid] = make_float4(proj(k, o.x, o.y, o.z), inv, omag * 4.0e-7f * fabsf(inv),
                                    kSSlabWiden + dmag * 4.0e-7f * fabsf(inv));
    }
}

// Entry distance of the ray into one child's three slabs (directions packed in `axes`, one per byte), widened by
// the ray's rounding terms; +inf when the slabs are missed, end before tmin or start beyond lim.
__device__ __forceinline__ float sobb_slab_box(const float4 (*s_ray)[kSThreads], int tid, int axes, float l0, float h0,
                                               float l1, float h1, float l2, float h2, float tmin, float lim) {
    float tn = __int_as_float(0xFF800000), tf = __int_as_float(0x7F800000);
    const float ls[3] = {l0, l1, l2}, hs[3] = {h0, h1, h2};
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const int k = (axes >> (8 * j)) & 0xFF;
        const float4 q = s_ray[k][tid];
        const float ok = q.x, inv = q.y, tol = q.z, rel = q.w;
        const float t0 = __fmul_rn(__fsub_rn(ls[j], ok), inv), t1 = __fmul_rn(__fsub_rn(hs[j], ok), inv);
        const float a0 = fminf(t0, t1), a1 = fmaxf(t0, t1);
        tn = fmaxf(tn, a0 - fabsf(a0) * rel - tol);
        tf = fminf(tf, a1 + fabsf(a1) * rel + tol);
    }
    return (tn <= tf && tf >= tmin && tn <= lim) ? tn : __int_as_float(0x7F800000);
}

// One SOBB node: both children's entry distances (t0, t1; +inf when missed) and their references (dd.x, dd.y).
__device__ __forceinline__ int4 sobb_children(const SNode* __restrict__ nodes, int cur,
                                              const float4 (*s_ray)[kSThreads], int tid, float tmin, float lim,
                                              float& t0, float& t1) {
    const float4* np = reinterpret_cast<const float4*>(nodes + cur);
    const float4 a = __ldg(np), b = __ldg(np + 1), c = __ldg(np + 2);
    const int4 dd = __ldg(reinterpret_cast<const int4*>(np + 3));
    t0 = sobb_slab_box(s_ray, tid, dd.z, a.x, a.y, a.z, a.w, b.x, b.y, tmin, lim);
    t1 = sobb_slab_box(s_ray, tid, dd.w, b.z, b.w, c.x, c.y, c.z, c.w, tmin, lim);
    return dd;
}

template <int LEAF, bool ANY, bool COUNT, int STACK>
__global__ void __launch_bounds__(kSThreads) sobb_trace_kernel(const SNode* __restrict__ nodes,
                                                               const float4* __restrict__ tris, int root,
                                                               int num_nodes, int dirs, const dipl_ray* __restrict__ rays,
                                                               int64_t n, dipl_hit* __restrict__ hits,
                                                               uint8_t* __restrict__ occluded, uint32_t flags,
                                                               unsigned long long* __restrict__ counters,
                                                               uint32_t* __restrict__ err, uint32_t step_limit,
                                                               const uint32_t* __restrict__ order) {
    __shared__ float4 s_ray[kDirs][kSThreads];  // the rays' records per direction (sobb_ray_setup)
    const int64_t work = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;  // position in the work order
    unsigned visits = 0, tests = 0;
    if (work < n) {
        const int64_t i = order ? (int64_t)__ldg(order + work) : work;  // the ray's own index
        const int tid = threadIdx.x;
        const float4* r4 = reinterpret_cast<const float4*>(rays) + 2 * i;
        const float4 ra = __ldg(r4), rb = __ldg(r4 + 1);
        const float3 o = make_float3(ra.x, ra.y, ra.z), d = make_float3(rb.x, rb.y, rb.z);
        const float tmin = ra.w, tmax = rb.w;
        sobb_ray_setup(s_ray, tid, dirs, o, d);
        const bool backface = (flags & DIPL_TRACE_BACKFACE_CULLING) != 0u;
        WtRay w{};
        if (LEAF == DIPL_LEAF_WATERTIGHT) w = wt_setup(d);
        float best_t = tmax, best_u = 0.0f, best_v = 0.0f;
        int best_prim = -1;
        bool found = false, bad = false;
        int sref[STACK];
        float st[STACK];
        int sp = 0;
        int cur = num_nodes >= 0 ? root : 0x7FFFFFFF;
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
                if (COUNT) ++visits;
                float t0, t1;
                const int4 dd = sobb_children(nodes, cur, s_ray, tid, tmin, best_t + fabsf(best_t) * kSPruneSlack,
                                              t0, t1);
                const bool h0 = t0 != __int_as_float(0x7F800000), h1 = t1 != __int_as_float(0x7F800000);
                if (h0 && h1) {
                    const bool first0 = t0 <= t1;
                    if (sp >= STACK) {
                        bad = true;
                        break;
                    }
                    sref[sp] = first0 ? dd.y : dd.x;
                    st[sp] = first0 ? t1 : t0;
                    ++sp;
                    cur = first0 ? dd.x : dd.y;
                    continue;
                }
                if (h0) {
                    cur = dd.x;
                    continue;
                }
                if (h1) {
                    cur = dd.y;
                    continue;
                }
            } else {
                // one triangle per step (the rest of the leaf stays in cur), so a lane at a leaf does not hold
                // its warp for the leaf's other triangles
                const int first = leaf_first(cur), cnt = leaf_count(cur);
                const float4* tp = tris + 3 * (int64_t)first;
                const float4 p0 = __ldg(tp), p1 = __ldg(tp + 1), p2 = __ldg(tp + 2);
                const int prim = __float_as_int(p0.w);
                float b1 = 0.0f, b2 = 0.0f;
                const float t = sleaf_test<LEAF>(make_float3(p0.x, p0.y, p0.z), make_float3(p1.x, p1.y, p1.z),
                                                 make_float3(p2.x, p2.y, p2.z), o, d, w, backface, b1, b2);
                if (COUNT) ++tests;
                if (ANY) {
                    if (t > tmin && t < tmax && t < kInfinity) found = true;
                } else if (t > tmin && t < kInfinity && (t < best_t || (t == best_t && found && prim < best_prim))) {
                    best_t = t, best_prim = prim, best_u = b1, best_v = b2, found = true;
                }
                if (ANY && found) break;
                if (cnt > 1) {
                    cur = make_leaf_ref(first + 1, cnt - 1);
                    continue;
                }
            }
            cur = 0x7FFFFFFF;
            const float lim = best_t + fabsf(best_t) * kSPruneSlack;
            while (sp > 0) {
                --sp;
                if (st[sp] <= lim) {
                    cur = sref[sp];
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
    if (COUNT) {
        const unsigned v = __reduce_add_sync(0xffffffffu, visits);
        const unsigned t = __reduce_add_sync(0xffffffffu, tests);
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&counters[0], (unsigned long long)v);
            atomicAdd(&counters[1], (unsigned long long)t);
        }
    }
}

// Persistent form for rays in the given order: every lane advances its ray by one node, one leaf triangle or one
// pop per step and takes the warp's next ray when its own ends, and the warps take 32-ray groups interleaved over
// the batch (warp w takes groups w, w + W, ...), so no lane waits for its warp's longest ray (the one-thread-per-ray
// kernel above stays for the coherent order, where lanes that start neighbouring rays together matter more).
template <int LEAF, bool ANY, bool COUNT, int STACK>
__global__ void __launch_bounds__(kSThreads) sobb_persist_kernel(const SNode* __restrict__ nodes,
                                                                 const float4* __restrict__ tris, int root,
                                                                 int num_nodes, int dirs,
                                                                 const dipl_ray* __restrict__ rays, int64_t n,
                                                                 dipl_hit* __restrict__ hits,
                                                                 uint8_t* __restrict__ occluded, uint32_t flags,
                                                                 unsigned long long* __restrict__ counters,
                                                                 uint32_t* __restrict__ err, uint32_t step_limit,
                                                                 const uint32_t* __restrict__ order) {
    constexpr int kDone = 0x7FFFFFFF;
    __shared__ float4 s_ray[kDirs][kSThreads];
    const unsigned full = 0xffffffffu;
    const int tid = threadIdx.x, lane = tid & 31;
    const int64_t warp_id = (blockIdx.x * (int64_t)blockDim.x + tid) >> 5;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    auto position = [&](int64_t k) -> int64_t { return (((k >> 5) * warps + warp_id) << 5) + (k & 31); };
    const uint32_t lt_mask = lanemask_lt();
    const bool backface = (flags & DIPL_TRACE_BACKFACE_CULLING) != 0u;
    unsigned visits = 0, tests = 0;
    bool bad = false;
    int64_t next = 0;  // rays this warp has taken (warp-uniform)
    int64_t my = -1;   // this lane's ray, -1 when idle
    float3 o = make_float3(0.f, 0.f, 0.f), d = o;
    float tmin = 0.0f, tmax = 0.0f;
    WtRay w{};
    float best_t = 0.0f, best_u = 0.0f, best_v = 0.0f;
    int best_prim = -1;
    bool found = false;
    int sref[STACK];
    float st[STACK];
    int sp = 0;
    int cur = kDone;
    uint32_t steps = 0;
    for (;;) {
        // ---- refill idle lanes --------------------------------------------------------------------------
        const bool idle = my < 0;
        const uint32_t idle_mask = __ballot_sync(full, idle);
        if (idle_mask) {
            if (idle) {
                const int64_t cand = position(next + __popc(idle_mask & lt_mask));
                if (cand < n) {
                    my = order ? (int64_t)__ldg(order + cand) : cand;  // the ray's own index (hits go there)
                    const float4* r4 = reinterpret_cast<const float4*>(rays) + 2 * my;
                    const float4 ra = __ldg(r4), rb = __ldg(r4 + 1);
                    o = make_float3(ra.x, ra.y, ra.z);
                    d = make_float3(rb.x, rb.y, rb.z);
                    tmin = ra.w;
                    tmax = rb.w;
                    sobb_ray_setup(s_ray, tid, dirs, o, d);
                    if (LEAF == DIPL_LEAF_WATERTIGHT) w = wt_setup(d);
                    best_t = tmax, best_u = 0.0f, best_v = 0.0f, best_prim = -1, found = false;
                    sp = 0;
                    steps = 0;
                    cur = num_nodes >= 0 ? root : kDone;
                }
            }
            if (position(next) < n) next += __popc(idle_mask);
        }
        if (!__ballot_sync(full, my >= 0)) break;
        if (my < 0) continue;

        // ---- one step: an inner node, one leaf triangle, or a pop -------------------------------------------
        bool finished = false, pop = false;
        if (cur == kDone) {
            finished = true;  // empty BVH
        } else if (++steps > step_limit || (cur >= 0 && cur >= num_nodes)) {
            bad = true;  // only a corrupted tree gets here
            finished = true;
        } else if (cur >= 0) {
            if (COUNT) ++visits;
            float t0, t1;
            const int4 dd = sobb_children(nodes, cur, s_ray, tid, tmin, best_t + fabsf(best_t) * kSPruneSlack, t0, t1);
            const bool h0 = t0 != __int_as_float(0x7F800000), h1 = t1 != __int_as_float(0x7F800000);
            if (h0 && h1) {
                const bool first0 = t0 <= t1;
                if (sp >= STACK) {
                    bad = true;
                    finished = true;
                } else {
                    sref[sp] = first0 ? dd.y : dd.x;
                    st[sp] = first0 ? t1 : t0;
                    ++sp;
                    cur = first0 ? dd.x : dd.y;
                }
            } else if (h0) {
                cur = dd.x;
            } else if (h1) {
                cur = dd.y;
            } else {
                pop = true;
            }
        } else {
            // one triangle per step (the rest of the leaf stays in cur)
            const int first = leaf_first(cur), cnt = leaf_count(cur);
            const float4* tp = tris + 3 * (int64_t)first;
            const float4 p0 = __ldg(tp), p1 = __ldg(tp + 1), p2 = __ldg(tp + 2);
            const int prim = __float_as_int(p0.w);
            float b1 = 0.0f, b2 = 0.0f;
            const float t = sleaf_test<LEAF>(make_float3(p0.x, p0.y, p0.z), make_float3(p1.x, p1.y, p1.z),
                                             make_float3(p2.x, p2.y, p2.z), o, d, w, backface, b1, b2);
            if (COUNT) ++tests;
            if (ANY) {
                if (t > tmin && t < tmax && t < kInfinity) found = true;
            } else if (t > tmin && t < kInfinity && (t < best_t || (t == best_t && found && prim < best_prim))) {
                best_t = t, best_prim = prim, best_u = b1, best_v = b2, found = true;
            }
            if (ANY && found) finished = true;
            else if (cnt > 1) cur = make_leaf_ref(first + 1, cnt - 1);
            else pop = true;
        }
        if (pop) {
            cur = kDone;
            const float lim = best_t + fabsf(best_t) * kSPruneSlack;
            while (sp > 0) {
                --sp;
                if (st[sp] <= lim) {
                    cur = sref[sp];
                    break;
                }
            }
            if (cur == kDone) finished = true;
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
        const unsigned v = __reduce_add_sync(full, visits);
        const unsigned t = __reduce_add_sync(full, tests);
        if (lane == 0) {
            atomicAdd(&counters[0], (unsigned long long)v);
            atomicAdd(&counters[1], (unsigned long long)t);
        }
    }
}

// Resident blocks of a traversal kernel on the current device (probed once per device and kernel).
template <typename Kernel>
int sobb_grid(Kernel kernel) {
    static DeviceProbe probe;
    return probe_per_device(probe, [kernel] {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kSThreads, 0);
        (void)cudaGetLastError();
        return std::max(1, sms * std::max(1, per_sm));
    });
}

template <int LEAF, bool ANY, bool COUNT, int STACK>
dipl_status launch_sobb(const dipl_bvh* b, const dipl_ray* rays, int64_t n, dipl_hit* hits, uint8_t* occ,
                        uint32_t flags, unsigned long long* counters, cudaStream_t s) {
    const int num_nodes = b->num_triangles == 0 ? -1 : (int)b->node_capacity;
    RayOrder ro;
    if (reorder_rays(n, flags)) {
        const dipl_status st = make_ray_order(rays, n, b->d_err, s, ro);
        if (st != DIPL_OK) {
            if (ro.mem) device_free(ro.mem, s);
            return st;
        }
    }
    const uint32_t cap =
        trace_step_limit() ? trace_step_limit()
                           : (uint32_t)std::min<int64_t>(0xFFFFFFFFll, 2ll * std::max(num_nodes, 0) + b->num_refs + 64);
    if (ro.order) {
        sobb_trace_kernel<LEAF, ANY, COUNT, STACK><<<(unsigned)((n + kSThreads - 1) / kSThreads), kSThreads, 0, s>>>(
            static_cast<const SNode*>(b->nodes), b->tris, b->root, num_nodes, b->kdop / 2, rays, n, hits, occ, flags,
            counters, b->d_err, cap, ro.order);
    } else {
        auto kernel = sobb_persist_kernel<LEAF, ANY, COUNT, STACK>;
        const int64_t grid =
            std::max<int64_t>(1, std::min<int64_t>(sobb_grid(kernel), (n + kSThreads - 1) / kSThreads));
        kernel<<<(unsigned)grid, kSThreads, 0, s>>>(static_cast<const SNode*>(b->nodes), b->tris, b->root, num_nodes,
                                                    b->kdop / 2, rays, n, hits, occ, flags, counters, b->d_err, cap,
                                                    nullptr);
    }
    note_launches();
    const cudaError_t e = cudaGetLastError();
    if (ro.mem) device_free(ro.mem, s);
    DIPL_CUDA(e);
    return DIPL_OK;
}

template <int LEAF, bool ANY, bool COUNT>
dipl_status launch_sobb_stack(const dipl_bvh* b, const dipl_ray* rays, int64_t n, dipl_hit* hits, uint8_t* occ,
                              uint32_t flags, unsigned long long* counters, cudaStream_t s) {
    if (b->depth < 64) return launch_sobb<LEAF, ANY, COUNT, 64>(b, rays, n, hits, occ, flags, counters, s);
    if (b->depth < 128) return launch_sobb<LEAF, ANY, COUNT, 128>(b, rays, n, hits, occ, flags, counters, s);
    return launch_sobb<LEAF, ANY, COUNT, 512>(b, rays, n, hits, occ, flags, counters, s);
}

DeviceProbe g_triples_uploaded;  // per device: the table lives in each device's constant memory
int g_triples = 0;

dipl_status upload_triples() {
    static const float dirs[kDirs][3] = {
        {1.f, 0.f, 0.f}, {0.f, 1.f, 0.f}, {0.f, 0.f, 1.f},
        {0.57735026f, 0.57735026f, 0.57735026f}, {0.57735026f, 0.57735026f, -0.57735026f},
        {0.57735026f, -0.57735026f, 0.57735026f}, {-0.57735026f, 0.57735026f, 0.57735026f},
        {0.70710677f, 0.70710677f, 0.f}, {0.70710677f, -0.70710677f, 0.f}, {0.70710677f, 0.f, 0.70710677f},
        {0.70710677f, 0.f, -0.70710677f}, {0.f, 0.70710677f, 0.70710677f}, {0.f, 0.70710677f, -0.70710677f},
        {0.f, 0.52573111f, 0.85065081f}, {0.52573111f, 0.85065081f, 0.f}, {0.85065081f, 0.f, 0.52573111f},
    };
    static float inv[kDirs * kDirs * kDirs];
    int nt = 0;
    for (int a = 0; a < kDirs; ++a)
        for (int b = 0; b < kDirs; ++b)
            for (int c = 0; c < kDirs; ++c) {
                float& slot = inv[a * kDirs * kDirs + b * kDirs + c];
                slot = 0.0f;
                if (!(a < b && b < c)) continue;
                const float* A = dirs[a];
                const float* B = dirs[b];
                const float* Cc = dirs[c];
                const double det = (double)A[0] * (B[1] * Cc[2] - B[2] * Cc[1]) -
                                   (double)A[1] * (B[0] * Cc[2] - B[2] * Cc[0]) +
                                   (double)A[2] * (B[0] * Cc[1] - B[1] * Cc[0]);
                if (std::fabs(det) < 0.2) continue;
                slot = (float)(1.0 / std::fabs(det));
                ++nt;
            }
    DIPL_CUDA(cudaMemcpyToSymbol(c_inv3, inv, sizeof(inv)));
    g_triples = nt;
    return DIPL_OK;
}

}  // namespace

// Allocations of the SOBB refit (and the one-time upload of the direction triples).
dipl_status sobb_prepare(long long N, long long K, Storage& work, Storage& out, SobbScratch* sc, SNode** snodes) {
    dipl_status st = DIPL_OK;
    if (!probe_per_device(g_triples_uploaded, [] { return upload_triples() == DIPL_OK ? 1 : 0; })) {
        set_last_error("SOBB: upload of the direction-triple table failed");
        return DIPL_ERR_CUDA;
    }
    const long long Kalloc = std::max<long long>(K, 1);
    Kdop* kdop;
    if ((st = work.alloc(&kdop, (size_t)(N + Kalloc))) != DIPL_OK ||
        (st = work.alloc(&sc->mag, (size_t)(N + Kalloc))) != DIPL_OK ||
        (st = work.alloc(&sc->arrivals, (size_t)Kalloc)) != DIPL_OK || (st = out.alloc(snodes, (size_t)Kalloc)) != DIPL_OK)
        return st;
    sc->kdop = kdop;
    sc->triples = g_triples;
    return DIPL_OK;
}

// Refits SOBB child boxes over the binary layout (bnodes, final inner indices rev_index) into snodes.
dipl_status sobb_enqueue(const int4* child, const float4* node_lo, const float4* node_hi, const int* parent,
                         const int* leaf_start_of, const int* owner_leaf, const float4* btris, const BNode* bnodes,
                         const uint32_t* rev_index, int N, int K, int L, int kdop_size, const SobbScratch& sc,
                         const SobbRefs& refs, SNode* snodes, cudaStream_t s, uint32_t* d_err) {
    const int Kalloc = std::max(K, 1);
    Kdop* kdop = static_cast<Kdop*>(sc.kdop);
    DIPL_CUDA(cudaMemsetAsync(sc.arrivals, 0, sizeof(unsigned) * Kalloc, s));
    SobbIn S{child, node_lo, node_hi, parent, leaf_start_of, btris, N, L, kdop_size / 2};
    kdop_refit_kernel<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(S, owner_leaf, refs, kdop, sc.mag, sc.arrivals,
                                                                  d_err);
    note_launches();
    if (K > 0) {
        // persistent: each CTA stages the triple table once, then its warps stride over the nodes
        int dev = 0, sms = 0;
        DIPL_CUDA(cudaGetDevice(&dev));
        DIPL_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        const long long warps_needed = K;
        const long long grid = std::max<long long>(
            1, std::min<long long>((long long)sms * (2048 / kSobbNodeThreads),
                                   (warps_needed + kSobbNodeThreads / 32 - 1) / (kSobbNodeThreads / 32)));
        sobb_node_kernel<<<(unsigned)grid, kSobbNodeThreads, 0, s>>>(S, bnodes, rev_index, K, kdop, sc.mag, snodes,
                                                                     d_err);
        note_launches();
    }
    DIPL_CUDA(cudaGetLastError());
    return DIPL_OK;
}

dipl_status trace_sobb(const dipl_bvh* b, const dipl_ray* rays, int64_t n, dipl_hit* hits, uint8_t* occ, int leaf_test,
                       uint32_t flags, unsigned long long* counters, bool any, cudaStream_t s) {
    if (any)
        return leaf_test == DIPL_LEAF_REF_MT
                   ? launch_sobb_stack<DIPL_LEAF_REF_MT, true, false>(b, rays, n, nullptr, occ, flags, nullptr, s)
                   : launch_sobb_stack<DIPL_LEAF_WATERTIGHT, true, false>(b, rays, n, nullptr, occ, flags, nullptr, s);
    if (counters)
        return leaf_test == DIPL_LEAF_REF_MT
                   ? launch_sobb_stack<DIPL_LEAF_REF_MT, false, true>(b, rays, n, hits, nullptr, flags, counters, s)
                   : launch_sobb_stack<DIPL_LEAF_WATERTIGHT, false, true>(b, rays, n, hits, nullptr, flags, counters, s);
    return leaf_test == DIPL_LEAF_REF_MT
               ? launch_sobb_stack<DIPL_LEAF_REF_MT, false, false>(b, rays, n, hits, nullptr, flags, nullptr, s)
               : launch_sobb_stack<DIPL_LEAF_WATERTIGHT, false, false>(b, rays, n, hits, nullptr, flags, nullptr, s);
}

}  // namespace dipl
