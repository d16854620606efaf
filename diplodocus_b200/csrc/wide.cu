// Precision form: 8-wide BVH with 8-bit conservatively quantised child bounds (80-byte nodes, after Ylitie,
// Karras & Laine, "Efficient Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs", HPG 2017) and
// FP32 triangles re-tested at the leaves.
//
// Collapse: every wide node starts from one binary PLOC node with at least L triangles and repeatedly opens
// its child of largest surface area that is itself such a node, until it has 8 children or only leaves.
// Levels are built breadth first (one collapse kernel, two scans and one write kernel per level), so the
// inner children of a node are contiguous (child_base + rank) and its leaves' triangles are contiguous
// (tri_base + offset).
//
// Quantisation: per node an origin p (the min corner of the padded children) and per axis a power-of-two
// scale 2^e with extent / 2^e <= 255; child bounds q_lo = floor, q_hi = ceil, then adjusted until the FP32
// decode fmaf(q, 2^e, p) lies outside the padded child box. The traversal decodes with the same fmaf, so
// every decoded box contains its (already padded) child box: no ray can lose a hit against the FP32 nodes.
#include "internal.h"
#include "intersect.cuh"

namespace dipl {
namespace {

constexpr int kWideThreads = 256;

struct WideIn {
    const int4* child;
    const float4* node_lo;
    const float4* node_hi;
    const int* leaf_start_of;  // binary leaf range start by node id
    const float4* btris;       // binary leaf triangles
    int N;
    int L;
};

__device__ __forceinline__ int wcount(const WideIn& W, int id) {
    return id < W.N ? 1 : __float_as_int(W.node_lo[id - W.N].w);
}

__device__ __forceinline__ void wbox(const WideIn& W, int id, float3& lo, float3& hi) {
    if (id < W.N) {
        const float4* t = W.btris + 3 * (long long)W.leaf_start_of[id];
        const float4 a = t[0], b = t[1], c = t[2];
        if (!(isfinite(a.x) && isfinite(a.y) && isfinite(a.z) && isfinite(b.x) && isfinite(b.y) && isfinite(b.z) &&
              isfinite(c.x) && isfinite(c.y) && isfinite(c.z))) {
            // never hit (NaN t under both leaf tests): an empty box, like the build's cluster boxes
            lo = make_float3(__int_as_float(0x7F800000), __int_as_float(0x7F800000), __int_as_float(0x7F800000));
            hi = make_float3(__int_as_float(0xFF800000), __int_as_float(0xFF800000), __int_as_float(0xFF800000));
            return;
        }
        lo = make_float3(fminf(fminf(a.x, b.x), c.x), fminf(fminf(a.y, b.y), c.y), fminf(fminf(a.z, b.z), c.z));
        hi = make_float3(fmaxf(fmaxf(a.x, b.x), c.x), fmaxf(fmaxf(a.y, b.y), c.y), fmaxf(fmaxf(a.z, b.z), c.z));
    } else {
        const float4 a = W.node_lo[id - W.N], b = W.node_hi[id - W.N];
        lo = make_float3(a.x, a.y, a.z);
        hi = make_float3(b.x, b.y, b.z);
    }
}

__device__ __forceinline__ float wpad_down(float lo, float hi) {
    const float m = fmaxf(fabsf(lo), fabsf(hi));
    return lo - (m * 9.5367431640625e-07f + 1e-30f);
}
__device__ __forceinline__ float wpad_up(float lo, float hi) {
    const float m = fmaxf(fabsf(lo), fabsf(hi));
    return hi + (m * 9.5367431640625e-07f + 1e-30f);
}

// One thread per frontier node: the collapsed child list (binary node ids, inner ones first in list order).
__global__ void wide_collapse_kernel(WideIn W, const int* __restrict__ frontier, int n_front,
                                     int* __restrict__ kids /*8 per entry*/, uint32_t* __restrict__ n_inner,
                                     uint32_t* __restrict__ n_tris, const uint32_t* err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_front) return;
    if (*err != 0u) {
        n_inner[i] = 0;
        n_tris[i] = 0;
        return;
    }
    const int x = frontier[i];
    const int4 c = W.child[x - W.N];
    int list[8];
    int cnt = 2;
    list[0] = c.x;
    list[1] = c.y;
    while (cnt < 8) {
        int best = -1;
        double best_area = -1.0;
        for (int k = 0; k < cnt; ++k) {
            const int id = list[k];
            if (id < W.N || wcount(W, id) < W.L) continue;
            float3 lo, hi;
            wbox(W, id, lo, hi);
            const double dx = (double)hi.x - lo.x, dy = (double)hi.y - lo.y, dz = (double)hi.z - lo.z;
            const double area = dx * dy + dy * dz + dz * dx;
            if (area > best_area) {
                best_area = area;
                best = k;
            }
        }
        if (best < 0) break;
        const int4 cc = W.child[list[best] - W.N];
        list[best] = cc.x;
        list[cnt++] = cc.y;
    }
    uint32_t ni = 0, nt = 0;
    for (int k = 0; k < 8; ++k) {
        const int id = k < cnt ? list[k] : -1;
        kids[8 * i + k] = id;
        if (id < 0) continue;
        const int n = wcount(W, id);
        if (n >= W.L) ++ni;
        else nt += (uint32_t)n;
    }
    n_inner[i] = ni;
    n_tris[i] = nt;
}

__device__ __forceinline__ void quantise_axis(float p, float ext, const float* lo, const float* hi, uint32_t valid,
                                              unsigned char* qlo, unsigned char* qhi, unsigned char& ebiased) {
    int e = -126;
    if (ext > 0.0f) {
        int ex = 0;
        frexpf(ext / 255.0f, &ex);  // ext/255 = m * 2^ex, m in [0.5, 1)
        e = max(-126, min(127, ex));
    }
    for (int attempt = 0; attempt < 4; ++attempt, e = min(127, e + 1)) {
        const float scale = ldexpf(1.0f, e);
        bool ok = true;
        for (int k = 0; k < 8; ++k) {
            if (!((valid >> k) & 1u)) {
                qlo[k] = 0, qhi[k] = 0;
                continue;
            }
            float a = floorf((lo[k] - p) / scale);
            float b = ceilf((hi[k] - p) / scale);
            a = fminf(fmaxf(a, 0.0f), 255.0f);
            b = fminf(fmaxf(b, 0.0f), 255.0f);
            while (a > 0.0f && __fmaf_rn(a, scale, p) > lo[k]) a -= 1.0f;
            while (b < 255.0f && __fmaf_rn(b, scale, p) < hi[k]) b += 1.0f;
            if (__fmaf_rn(a, scale, p) > lo[k] || __fmaf_rn(b, scale, p) < hi[k]) ok = false;
            qlo[k] = (unsigned char)a;
            qhi[k] = (unsigned char)b;
        }
        if (ok) break;
    }
    ebiased = (unsigned char)(e + 127);
}

// Writes one wide node per frontier entry. Children go to slots by octant (after Ylitie et al.): slot s
// stands for the direction (s&1 ? +x : -x, s&2 ? +y : -y, s&4 ? +z : -z) from the node centre, and the
// (child, slot) pairs are taken greedily by the largest projection of the child's centre offset on the
// slot direction. A ray whose direction signs form octant o then visits slots in the order s ^ o, which
// is roughly front to back. Inner children are ranked, and leaf triangles placed, in slot order.
__global__ void wide_write_kernel(WideIn W, const int* __restrict__ frontier, int n_front,
                                  const int* __restrict__ kids, const uint32_t* __restrict__ inner_prefix,
                                  const uint32_t* __restrict__ tri_prefix, int base, int next_base, int tri_next,
                                  WNode* __restrict__ nodes, float4* __restrict__ tris, int* __restrict__ frontier_out,
                                  const uint32_t* err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_front || *err != 0u) return;
    const int child_base = next_base + (int)inner_prefix[i];
    const int tri_base = tri_next + (int)tri_prefix[i];
    int cnt = 0;
    int ids[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        ids[k] = kids[8 * i + k];
        if (ids[k] >= 0) cnt = k + 1;
    }
    float clo[3][8], chi[3][8];
    float3 p = make_float3(__int_as_float(0x7F800000), __int_as_float(0x7F800000), __int_as_float(0x7F800000));
    float3 q = make_float3(-p.x, -p.y, -p.z);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        if (k >= cnt) continue;
        float3 l, h;
        wbox(W, ids[k], l, h);
        clo[0][k] = wpad_down(l.x, h.x), chi[0][k] = wpad_up(l.x, h.x);
        clo[1][k] = wpad_down(l.y, h.y), chi[1][k] = wpad_up(l.y, h.y);
        clo[2][k] = wpad_down(l.z, h.z), chi[2][k] = wpad_up(l.z, h.z);
        p = make_float3(fminf(p.x, clo[0][k]), fminf(p.y, clo[1][k]), fminf(p.z, clo[2][k]));
        q = make_float3(fmaxf(q.x, chi[0][k]), fmaxf(q.y, chi[1][k]), fmaxf(q.z, chi[2][k]));
    }
    // ---- greedy octant slot assignment -----------------------------------------------------------------
    const float cx = 0.5f * (p.x + q.x), cy = 0.5f * (p.y + q.y), cz = 0.5f * (p.z + q.z);
    float ox[8], oy[8], oz[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        ox[k] = k < cnt ? 0.5f * (clo[0][k] + chi[0][k]) - cx : 0.0f;
        oy[k] = k < cnt ? 0.5f * (clo[1][k] + chi[1][k]) - cy : 0.0f;
        oz[k] = k < cnt ? 0.5f * (clo[2][k] + chi[2][k]) - cz : 0.0f;
    }
    uint32_t free_k = (1u << cnt) - 1u, free_s = 0xFFu;
    int slot_of[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int round = 0; round < cnt; ++round) {
        float best = -__int_as_float(0x7F800000);
        int bk = -1, bs = -1;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (!((free_k >> k) & 1u)) continue;
#pragma unroll
            for (int s = 0; s < 8; ++s) {
                if (!((free_s >> s) & 1u)) continue;
                const float v = ((s & 1) ? ox[k] : -ox[k]) + ((s & 2) ? oy[k] : -oy[k]) + ((s & 4) ? oz[k] : -oz[k]);
                if (bk < 0 || v > best) {
                    best = v;
                    bk = k;
                    bs = s;
                }
            }
        }
        free_k &= ~(1u << bk);
        free_s &= ~(1u << bs);
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (k == bk) slot_of[k] = bs;
    }
    // children and padded boxes by slot
    int sid[8];
    float lo[3][8], hi[3][8];
    uint32_t valid = 0;
#pragma unroll
    for (int s = 0; s < 8; ++s) {
        sid[s] = -1;
        lo[0][s] = lo[1][s] = lo[2][s] = 0.0f;
        hi[0][s] = hi[1][s] = hi[2][s] = 0.0f;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (k < cnt && slot_of[k] == s) {
                sid[s] = ids[k];
                lo[0][s] = clo[0][k], lo[1][s] = clo[1][k], lo[2][s] = clo[2][k];
                hi[0][s] = chi[0][k], hi[1][s] = chi[1][k], hi[2][s] = chi[2][k];
            }
        }
        if (sid[s] >= 0) valid |= 1u << s;
    }
    WNode nd;
    nd.px = p.x, nd.py = p.y, nd.pz = p.z;
    quantise_axis(p.x, q.x - p.x, lo[0], hi[0], valid, nd.qlox, nd.qhix, nd.ex);
    quantise_axis(p.y, q.y - p.y, lo[1], hi[1], valid, nd.qloy, nd.qhiy, nd.ey);
    quantise_axis(p.z, q.z - p.z, lo[2], hi[2], valid, nd.qloz, nd.qhiz, nd.ez);
    nd.child_base = child_base;
    nd.tri_base = tri_base;
    unsigned char imask = 0;
    int rank = 0, toff = 0;
    for (int s = 0; s < 8; ++s) {
        nd.meta[s] = 0;
        const int id = sid[s];
        if (id < 0) continue;
        const int n = wcount(W, id);
        if (n >= W.L) {
            imask |= (unsigned char)(1u << s);
            frontier_out[(int)inner_prefix[i] + rank] = id;
            nd.meta[s] = (unsigned char)rank;
            ++rank;
        } else {
            nd.meta[s] = (unsigned char)((n << 5) | toff);
            const float4* src = W.btris + 3 * (long long)W.leaf_start_of[id];
            float4* dst = tris + 3 * (long long)(tri_base + toff);
            for (int t = 0; t < 3 * n; ++t) dst[t] = src[t];
            toff += n;
        }
    }
    nd.imask = imask;
    nodes[base + i] = nd;
}

__global__ void copy_tris_kernel(const float4* __restrict__ src, float4* __restrict__ dst, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 3 * count) dst[i] = src[i];
}

// ------------------------------------------------------------------------------------------------
// Traversal (after Ylitie et al.): the stack holds node groups, one 8-byte entry per wide node with
// children still to visit: the node's child base, its inner-slot mask and the not-yet-visited hit
// children as bits in visiting order (bit b = slot b ^ octant of the ray). Leaf triangles of a node are
// tested as soon as the node is intersected. A node taken from a group is not re-tested against its own
// box: its children's boxes are tested against the best t when it is visited.
// ------------------------------------------------------------------------------------------------
constexpr int kWTraceThreads = 128;
constexpr int kWTraceMinBlocks = 8;  // 8 resident blocks of 128 threads per SM: at most 64 registers
constexpr float kWSlabWiden = 1e-6f;
constexpr float kWPruneSlack = 1e-5f;

struct WRay {
    float3 o, d, inv;
    float tmin, tmax;
};

template <int LEAF>
__device__ __forceinline__ float wleaf_test(float3 a, float3 b, float3 c, const WRay& r, const WtRay& w, bool backface,
                                            float& b1, float& b2) {
    if (LEAF == DIPL_LEAF_REF_MT) return mt_ref(a, b, c, r.o, r.d, backface, b1, b2);
    return wt_test(a, b, c, r.o, w, backface, b1, b2);
}

// A ray of the 8-wide traversal (1/direction rounded to nearest) and its octant bits: slot s lies towards
// (s&1 ? +x : -x, ...), so a ray going -x meets the +x children first.
__device__ __forceinline__ WRay wide_load_ray(const dipl_ray* __restrict__ rays, int64_t i, uint32_t& oct) {
    const float4* r4 = reinterpret_cast<const float4*>(rays) + 2 * i;
    const float4 ra = __ldg(r4), rb = __ldg(r4 + 1);
    WRay r;
    r.o = make_float3(ra.x, ra.y, ra.z);
    r.d = make_float3(rb.x, rb.y, rb.z);
    r.tmin = ra.w;
    r.tmax = rb.w;
    auto safe = [](float x) { return fabsf(x) < 1e-20f ? copysignf(1e-20f, x) : x; };
    r.inv = make_float3(__frcp_rn(safe(r.d.x)), __frcp_rn(safe(r.d.y)), __frcp_rn(safe(r.d.z)));
    oct = (r.inv.x < 0.0f ? 1u : 0u) | (r.inv.y < 0.0f ? 2u : 0u) | (r.inv.z < 0.0f ? 4u : 0u);
    return r;
}

// The children of one wide node that the ray enters before `lim`: inner children as bits in visiting order
// (bit slot ^ octant), and the triangles of the hit leaf slots as bits over the node's triangle range.
struct WideHits {
    uint32_t inner, tris, imask;
    int child_base, tri_base;
};

__device__ __forceinline__ WideHits wide_node_hits(const WNode* __restrict__ nodes, int node, const WRay& r,
                                                   uint32_t oct, float lim) {
    const float4* np = reinterpret_cast<const float4*>(nodes + node);
    const float4 f0 = __ldg(np), f1 = __ldg(np + 1), f2 = __ldg(np + 2), f3 = __ldg(np + 3), f4 = __ldg(np + 4);
    const uint32_t eb = __float_as_uint(f0.w);
    const float sx = __uint_as_float((eb & 0xFFu) << 23), sy = __uint_as_float(((eb >> 8) & 0xFFu) << 23),
                sz = __uint_as_float(((eb >> 16) & 0xFFu) << 23);
    WideHits h;
    h.imask = eb >> 24;
    h.child_base = __float_as_int(f1.x);
    h.tri_base = __float_as_int(f1.y);
    h.inner = 0u;
    h.tris = 0u;
    const uint32_t meta_lo = __float_as_uint(f1.z), meta_hi = __float_as_uint(f1.w);
    const uint32_t qw[12] = {__float_as_uint(f2.x), __float_as_uint(f2.y), __float_as_uint(f2.z), __float_as_uint(f2.w),
                             __float_as_uint(f3.x), __float_as_uint(f3.y), __float_as_uint(f3.z), __float_as_uint(f3.w),
                             __float_as_uint(f4.x), __float_as_uint(f4.y), __float_as_uint(f4.z), __float_as_uint(f4.w)};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const uint32_t meta = ((k < 4 ? meta_lo : meta_hi) >> (8 * (k & 3))) & 0xFFu;
        const bool inner = (h.imask >> k) & 1u;
        if (!inner && meta == 0u) continue;
        auto qb = [&](int arr) { return (float)((qw[2 * arr + (k >> 2)] >> (8 * (k & 3))) & 0xFFu); };
        const float lx = __fmaf_rn(qb(0), sx, f0.x), ly = __fmaf_rn(qb(1), sy, f0.y), lz = __fmaf_rn(qb(2), sz, f0.z);
        const float hx = __fmaf_rn(qb(3), sx, f0.x), hy = __fmaf_rn(qb(4), sy, f0.y), hz = __fmaf_rn(qb(5), sz, f0.z);
        const float tx0 = __fmul_rn(__fsub_rn(lx, r.o.x), r.inv.x), tx1 = __fmul_rn(__fsub_rn(hx, r.o.x), r.inv.x);
        const float ty0 = __fmul_rn(__fsub_rn(ly, r.o.y), r.inv.y), ty1 = __fmul_rn(__fsub_rn(hy, r.o.y), r.inv.y);
        const float tz0 = __fmul_rn(__fsub_rn(lz, r.o.z), r.inv.z), tz1 = __fmul_rn(__fsub_rn(hz, r.o.z), r.inv.z);
        float tn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fminf(tz0, tz1));
        float tf = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fmaxf(tz0, tz1));
        tn = tn - fabsf(tn) * kWSlabWiden;
        tf = tf + fabsf(tf) * kWSlabWiden;
        if (!(tn <= tf && tf >= r.tmin && tn <= lim)) continue;
        if (inner) h.inner |= 1u << (k ^ oct);
        else h.tris |= ((1u << (meta >> 5)) - 1u) << (meta & 31u);
    }
    return h;
}

// After a visit: the first inner child hit is next, the others go on the stack as one group (child base, inner
// mask, remaining hits). False when the stack is full.
template <int STACK>
__device__ __forceinline__ bool wide_descend(const WideHits& h, uint32_t oct, int& node, int2* stack, int& sp) {
    node = -1;
    if (!h.inner) return true;
    uint32_t hits = h.inner;
    const int b = __ffs(hits) - 1;
    hits &= hits - 1u;
    node = h.child_base + __popc(h.imask & ((1u << ((uint32_t)b ^ oct)) - 1u));
    if (!hits) return true;
    if (sp >= STACK) return false;
    stack[sp++] = make_int2(h.child_base, (int)((hits << 8) | h.imask));
    return true;
}

// The next child of the top group (the group leaves the stack with its last child), -1 on an empty stack.
__device__ __forceinline__ int wide_pop(int2* stack, int& sp, uint32_t oct) {
    if (sp == 0) return -1;
    const int2 e = stack[sp - 1];
    uint32_t gh = (uint32_t)e.y >> 8;
    const uint32_t gi = (uint32_t)e.y & 0xFFu;
    const int b = __ffs(gh) - 1;
    gh &= gh - 1u;
    const int next = e.x + __popc(gi & ((1u << ((uint32_t)b ^ oct)) - 1u));
    if (gh) stack[sp - 1].y = (int)((gh << 8) | gi);
    else --sp;
    return next;
}

// One thread per ray in the work order, blocks launched in order: at any time the GPU traces one window of the
// order, and a warp's lanes start their rays together. Used for rays in the coherent order, where keeping the
// lanes of a warp on neighbouring rays matters more than not waiting for a warp's longest ray (16M-ray pre-split
// soup: 162.5 ms against 202 ms for the persistent kernel; given order 206.7 against 215.4 ms).
template <int LEAF, bool ANY, bool COUNT, int STACK>
__global__ void __launch_bounds__(kWTraceThreads) wide_block_kernel(
    const WNode* __restrict__ nodes, const float4* __restrict__ tris, int root, int num_nodes,
    const dipl_ray* __restrict__ rays, int64_t n, dipl_hit* __restrict__ hits, uint8_t* __restrict__ occluded,
    uint32_t flags, unsigned long long* __restrict__ counters, uint32_t* __restrict__ err, uint32_t step_limit,
    const uint32_t* __restrict__ order) {
    const int64_t work = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;  // position in the work order
    unsigned visits = 0, tests = 0;
    if (work < n) {
        const int64_t i = order ? (int64_t)__ldg(order + work) : work;  // the ray's own index
        uint32_t oct = 0;
        const WRay r = wide_load_ray(rays, i, oct);
        const bool backface = (flags & DIPL_TRACE_BACKFACE_CULLING) != 0u;
        WtRay w{};
        if (LEAF == DIPL_LEAF_WATERTIGHT) w = wt_setup(r.d);
        float best_t = r.tmax, best_u = 0.0f, best_v = 0.0f;
        int best_prim = -1;
        bool found = false, bad = false, done = false;
        auto test_tri = [&](int idx) {
            const float4* tp = tris + 3 * (int64_t)idx;
            const float4 p0 = __ldg(tp), p1 = __ldg(tp + 1), p2 = __ldg(tp + 2);
            const int prim = __float_as_int(p0.w);
            float b1 = 0.0f, b2 = 0.0f;
            const float t = wleaf_test<LEAF>(make_float3(p0.x, p0.y, p0.z), make_float3(p1.x, p1.y, p1.z),
                                             make_float3(p2.x, p2.y, p2.z), r, w, backface, b1, b2);
            if (COUNT) ++tests;
            if (ANY) {
                if (t > r.tmin && t < r.tmax && t < kInfinity) found = true;
            } else if (t > r.tmin && t < kInfinity && (t < best_t || (t == best_t && found && prim < best_prim))) {
                best_t = t, best_prim = prim, best_u = b1, best_v = b2, found = true;
            }
        };
        int2 stack[STACK];
        int sp = 0;
        int node = -1;
        if (num_nodes < 0) {
            done = true;  // empty BVH
        } else if (root < 0) {
            for (int k = 0, c = leaf_count(root); k < c && !(ANY && found); ++k) test_tri(leaf_first(root) + k);
            done = true;
        } else {
            node = root;
        }
        uint32_t steps = 0;
        while (!done) {
            if (++steps > step_limit) {
                bad = true;
                break;
            }
            if (node >= 0) {
                if (node >= num_nodes) {
                    bad = true;
                    break;
                }
                if (COUNT) ++visits;
                const WideHits h = wide_node_hits(nodes, node, r, oct, best_t + fabsf(best_t) * kWPruneSlack);
                for (uint32_t tm = h.tris; tm; tm &= tm - 1u) {
                    test_tri(h.tri_base + __ffs(tm) - 1);
                    if (ANY && found) break;
                }
                if (ANY && found) break;
                if (!wide_descend<STACK>(h, oct, node, stack, sp)) {
                    bad = true;
                    break;
                }
            } else {
                node = wide_pop(stack, sp, oct);
                if (node < 0) break;
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

// Persistent: every lane advances its ray by one wide node (its leaf triangles included) or one stack group per
// step; a lane whose ray has ended takes the warp's next ray at the following step, so lanes do not idle behind
// the warp's longest ray (the 1M sphere's 4M rays: 0.82 ms against 1.75 ms with one thread per ray). Used for rays
// in the given order.
template <int LEAF, bool ANY, bool COUNT, int STACK>
__global__ void __launch_bounds__(kWTraceThreads, kWTraceMinBlocks) wide_trace_kernel(
    const WNode* __restrict__ nodes, const float4* __restrict__ tris, int root, int num_nodes,
    const dipl_ray* __restrict__ rays, int64_t n, dipl_hit* __restrict__ hits, uint8_t* __restrict__ occluded,
    uint32_t flags, unsigned long long* __restrict__ counters, uint32_t* __restrict__ err, uint32_t step_limit,
    const uint32_t* __restrict__ order) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int64_t warp_id = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    // the k-th ray a warp takes is at position ((k / 32) * warps + warp) * 32 + k % 32 of the work order: all warps
    // walk the order together, so the rays in flight are one window of it (a coherent order then keeps the whole
    // GPU in one region of the tree)
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    auto position = [&](int64_t k) -> int64_t { return (((k >> 5) * warps + warp_id) << 5) + (k & 31); };
    const uint32_t lt_mask = lanemask_lt();
    const bool backface = (flags & DIPL_TRACE_BACKFACE_CULLING) != 0u;
    unsigned visits = 0, tests = 0;
    bool bad = false;
    int64_t next = 0;  // rays this warp has taken (warp-uniform)
    int64_t my = -1;   // this lane's ray, -1 when idle
    WRay r{};
    WtRay w{};
    uint32_t oct = 0;
    float best_t = 0.0f, best_u = 0.0f, best_v = 0.0f;
    int best_prim = -1;
    bool found = false;
    int2 stack[STACK];
    int sp = 0;
    int node = -1;
    uint32_t steps = 0;
    auto test_tri = [&](int idx) {
        const float4* tp = tris + 3 * (int64_t)idx;
        const float4 p0 = __ldg(tp), p1 = __ldg(tp + 1), p2 = __ldg(tp + 2);
        const int prim = __float_as_int(p0.w);
        float b1 = 0.0f, b2 = 0.0f;
        const float t = wleaf_test<LEAF>(make_float3(p0.x, p0.y, p0.z), make_float3(p1.x, p1.y, p1.z),
                                         make_float3(p2.x, p2.y, p2.z), r, w, backface, b1, b2);
        if (COUNT) ++tests;
        if (ANY) {
            if (t > r.tmin && t < r.tmax && t < kInfinity) found = true;
        } else if (t > r.tmin && t < kInfinity && (t < best_t || (t == best_t && found && prim < best_prim))) {
            best_t = t, best_prim = prim, best_u = b1, best_v = b2, found = true;
        }
    };
    for (;;) {
        // ---- refill idle lanes --------------------------------------------------------------------------
        const bool idle = my < 0;
        const uint32_t idle_mask = __ballot_sync(full, idle);
        bool done = false;
        if (idle_mask) {
            if (idle) {
                const int64_t cand = position(next + __popc(idle_mask & lt_mask));
                if (cand < n) {
                    my = order ? (int64_t)__ldg(order + cand) : cand;  // the ray's own index (hits go there)
                    r = wide_load_ray(rays, my, oct);
                    if (LEAF == DIPL_LEAF_WATERTIGHT) w = wt_setup(r.d);
                    best_t = r.tmax, best_u = 0.0f, best_v = 0.0f, best_prim = -1, found = false;
                    sp = 0;
                    steps = 0;
                    node = -1;
                    if (num_nodes < 0) {
                        done = true;  // empty BVH
                    } else if (root < 0) {
                        for (int k = 0, c = leaf_count(root); k < c && !(ANY && found); ++k) test_tri(leaf_first(root) + k);
                        done = true;
                    } else {
                        node = root;
                    }
                }
            }
            if (position(next) < n) next += __popc(idle_mask);
        }
        if (!__ballot_sync(full, my >= 0)) break;
        if (my < 0) continue;

        // ---- one step: a wide node (and its hit leaf triangles) or a stack group ----------------------------
        if (!done && ++steps > step_limit) {
            bad = true;
            done = true;
        } else if (!done && node >= 0) {
            if (node >= num_nodes) {
                bad = true;
                done = true;
            } else {
                if (COUNT) ++visits;
                const WideHits h = wide_node_hits(nodes, node, r, oct, best_t + fabsf(best_t) * kWPruneSlack);
                for (uint32_t tm = h.tris; tm; tm &= tm - 1u) {
                    test_tri(h.tri_base + __ffs(tm) - 1);
                    if (ANY && found) break;
                }
                if (ANY && found) {
                    node = -1;
                    done = true;
                } else if (!wide_descend<STACK>(h, oct, node, stack, sp)) {
                    bad = true;
                    done = true;
                }
            }
        } else if (!done) {
            node = wide_pop(stack, sp, oct);
            if (node < 0) done = true;
        }
        if (done) {
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

// Resident blocks of the traversal kernel on the current device (probed once per device and kernel).
template <typename Kernel>
int wide_grid(Kernel kernel) {
    static DeviceProbe probe;
    return probe_per_device(probe, [kernel] {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kWTraceThreads, 0);
        (void)cudaGetLastError();
        return std::max(1, sms * std::max(1, per_sm));
    });
}

template <int LEAF, bool ANY, bool COUNT, int STACK>
dipl_status launch_wide(const dipl_bvh* b, const dipl_ray* rays, int64_t n, dipl_hit* hits, uint8_t* occ, uint32_t flags,
                        unsigned long long* counters, cudaStream_t s) {
    const int num_nodes = b->num_triangles == 0 ? -1 : (int)b->node_capacity;
    RayOrder ro;
    if (reorder_rays(n, flags)) {
        const dipl_status st = make_ray_order(rays, n, b->d_err, s, ro);
        if (st != DIPL_OK) {
            if (ro.mem) device_free(ro.mem, s);
            return st;
        }
    }
    const uint32_t cap = trace_step_limit() ? trace_step_limit() : 2u * (uint32_t)std::max(num_nodes, 0) + 64u;
    if (ro.order) {
        wide_block_kernel<LEAF, ANY, COUNT, STACK><<<(unsigned)((n + kWTraceThreads - 1) / kWTraceThreads),
                                                     kWTraceThreads, 0, s>>>(
            static_cast<const WNode*>(b->nodes), b->tris, b->root, num_nodes, rays, n, hits, occ, flags, counters,
            b->d_err, cap, ro.order);
    } else {
        auto kernel = wide_trace_kernel<LEAF, ANY, COUNT, STACK>;
        const int64_t grid =
            std::max<int64_t>(1, std::min<int64_t>(wide_grid(kernel), (n + kWTraceThreads - 1) / kWTraceThreads));
        kernel<<<(unsigned)grid, kWTraceThreads, 0, s>>>(static_cast<const WNode*>(b->nodes), b->tris, b->root,
                                                         num_nodes, rays, n, hits, occ, flags, counters, b->d_err, cap,
                                                         nullptr);
    }
    note_launches();
    const cudaError_t e = cudaGetLastError();
    if (ro.mem) device_free(ro.mem, s);
    DIPL_CUDA(e);
    return DIPL_OK;
}

// At most one group per wide level is on the stack (depth = wide levels of the layout).
template <int LEAF, bool ANY, bool COUNT>
dipl_status launch_wide_stack(const dipl_bvh* b, const dipl_ray* rays, int64_t n, dipl_hit* hits, uint8_t* occ,
                              uint32_t flags, unsigned long long* counters, cudaStream_t s) {
    const int need = b->depth + 1;
    if (need <= 32) return launch_wide<LEAF, ANY, COUNT, 32>(b, rays, n, hits, occ, flags, counters, s);
    if (need <= 96) return launch_wide<LEAF, ANY, COUNT, 96>(b, rays, n, hits, occ, flags, counters, s);
    return launch_wide<LEAF, ANY, COUNT, 512>(b, rays, n, hits, occ, flags, counters, s);
}

}  // namespace

// Builds the wide layout of every mesh of a batch from the binary PLOC tree. root_ids[k] = PLOC node id of
// mesh k's root, root_counts[k] its triangle count. Outputs the wide nodes/triangles (in `storage`), each
// mesh's root reference (wide node index or leaf reference), the number of wide levels per mesh, and the
// node count.
dipl_status build_wide(const int4* child, const float4* node_lo, const float4* node_hi, const int* leaf_start_of,
                       const float4* btris, int N, int L, const std::vector<int>& root_ids,
                       const std::vector<int>& root_counts, Storage& storage, cudaStream_t s, uint32_t* d_err,
                       WNode** out_nodes, float4** out_tris, int64_t* out_num_nodes, std::vector<int>& out_root_refs,
                       std::vector<int>& out_levels) {
    const int m = (int)root_ids.size();
    const int K = std::max(N - m, 1);
    ScratchArena scratch(s);
    WNode* nodes;
    float4* tris;
    int *front0, *front1, *kids;
    uint32_t *ninner, *ntris, *totals;
    unsigned char* scan_scratch;
    dipl_status st;
    if ((st = storage.alloc(&nodes, K)) != DIPL_OK || (st = storage.alloc(&tris, 3 * (size_t)std::max(N, 1))) != DIPL_OK ||
        (st = scratch.alloc(&front0, K)) != DIPL_OK || (st = scratch.alloc(&front1, K)) != DIPL_OK ||
        (st = scratch.alloc(&kids, 8 * (size_t)K)) != DIPL_OK || (st = scratch.alloc(&ninner, K)) != DIPL_OK ||
        (st = scratch.alloc(&ntris, K)) != DIPL_OK || (st = scratch.alloc(&totals, 4)) != DIPL_OK ||
        (st = scratch.alloc(&scan_scratch, scan_scratch_bytes(K))) != DIPL_OK)
        return st;
    WideIn W{child, node_lo, node_hi, leaf_start_of, btris, N, L};
    out_root_refs.assign(m, 0);
    out_levels.assign(m, 0);
    // meshes whose root is a leaf: copy their triangles first
    int tri_next = 0;
    std::vector<int> inner_roots;
    for (int k = 0; k < m; ++k) {
        if (root_counts[k] < L) {
            // the binary leaf range of the root: its leaf_start_of entry
            int start = 0;
            DIPL_CUDA(cudaMemcpyAsync(&start, leaf_start_of + root_ids[k], 4, cudaMemcpyDeviceToHost, s));
            DIPL_CUDA(cudaStreamSynchronize(s));
            copy_tris_kernel<<<1, 32, 0, s>>>(btris + 3 * (long long)start, tris + 3 * (long long)tri_next,
                                              root_counts[k]);
            note_launches();
            out_root_refs[k] = make_leaf_ref(tri_next, root_counts[k]);
            tri_next += root_counts[k];
        } else {
            out_root_refs[k] = (int)inner_roots.size();
            inner_roots.push_back(root_ids[k]);
        }
    }
    int n_front = (int)inner_roots.size();
    if (n_front > 0)
        DIPL_CUDA(cudaMemcpyAsync(front0, inner_roots.data(), 4 * n_front, cudaMemcpyHostToDevice, s));
    int base = 0, levels = 0;
    int* fin = front0;
    int* fout = front1;
    while (n_front > 0) {
        const unsigned grid = (unsigned)((n_front + kWideThreads - 1) / kWideThreads);
        wide_collapse_kernel<<<grid, kWideThreads, 0, s>>>(W, fin, n_front, kids, ninner, ntris, d_err);
        note_launches();
        if ((st = exclusive_scan_u32(ninner, ninner, n_front, totals, scan_scratch, s, d_err)) != DIPL_OK) return st;
        if ((st = exclusive_scan_u32(ntris, ntris, n_front, totals + 1, scan_scratch, s, d_err)) != DIPL_OK) return st;
        wide_write_kernel<<<grid, kWideThreads, 0, s>>>(W, fin, n_front, kids, ninner, ntris, base, base + n_front,
                                                        tri_next, nodes, tris, fout, d_err);
        note_launches();
        DIPL_CUDA(cudaGetLastError());
        uint32_t h[3] = {0, 0, 0};
        DIPL_CUDA(cudaMemcpyAsync(h, totals, 8, cudaMemcpyDeviceToHost, s));
        DIPL_CUDA(cudaMemcpyAsync(h + 2, d_err, 4, cudaMemcpyDeviceToHost, s));
        DIPL_CUDA(cudaStreamSynchronize(s));
        if (h[2] != 0u) {
            set_last_error("wide build: device error");
            return (h[2] & kErrTimeout) ? DIPL_ERR_TIMEOUT : DIPL_ERR_INTERNAL;
        }
        base += n_front;
        tri_next += (int)h[1];
        n_front = (int)h[0];
        std::swap(fin, fout);
        ++levels;
        if (base + n_front > K) {
            set_last_error("wide build: node capacity exceeded (internal)");
            return DIPL_ERR_INTERNAL;
        }
    }
    for (int k = 0; k < m; ++k) out_levels[k] = levels;
    *out_nodes = nodes;
    *out_tris = tris;
    *out_num_nodes = base;
    return DIPL_OK;
}

dipl_status trace_wide(const dipl_bvh* b, const dipl_ray* rays, int64_t n, dipl_hit* hits, uint8_t* occ, int leaf_test,
                       uint32_t flags, unsigned long long* counters, bool any, cudaStream_t s) {
    if (any)
        return leaf_test == DIPL_LEAF_REF_MT
                   ? launch_wide_stack<DIPL_LEAF_REF_MT, true, false>(b, rays, n, nullptr, occ, flags, nullptr, s)
                   : launch_wide_stack<DIPL_LEAF_WATERTIGHT, true, false>(b, rays, n, nullptr, occ, flags, nullptr, s);
    if (counters)
        return leaf_test == DIPL_LEAF_REF_MT
                   ? launch_wide_stack<DIPL_LEAF_REF_MT, false, true>(b, rays, n, hits, nullptr, flags, counters, s)
                   : launch_wide_stack<DIPL_LEAF_WATERTIGHT, false, true>(b, rays, n, hits, nullptr, flags, counters, s);
    return leaf_test == DIPL_LEAF_REF_MT
               ? launch_wide_stack<DIPL_LEAF_REF_MT, false, false>(b, rays, n, hits, nullptr, flags, nullptr, s)
               : launch_wide_stack<DIPL_LEAF_WATERTIGHT, false, false>(b, rays, n, hits, nullptr, flags, nullptr, s);
}

}  // namespace dipl
