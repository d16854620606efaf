// BVH build on the device: scene bounds -> Morton30 / EMC60 codes -> LSD radix sort -> PLOC clustering
// (one persistent cooperative launch for every iteration) -> leaf collapse and node layout.
//
// The reference builds top-down on one CPU thread (SBvh::Build, src/acceleration/sbvh.cc:17-58, binned SAH
// in FindBestSplit :193-266, partition in Subdivide :268-341). This is the bottom-up GPU replacement the
// reference plans but does not contain (README.md:156-161; src/gpu/acceleration/ is empty): PLOC after
// Meister & Bittner (2017), codes after Karras (2012) and Vinkler et al. (2017).
//
// Batching: a build of M meshes runs as one pipeline over the concatenation of their triangles. Sort
// keys carry the mesh index above the code, so every mesh is a contiguous run of the sorted order, and
// PLOC never pairs clusters of different meshes; it stops when one cluster per mesh is left.
#include <cooperative_groups.h>

#include <cmath>
#include <cstring>

#include "internal.h"

namespace dipl {

struct MeshDesc {
    const float* v0;
    const float* v1;
    const float* v2;
    long long first;  // first global triangle index
    long long count;
};

// Per-mesh code parameters (computed on the device from the bounds).
struct CodeParams {
    float lo[4];
    float s[4];
    unsigned long long top[4];
    unsigned long long mask[4];
    int bits[4];
    // EMC60: dep[a][c][v] = the bits of nibble v of dimension a's cell index, chunk c (bits 4c..4c+3),
    // deposited at their code positions, so a code is an OR of table entries instead of a bit loop.
    unsigned long long dep[4][16][16];
};

struct PlocCtrl {
    uint32_t n[2];       // cluster count at the start of an iteration (by parity)
    uint32_t merges[2];  // internal nodes created before an iteration (by parity)
    uint32_t iterations;
    uint32_t roots_second;    // 1: the roots are in the second cluster buffer (hierarchical clustering)
    uint32_t tiles_taken[2];  // tiles claimed in an iteration (by parity)
    GridBarrier barrier;
};

namespace {

constexpr int kRadiusMax = 32;
// Positions per thread at most in a ploc_kernel tile: 1024-position tiles at 256 and 512 threads (512 at 128).
__host__ __device__ constexpr int ploc_ipt_max(int B) { return B >= 512 ? 2 : 4; }
constexpr uint32_t kMaxPlocIterations = 1u << 16;

__device__ __forceinline__ int find_mesh(const long long* __restrict__ offsets, int m, long long g) {
    int lo = 0, hi = m - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (offsets[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

struct Tri {
    float3 a, b, c;
};

__device__ __forceinline__ Tri load_tri(const MeshDesc& md, long long local) {
    const float* p0 = md.v0 + 3 * local;
    const float* p1 = md.v1 + 3 * local;
    const float* p2 = md.v2 + 3 * local;
    Tri t;
    t.a = make_float3(__ldg(p0), __ldg(p0 + 1), __ldg(p0 + 2));
    t.b = make_float3(__ldg(p1), __ldg(p1 + 1), __ldg(p1 + 2));
    t.c = make_float3(__ldg(p2), __ldg(p2 + 1), __ldg(p2 + 2));
    return t;
}

// Centroid ((v0 + v1) + v2) / 3, the reference's CalculateTriangleCentroid (src/scene/triangle.h:36).
__device__ __forceinline__ float3 centroid(const Tri& t) {
    return make_float3(__fdiv_rn(__fadd_rn(__fadd_rn(t.a.x, t.b.x), t.c.x), 3.0f),
                       __fdiv_rn(__fadd_rn(__fadd_rn(t.a.y, t.b.y), t.c.y), 3.0f),
                       __fdiv_rn(__fadd_rn(__fadd_rn(t.a.z, t.b.z), t.c.z), 3.0f));
}

// A triangle with a NaN or infinite coordinate can never be hit: both leaf tests then compute t as NaN
// (an infinite edge meets a zero reciprocal or a NaN product). Such a triangle gets an empty box (lo = +inf,
// hi = -inf) and stays out of the scene bounds, so no box above it becomes infinite or NaN.
__device__ __forceinline__ bool tri_finite(const Tri& t) {
    return isfinite(t.a.x) && isfinite(t.a.y) && isfinite(t.a.z) && isfinite(t.b.x) && isfinite(t.b.y) &&
           isfinite(t.b.z) && isfinite(t.c.x) && isfinite(t.c.y) && isfinite(t.c.z);
}

__device__ __forceinline__ void tri_box(const Tri& t, float3& lo, float3& hi) {
    if (!tri_finite(t)) {
        lo = make_float3(__int_as_float(0x7F800000), __int_as_float(0x7F800000), __int_as_float(0x7F800000));
        hi = make_float3(__int_as_float(0xFF800000), __int_as_float(0xFF800000), __int_as_float(0xFF800000));
        return;
    }
    lo = make_float3(fminf(fminf(t.a.x, t.b.x), t.c.x), fminf(fminf(t.a.y, t.b.y), t.c.y),
                     fminf(fminf(t.a.z, t.b.z), t.c.z));
    hi = make_float3(fmaxf(fmaxf(t.a.x, t.b.x), t.c.x), fmaxf(fmaxf(t.a.y, t.b.y), t.c.y),
                     fmaxf(fmaxf(t.a.z, t.b.z), t.c.z));
}

// ------------------------------------------------------------------------------------------------
// Scene bounds: centroid box and vertex box per mesh, as order-preserving ints (atomic min/max).
// ------------------------------------------------------------------------------------------------
struct Bounds {
    int v[12];  // cmin xyz, cmax xyz, bmin xyz, bmax xyz
};

__global__ void bounds_init_kernel(Bounds* b, int m) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    int pinf = float_to_ordered(__int_as_float(0x7F800000)), ninf = float_to_ordered(__int_as_float(0xFF800000));
    for (int a = 0; a < 3; ++a) {
        b[k].v[a] = pinf;
        b[k].v[3 + a] = ninf;
        b[k].v[6 + a] = pinf;
        b[k].v[9 + a] = ninf;
    }
}

__device__ __forceinline__ void flush_bounds(Bounds* b, const float* acc) {
    for (int a = 0; a < 3; ++a) {
        atomicMin(&b->v[a], float_to_ordered(acc[a]));
        atomicMax(&b->v[3 + a], float_to_ordered(acc[3 + a]));
        atomicMin(&b->v[6 + a], float_to_ordered(acc[6 + a]));
        atomicMax(&b->v[9 + a], float_to_ordered(acc[9 + a]));
    }
}

__device__ __forceinline__ void reset_acc(float* acc) {
    for (int a = 0; a < 3; ++a) {
        acc[a] = acc[6 + a] = __int_as_float(0x7F800000);
        acc[3 + a] = acc[9 + a] = __int_as_float(0xFF800000);
    }
}

__global__ void __launch_bounds__(256) bounds_kernel(const MeshDesc* __restrict__ meshes,
                                                     const long long* __restrict__ offsets, int m, long long n,
                                                     long long chunk, Bounds* __restrict__ out) {
    const long long beg = blockIdx.x * chunk, end = min(n, beg + chunk);
    if (beg >= end) return;
    const int m_first = find_mesh(offsets, m, beg), m_last = find_mesh(offsets, m, end - 1);
    float acc[12];
    reset_acc(acc);
    int cur = -1;
    bool any = false;
    for (long long g = beg + threadIdx.x; g < end; g += blockDim.x) {
        int k = (m_first == m_last) ? m_first : find_mesh(offsets, m, g);
        if (k != cur) {
            if (any && m_first != m_last) {
                flush_bounds(&out[cur], acc);
                reset_acc(acc);
            }
            cur = k;
        }
        any = true;
        Tri t = load_tri(meshes[k], g - meshes[k].first);
        if (!tri_finite(t)) continue;  // never hit: left out of the bounds
        float3 c = centroid(t), lo, hi;
        tri_box(t, lo, hi);
        acc[0] = fminf(acc[0], c.x), acc[1] = fminf(acc[1], c.y), acc[2] = fminf(acc[2], c.z);
        acc[3] = fmaxf(acc[3], c.x), acc[4] = fmaxf(acc[4], c.y), acc[5] = fmaxf(acc[5], c.z);
        acc[6] = fminf(acc[6], lo.x), acc[7] = fminf(acc[7], lo.y), acc[8] = fminf(acc[8], lo.z);
        acc[9] = fmaxf(acc[9], hi.x), acc[10] = fmaxf(acc[10], hi.y), acc[11] = fmaxf(acc[11], hi.z);
    }
    if (m_first != m_last) {
        if (any) flush_bounds(&out[cur], acc);
        return;
    }
    // single mesh in this block: warp + block reduction, then 12 atomics
    __shared__ float s_acc[8][12];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        float v = acc[i];
        bool is_min = (i % 6) < 3;
        for (int o = 16; o > 0; o >>= 1) {
            float w = __shfl_xor_sync(0xffffffffu, v, o);
            v = is_min ? fminf(v, w) : fmaxf(v, w);
        }
        if (lane == 0) s_acc[warp][i] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float r[12];
        for (int i = 0; i < 12; ++i) {
            float v = s_acc[0][i];
            bool is_min = (i % 6) < 3;
            for (int w = 1; w < (int)(blockDim.x >> 5); ++w) v = is_min ? fminf(v, s_acc[w][i]) : fmaxf(v, s_acc[w][i]);
            r[i] = v;
        }
        flush_bounds(&out[m_first], r);
    }
}

// ------------------------------------------------------------------------------------------------
// Codes.
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t expand10(uint32_t x) {
    x &= 0x3FFu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

__device__ __forceinline__ unsigned long long deposit_bits(unsigned long long value, unsigned long long mask) {
    unsigned long long out = 0;
    while (mask) {
        unsigned long long low = mask & (~mask + 1ull);
        if (value & 1ull) out |= low;
        value >>= 1;
        mask &= mask - 1ull;
    }
    return out;
}

// One thread per mesh: Morton30 scales, or the EMC60 bit plan (60 positions MSB first, each to the
// dimension x, y, z, size with the largest remaining extent, which is then halved).
__global__ void code_params_kernel(const Bounds* __restrict__ bounds, int m, int code_type, CodeParams* out) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    float cmin[3], cmax[3], bmin[3], bmax[3];
    for (int a = 0; a < 3; ++a) {
        cmin[a] = ordered_to_float(bounds[k].v[a]);
        cmax[a] = ordered_to_float(bounds[k].v[3 + a]);
        bmin[a] = ordered_to_float(bounds[k].v[6 + a]);
        bmax[a] = ordered_to_float(bounds[k].v[9 + a]);
    }
    CodeParams p;  // scalar fields only; the deposit tables are written to out[k] directly
    if (code_type == DIPL_CODE_MORTON30) {
        for (int a = 0; a < 3; ++a) {
            float ext = __fsub_rn(cmax[a], cmin[a]);
            p.lo[a] = cmin[a];
            p.s[a] = ext > 0.0f ? __fdiv_rn(1024.0f, ext) : 0.0f;
            p.bits[a] = 10;
            p.top[a] = 1023;
            p.mask[a] = 0;
        }
        p.lo[3] = 0.0f, p.s[3] = 0.0f, p.bits[3] = 0, p.top[3] = 0, p.mask[3] = 0;
    } else {
        float dx = __fsub_rn(bmax[0], bmin[0]), dy = __fsub_rn(bmax[1], bmin[1]), dz = __fsub_rn(bmax[2], bmin[2]);
        float diag = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
        float ext[4] = {__fsub_rn(cmax[0], cmin[0]), __fsub_rn(cmax[1], cmin[1]), __fsub_rn(cmax[2], cmin[2]), diag};
        float e[4];
        for (int a = 0; a < 4; ++a) {
            e[a] = ext[a] > 0.0f ? ext[a] : 0.0f;
            p.bits[a] = 0;
            p.mask[a] = 0;
        }
        for (int pos = 59; pos >= 0; --pos) {
            int best = 0;
            for (int a = 1; a < 4; ++a)
                if (e[a] > e[best]) best = a;
            p.bits[best] += 1;
            p.mask[best] |= 1ull << pos;
            e[best] = __fmul_rn(e[best], 0.5f);
        }
        for (int a = 0; a < 4; ++a) {
            float cells = ldexpf(1.0f, p.bits[a]);
            p.lo[a] = a < 3 ? cmin[a] : 0.0f;
            p.s[a] = (ext[a] > 0.0f && p.bits[a] > 0) ? __fdiv_rn(cells, ext[a]) : 0.0f;
            p.top[a] = p.bits[a] >= 64 ? ~0ull : ((1ull << p.bits[a]) - 1ull);
        }
    }
    for (int a = 0; a < 4; ++a) {
        out[k].lo[a] = p.lo[a];
        out[k].s[a] = p.s[a];
        out[k].top[a] = p.top[a];
        out[k].mask[a] = p.mask[a];
        out[k].bits[a] = p.bits[a];
    }
}

// EMC60 deposit tables of every mesh: one block per mesh, one thread per (dimension, chunk, nibble) entry.
__global__ void __launch_bounds__(256) emc_tables_kernel(CodeParams* params) {
    CodeParams& p = params[blockIdx.x];
    for (int e = threadIdx.x; e < 4 * 16 * 16; e += blockDim.x) {
        const int a = e >> 8, c = (e >> 4) & 15, v = e & 15;
        p.dep[a][c][v] = deposit_bits((unsigned long long)v << (4 * c), p.mask[a]);
    }
}

// The code of a point c with a size given by box extents (dx, dy, dz): Morton30 uses c, EMC60 also the box diagonal.
__device__ __forceinline__ unsigned long long point_code(float3 c, float dx, float dy, float dz, const CodeParams& p,
                                                         int code_type) {
    if (code_type == DIPL_CODE_MORTON30) {
        float xs[3] = {c.x, c.y, c.z};
        uint32_t q[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            float x = __fmul_rn(__fsub_rn(xs[a], p.lo[a]), p.s[a]);
            x = fminf(fmaxf(x, 0.0f), 1023.0f);
            q[a] = (uint32_t)x;
        }
        return (expand10(q[0]) << 2) | (expand10(q[1]) << 1) | expand10(q[2]);
    }
    float xs[4] = {c.x, c.y, c.z,
                   __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)))};
    unsigned long long code = 0;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        if (p.bits[a] == 0) continue;
        float q = fmaxf(__fmul_rn(__fsub_rn(xs[a], p.lo[a]), p.s[a]), 0.0f);
        unsigned long long qi = q < 1.8e19f ? (unsigned long long)q : p.top[a];
        if (qi > p.top[a]) qi = p.top[a];
        const int chunks = (p.bits[a] + 3) >> 2;
        for (int c = 0; c < chunks; ++c) code |= p.dep[a][c][(qi >> (4 * c)) & 15ull];
    }
    return code;
}

// A triangle's code: its centroid (the reference's, triangle.h:36) and, for EMC60, its box diagonal.
__device__ __forceinline__ unsigned long long tri_code(const Tri& t, const CodeParams& p, int code_type) {
    const float dx = __fsub_rn(fmaxf(fmaxf(t.a.x, t.b.x), t.c.x), fminf(fminf(t.a.x, t.b.x), t.c.x));
    const float dy = __fsub_rn(fmaxf(fmaxf(t.a.y, t.b.y), t.c.y), fminf(fminf(t.a.y, t.b.y), t.c.y));
    const float dz = __fsub_rn(fmaxf(fmaxf(t.a.z, t.b.z), t.c.z), fminf(fminf(t.a.z, t.b.z), t.c.z));
    return point_code(centroid(t), dx, dy, dz, p, code_type);
}

template <typename K>
__global__ void __launch_bounds__(256) codes_kernel(const MeshDesc* __restrict__ meshes,
                                                    const long long* __restrict__ offsets, int m, long long n,
                                                    const CodeParams* __restrict__ params, int code_type,
                                                    int code_shift, int mesh_shift, K* __restrict__ keys,
                                                    float4* __restrict__ tbox) {
    long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (g >= n) return;
    int k = find_mesh(offsets, m, g);
    const MeshDesc md = meshes[k];
    Tri t = load_tri(md, g - md.first);
    unsigned long long code = tri_code(t, params[k], code_type) >> code_shift;
    if (mesh_shift > 0) code |= (unsigned long long)k << mesh_shift;
    keys[g] = static_cast<K>(code);
    if (tbox) {  // one 32-byte record per triangle: later gathers by sorted position read one sector
        float3 lo, hi;
        tri_box(t, lo, hi);
        tbox[2 * g] = make_float4(lo.x, lo.y, lo.z, 0.0f);
        tbox[2 * g + 1] = make_float4(hi.x, hi.y, hi.z, 0.0f);
    }
}

// ------------------------------------------------------------------------------------------------
// Pre-splitting of large triangles (early split clipping, after Ernst & Greiner 2007 and the pre-splitting of
// Karras & Aila 2013): a triangle whose box is large compared with its mesh's other triangles enters the
// clustering as several references, each with the box of the part of the triangle inside one half of its box
// (recursively halved at the longest axis' midpoint). Leaves still hold the whole triangle, so a ray tests the
// same triangles with the same arithmetic and gets the same closest hit; it only meets far fewer boxes that
// are mostly empty (a log-normal soup's large triangles cover every point of the cube many times over).
//
// Split counts are deterministic: w = (dx dy + dy dz) + dz dx of the triangle's box in FP32, quantised to an
// integer q = floor(w 2^32 / D^2) (D = the mesh's vertex-box diagonal) so the per-mesh sum Q is exact; the
// triangle gets s = floor(q budget N / (100 Q)) splits (FP64, one rounding per operation), at most
// kMaxPieces - 1, and s + 1 references. Every reference of a split triangle codes by its box centre and box
// diagonal; an unsplit triangle codes exactly as without splitting. oracle/dipl_oracle.c orc_presplit restates
// this bit for bit.
// ------------------------------------------------------------------------------------------------
constexpr int kMaxPieces = 64;

__device__ __forceinline__ unsigned long long split_weight(const Tri& t, float diag) {
    if (!tri_finite(t) || !(diag > 0.0f)) return 0ull;
    float3 lo, hi;
    tri_box(t, lo, hi);
    const float dx = __fsub_rn(hi.x, lo.x), dy = __fsub_rn(hi.y, lo.y), dz = __fsub_rn(hi.z, lo.z);
    const float w = __fadd_rn(__fadd_rn(__fmul_rn(dx, dy), __fmul_rn(dy, dz)), __fmul_rn(dz, dx));
    const double scale = __ddiv_rn(4294967296.0, __dmul_rn((double)diag, (double)diag));
    const double q = __dmul_rn((double)w, scale);
    return q < 1.8e19 ? (unsigned long long)q : 18000000000000000000ull;
}

__device__ __forceinline__ float mesh_diag(const Bounds& b) {
    float e[3];
    for (int a = 0; a < 3; ++a) e[a] = __fsub_rn(ordered_to_float(b.v[9 + a]), ordered_to_float(b.v[6 + a]));
    return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(e[0], e[0]), __fmul_rn(e[1], e[1])), __fmul_rn(e[2], e[2])));
}

__global__ void __launch_bounds__(256) split_weight_kernel(const MeshDesc* __restrict__ meshes,
                                                           const long long* __restrict__ offsets, int m, long long n,
                                                           const Bounds* __restrict__ bounds,
                                                           unsigned long long* __restrict__ mesh_sum) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    unsigned long long q = 0ull;
    int k = 0;
    if (g < n) {
        k = find_mesh(offsets, m, g);
        q = split_weight(load_tri(meshes[k], g - meshes[k].first), mesh_diag(bounds[k]));
    }
    // integer sums are exact in any order: one atomic per warp when the warp lies in one mesh, else one per thread
    const int k0 = __shfl_sync(0xffffffffu, k, 0);
    if (__all_sync(0xffffffffu, k == k0)) {
        for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
        if ((threadIdx.x & 31) == 0 && q) atomicAdd(mesh_sum + k0, q);
    } else if (q) {
        atomicAdd(mesh_sum + k, q);
    }
}

__device__ __forceinline__ uint32_t split_pieces(unsigned long long q, unsigned long long sum, long long mesh_tris,
                                                 int budget) {
    if (sum == 0ull || q == 0ull) return 1u;
    const double num = __dmul_rn(__dmul_rn((double)q, (double)budget), (double)mesh_tris);
    const double den = __dmul_rn(100.0, (double)sum);
    const double s = floor(__ddiv_rn(num, den));
    return 1u + (uint32_t)fmin(s, (double)(kMaxPieces - 1));
}

__global__ void __launch_bounds__(256) split_count_kernel(const MeshDesc* __restrict__ meshes,
                                                          const long long* __restrict__ offsets, int m, long long n,
                                                          const Bounds* __restrict__ bounds,
                                                          const unsigned long long* __restrict__ mesh_sum, int budget,
                                                          uint32_t* __restrict__ pieces) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (g >= n) return;
    const int k = find_mesh(offsets, m, g);
    const unsigned long long q = split_weight(load_tri(meshes[k], g - meshes[k].first), mesh_diag(bounds[k]));
    pieces[g] = split_pieces(q, mesh_sum[k], meshes[k].count, budget);
}

// First reference of every mesh (cluster positions of the meshes) from the exclusive scan of the piece counts.
__global__ void mesh_ref_offsets_kernel(const long long* __restrict__ offsets, int m, const uint32_t* __restrict__ first,
                                        const uint32_t* __restrict__ total, long long* __restrict__ coffsets) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m) coffsets[k] = first[offsets[k]];
    if (k == m) coffsets[m] = *total;
}

__device__ __forceinline__ float axis_of(const float3& v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }
__device__ __forceinline__ void set_axis(float3& v, int a, float x) {
    if (a == 0) v.x = x;
    else if (a == 1) v.y = x;
    else v.z = x;
}

constexpr int kSplitThreads = 128;
constexpr int kPolyMax = 9;  // a triangle clipped by at most 6 planes

// A piece's polygon in shared memory, one column per thread (vertex v, coordinate c of thread j at
// [(v * 3 + c) * kSplitThreads + j]: a warp's accesses never share a bank).
struct Poly {
    float* s;
    __device__ __forceinline__ float& at(int v, int c) const { return s[(v * 3 + c) * kSplitThreads]; }
};

// One halving of a piece (early split clipping): the piece is the part of the triangle inside its box [lo, hi],
// kept as a polygon P of np vertices (the triangle clipped by the planes of the halvings so far). The plane
// x_a = mid cuts it; the lower (x_a <= mid) or upper half's polygon Q is P clipped by that plane
// (Sutherland-Hodgman: vertices on the plane are inside, a crossing point takes mid exactly on axis a), and its box
// is Q's box intersected with the half of [lo, hi]. An empty Q or box (only rounding can make one) gives the half
// itself, which is conservative. Returns Q's vertex count.
__device__ __forceinline__ int split_half(const Poly& P, int np, const Poly& Q, int a, float mid, bool lower,
                                          float3& lo, float3& hi) {
    const float inf = __int_as_float(0x7F800000);
    float3 bl = make_float3(inf, inf, inf), bh = make_float3(-inf, -inf, -inf);
    int nq = 0;
    for (int i = 0; i < np; ++i) {
        const int j = i + 1 < np ? i + 1 : 0;
        const float3 p = make_float3(P.at(i, 0), P.at(i, 1), P.at(i, 2));
        const float3 q = make_float3(P.at(j, 0), P.at(j, 1), P.at(j, 2));
        const float pa = axis_of(p, a), qa = axis_of(q, a);
        const bool ip = lower ? pa <= mid : pa >= mid, iq = lower ? qa <= mid : qa >= mid;
        if (ip && nq < kPolyMax) {
            Q.at(nq, 0) = p.x, Q.at(nq, 1) = p.y, Q.at(nq, 2) = p.z, ++nq;
            bl = make_float3(fminf(bl.x, p.x), fminf(bl.y, p.y), fminf(bl.z, p.z));
            bh = make_float3(fmaxf(bh.x, p.x), fmaxf(bh.y, p.y), fmaxf(bh.z, p.z));
        }
        if (ip != iq && nq < kPolyMax) {
            const float sc = __fdiv_rn(__fsub_rn(mid, pa), __fsub_rn(qa, pa));
            float3 x = make_float3(__fadd_rn(p.x, __fmul_rn(sc, __fsub_rn(q.x, p.x))),
                                   __fadd_rn(p.y, __fmul_rn(sc, __fsub_rn(q.y, p.y))),
                                   __fadd_rn(p.z, __fmul_rn(sc, __fsub_rn(q.z, p.z))));
            set_axis(x, a, mid);
            Q.at(nq, 0) = x.x, Q.at(nq, 1) = x.y, Q.at(nq, 2) = x.z, ++nq;
            bl = make_float3(fminf(bl.x, x.x), fminf(bl.y, x.y), fminf(bl.z, x.z));
            bh = make_float3(fmaxf(bh.x, x.x), fmaxf(bh.y, x.y), fmaxf(bh.z, x.z));
        }
    }
    if (lower) set_axis(hi, a, mid);
    else set_axis(lo, a, mid);
    const float3 nl = make_float3(fmaxf(bl.x, lo.x), fmaxf(bl.y, lo.y), fmaxf(bl.z, lo.z));
    const float3 nh = make_float3(fminf(bh.x, hi.x), fminf(bh.y, hi.y), fminf(bh.z, hi.z));
    if (nq > 0 && nl.x <= nh.x && nl.y <= nh.y && nl.z <= nh.z) lo = nl, hi = nh;
    return nq;
}

// The triangle of every reference: triangle g owns the pieces[g] references from its scanned position first[g].
__global__ void __launch_bounds__(256) ref_tri_kernel(long long n, const uint32_t* __restrict__ pieces,
                                                      const uint32_t* __restrict__ first, int* __restrict__ ref_tri) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (g >= n) return;
    const uint32_t c = pieces[g];
    const long long r = first[g];
    for (uint32_t i = 0; i < c; ++i) ref_tri[r + i] = (int)g;
}

// One thread per reference: its box and its code. An unsplit triangle's reference takes the triangle's box and
// codes exactly as codes_kernel; piece j of a triangle split into c pieces follows its own path of halvings from
// the triangle's box: a box of c pieces is cut at the midpoint of its longest axis, the lower half takes the
// first ceil(c/2) pieces and the upper half the rest, and each half's box comes from split_half. The
// pieces of one triangle are the leaves of that binary recursion in depth-first order (lower half first), and
// every box is computed with the same operations whichever thread computes it. A piece codes by the centre and
// the diagonal of its box.
template <typename K>
__global__ void __launch_bounds__(kSplitThreads) split_refs_kernel(const MeshDesc* __restrict__ meshes,
                                                                   const long long* __restrict__ offsets, int m,
                                                                   long long n_refs, const int* __restrict__ ref_tri,
                                                                   const uint32_t* __restrict__ pieces,
                                                                   const uint32_t* __restrict__ first,
                                                                   const CodeParams* __restrict__ params,
                                                                   int code_type, int code_shift, int mesh_shift,
                                                                   float4* __restrict__ rbox, K* __restrict__ keys) {
    __shared__ float s_poly[2 * kPolyMax * 3 * kSplitThreads];
    const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (r >= n_refs) return;
    const long long g = ref_tri[r];
    const int k = find_mesh(offsets, m, g);
    const Tri t = load_tri(meshes[k], g - meshes[k].first);
    int c = (int)pieces[g];
    float3 blo, bhi;
    tri_box(t, blo, bhi);
    unsigned long long code;
    if (c == 1) {
        code = tri_code(t, params[k], code_type);
    } else {
        Poly P{s_poly + threadIdx.x}, Q{s_poly + kPolyMax * 3 * kSplitThreads + threadIdx.x};
        P.at(0, 0) = t.a.x, P.at(0, 1) = t.a.y, P.at(0, 2) = t.a.z;
        P.at(1, 0) = t.b.x, P.at(1, 1) = t.b.y, P.at(1, 2) = t.b.z;
        P.at(2, 0) = t.c.x, P.at(2, 1) = t.c.y, P.at(2, 2) = t.c.z;
        int np = 3;
        int j = (int)(r - (long long)first[g]);
        for (int depth = 0; depth < 8 && c > 1; ++depth) {  // c <= kMaxPieces: at most 6 halvings
            const float e0 = __fsub_rn(bhi.x, blo.x), e1 = __fsub_rn(bhi.y, blo.y), e2 = __fsub_rn(bhi.z, blo.z);
            const int a = (e0 >= e1 && e0 >= e2) ? 0 : (e1 >= e2 ? 1 : 2);
            const float la = axis_of(blo, a);
            const float mid = __fadd_rn(la, __fmul_rn(__fsub_rn(axis_of(bhi, a), la), 0.5f));
            const int lower = (c + 1) / 2;
            const bool in_lower = j < lower;
            if (in_lower) {
                c = lower;
            } else {
                j -= lower;
                c -= lower;
            }
            np = split_half(P, np, Q, a, mid, in_lower, blo, bhi);
            const Poly tmp = P;
            P = Q;
            Q = tmp;
        }
        const float3 ctr = make_float3(__fmul_rn(__fadd_rn(blo.x, bhi.x), 0.5f), __fmul_rn(__fadd_rn(blo.y, bhi.y), 0.5f),
                                       __fmul_rn(__fadd_rn(blo.z, bhi.z), 0.5f));
        code = point_code(ctr, __fsub_rn(bhi.x, blo.x), __fsub_rn(bhi.y, blo.y), __fsub_rn(bhi.z, blo.z), params[k],
                          code_type);
    }
    rbox[2 * r] = make_float4(blo.x, blo.y, blo.z, 0.0f);
    rbox[2 * r + 1] = make_float4(bhi.x, bhi.y, bhi.z, 0.0f);
    code >>= code_shift;
    if (mesh_shift > 0) code |= (unsigned long long)k << mesh_shift;
    keys[r] = static_cast<K>(code);
}

// ------------------------------------------------------------------------------------------------
// PLOC.
//
// Clusters live in two ping-pong buffers of float4 pairs: lo = (min xyz, node id bits),
// hi = (max xyz, mesh index bits). Internal node k (creation order) stores children (left, right,
// height, 0), lo = (min xyz, triangle count bits), hi = (max xyz, first sorted position bits); node id
// of internal node k is num_leaves + k; parent[] maps every node id to its parent (-1 at roots).
//
// Nearest neighbour of cluster i: argmin over j in [i-r, i+r], j != i, same mesh, of the 64-bit key
// (distance bits << 32) | (|i-j| << 2) | ((min(i,j) & 1) << 1) | (j > i). The key order restricts one
// strict total order on unordered pairs (distance, gap, parity of the lower index, lower index), so a
// mutual pair always exists while a mesh has two clusters, ties are deterministic, and runs of equal
// distances (duplicate geometry) still pair up neighbour with neighbour instead of chaining.
// ------------------------------------------------------------------------------------------------
struct PlocParams {
    float4* lo[2];   // clusters by iteration parity: min xyz, node id bits
    float4* hi[2];   //                              max xyz, mesh index bits
    int4* info[2];   //                              triangle count, first sorted position, height, 0
    int4* child;     // internal node k: left, right, height, 0
    float4* node_lo; // internal node k: min xyz, triangle count bits
    float4* node_hi; // internal node k: max xyz, first sorted position bits
    int* parent;
    unsigned long long* status[2];
    PlocCtrl* ctrl;
    uint32_t* err;
    int num_leaves;
    int num_meshes;
    int radius;
    int grid_stop;  // ploc_kernel runs while more clusters than this remain (the middle phase's capacity, or kTailMax)
    uint32_t max_iterations;  // the build gives up (kErrIterations) at this many iterations
};

// Parity-selected pointers of PlocParams (a select, so the parameter block is never copied to the stack for
// a run-time array index).
template <typename T>
__device__ __forceinline__ T by_parity(T const (&a)[2], int parity) {
    return parity ? a[1] : a[0];
}
template <typename T>
__device__ __forceinline__ T& parity_slot(T (&a)[2], int parity) {
    return parity ? a[1] : a[0];
}

// Clusters at most this many are finished by the single-CTA tail kernel, resident in shared memory.
constexpr int kTailMax = 2048;
constexpr int kTailThreads = 1024;
// At most this many clusters: CTA 0 finishes alone (no cluster exchange per iteration). Below this size a
// search over all positions costs less than one cluster barrier plus the exchange of the slices.
constexpr int kTailSolo = 128;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// Nearest neighbour of every position in [q0, q1) among clusters stored at smem index (position - base).
// Candidates are visited in the order of the key's tie fields (gap, then parity of the lower index,
// then side), so a strict "<" on the distance alone yields the minimum of the oracle's 64-bit key.
template <int NT>
__device__ __forceinline__ void nn_search(const float4* __restrict__ slo, const float4* __restrict__ shi, int base,
                                          int n, int q0, int q1, int r, int* __restrict__ nn, int nn_base) {
    for (int q = q0 + (int)threadIdx.x; q < q1; q += NT) {
        const float4 a = slo[q - base], b = shi[q - base];
        const int sg = __float_as_int(b.w);
        float bestd = __int_as_float(0x7F800000);
        int bestj = -1;
        auto consider = [&](int j) {
            if (j < 0 || j >= n) return;
            const float4 c = slo[j - base], e = shi[j - base];
            if (__float_as_int(e.w) != sg) return;
            const float d = ploc_distance(a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z, e.x, e.y, e.z);
            if (d < bestd || bestj < 0) {
                bestd = d;
                bestj = j;
            }
        };
#pragma unroll 4
        for (int k = 1; k <= r; ++k) {
            // gap k: lower index q-k (backward) or q (forward); an even lower index wins, then backward.
            const bool fwd_first = (k & 1) && !(q & 1);
            consider(fwd_first ? q + k : q - k);
            consider(fwd_first ? q - k : q + k);
        }
        nn[q - nn_base] = bestj;
    }
}

// Symmetric variant for the grid tiles: each pair (p, p+k) is evaluated once by the thread of its lower
// position; the lower side keeps its running minimum in registers, the upper side receives its key by a
// 64-bit shared-memory atomicMin. Keys are the oracle's (distance bits << 32 | gap << 2 | parity << 1 | side);
// positions [q0, q1) get their nearest neighbour in nn[q - q0]; key is scratch of the same extent.
template <int NT>
__device__ __forceinline__ void nn_search_sym(const float4* __restrict__ slo, const float4* __restrict__ shi, int base,
                                              int n, int q0, int q1, int r, int* __restrict__ nn,
                                              unsigned long long* __restrict__ key) {
    for (int q = q0 + (int)threadIdx.x; q < q1; q += NT) key[q - q0] = ~0ull;
    __syncthreads();
    const int p0 = max(q0 - r, 0);
    for (int p = p0 + (int)threadIdx.x; p < q1; p += NT) {
        const float4 a = slo[p - base], b = shi[p - base];
        const int sg = __float_as_int(b.w);
        const bool own = p >= q0;
        const unsigned long long par = (unsigned long long)((p & 1) << 1);
        unsigned long long best = ~0ull;
        const int kmax = min(r, n - 1 - p);
#pragma unroll 4
        for (int k = 1; k <= kmax; ++k) {
            const int j = p + k;
            const float4 c = slo[j - base], e = shi[j - base];
            if (__float_as_int(e.w) != sg) continue;
            const float d = ploc_distance(a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z, e.x, e.y, e.z);
            const unsigned long long kd = ((unsigned long long)__float_as_uint(d) << 32) |
                                          ((unsigned long long)k << 2) | par;
            const unsigned long long kp = kd | 1ull;  // seen from p: partner above (side 1)
            best = kp < best ? kp : best;
            if (j >= q0 && j < q1) atomicMin(&key[j - q0], kd);  // seen from j: partner below (side 0)
        }
        if (own && best != ~0ull) atomicMin(&key[p - q0], best);
    }
    __syncthreads();
    for (int q = q0 + (int)threadIdx.x; q < q1; q += NT) {
        const unsigned long long kq = key[q - q0];
        int j = -1;
        if (kq != ~0ull) {
            const unsigned tie = (unsigned)kq;
            const int gap = (int)(tie >> 2);
            j = (tie & 1u) ? q + gap : q - gap;
        }
        nn[q - q0] = j;
    }
}

// Tail variant: every position's candidates are split over P consecutive threads (P a power of two, up to
// 16) when there are few clusters, then the per-thread minima are combined with a 64-bit min over the
// oracle's key (distance bits << 32 | gap << 2 | parity << 1 | side). Each thread visits its own gaps in
// increasing order, so its local strict-"<" minimum is its subset's key minimum.
template <int NT>
// slo / shi hold positions [wbase, ...) and nn receives positions [nbase, ...) (both 0 when the whole set is
// resident).
__device__ __forceinline__ void nn_search_split(const float4* __restrict__ slo, const float4* __restrict__ shi, int n,
                                                int q0, int q1, int r, int* __restrict__ nn, int wbase = 0,
                                                int nbase = 0) {
    const int m = q1 - q0;
    int P = 1;
    while (P < 16 && 2 * P * m <= NT) P *= 2;
    const int sub = (int)threadIdx.x & (P - 1);
    const int lanes = NT / P;
    const int rounds = (m + lanes - 1) / lanes;
    for (int rd = 0; rd < rounds; ++rd) {
        const int q = q0 + (int)threadIdx.x / P + rd * lanes;
        // a warp covers 32 / P consecutive positions: warps past the last one have nothing to do
        if (q0 + (int)(threadIdx.x & ~31u) / P + rd * lanes >= q1) break;
        unsigned long long key = ~0ull;
        if (q < q1) {
            const float4 a = slo[q - wbase], b = shi[q - wbase];
            const int sg = __float_as_int(b.w);
            float bestd = __int_as_float(0x7F800000);
            int bestj = -1;
            auto consider = [&](int j) {
                if (j < 0 || j >= n) return;
                const float4 c = slo[j - wbase], e = shi[j - wbase];
                if (__float_as_int(e.w) != sg) return;
                const float d = ploc_distance(a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z, e.x, e.y, e.z);
                if (d < bestd || bestj < 0) {
                    bestd = d;
                    bestj = j;
                }
            };
            for (int k = 1 + sub; k <= r; k += P) {
                const bool fwd_first = (k & 1) && !(q & 1);
                consider(fwd_first ? q + k : q - k);
                consider(fwd_first ? q - k : q + k);
            }
            if (bestj >= 0) {
                const unsigned gap = (unsigned)abs(bestj - q);
                const unsigned mn = (unsigned)min(bestj, q);
                key = ((unsigned long long)__float_as_uint(bestd) << 32) |
                      (unsigned long long)((gap << 2) | ((mn & 1u) << 1) | (bestj > q ? 1u : 0u));
            }
        }
        for (int o = P / 2; o > 0; o >>= 1) {
            const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
            key = other < key ? other : key;
        }
        if (q < q1 && sub == 0) {
            int j = -1;
            if (key != ~0ull) {
                const unsigned tie = (unsigned)key;
                const int gap = (int)(tie >> 2);
                j = (tie & 1u) ? q + gap : q - gap;
            }
            nn[q - nbase] = j;
        }
    }
}

// Writes internal node `knew` = merge of clusters (la, lb, li) and (ra, rb, ri); returns the merged cluster.
__device__ __forceinline__ void emit_node(const PlocParams& P, int knew, const float4& la, const float4& lb,
                                          const int4& li, const float4& ra, const float4& rb, const int4& ri,
                                          float4& oa, float4& ob, int4& oi) {
    const int left = __float_as_int(la.w), right = __float_as_int(ra.w);
    const int node = P.num_leaves + knew;
    oa = make_float4(fminf(la.x, ra.x), fminf(la.y, ra.y), fminf(la.z, ra.z), __int_as_float(node));
    ob = make_float4(fmaxf(lb.x, rb.x), fmaxf(lb.y, rb.y), fmaxf(lb.z, rb.z), lb.w);
    oi = make_int4(li.x + ri.x, min(li.y, ri.y), max(li.z, ri.z) + 1, 0);
    P.child[knew] = make_int4(left, right, oi.z, 0);
    P.node_lo[knew] = make_float4(oa.x, oa.y, oa.z, __int_as_float(oi.x));
    P.node_hi[knew] = make_float4(ob.x, ob.y, ob.z, __int_as_float(oi.y));
    P.parent[left] = node;
    P.parent[right] = node;
}

template <int B>
struct PlocSmem {
    static constexpr int T = B * ploc_ipt_max(B);
    static constexpr int W = T + 4 * kRadiusMax;
    float4 lo[W];  // min xyz, node id bits
    float4 hi[W];  // max xyz, mesh index bits
    int4 info[W];  // count, first position, height
    int nn[T + 2 * kRadiusMax];
    unsigned long long key[T + 2 * kRadiusMax];
    uint32_t warp_sum[B / 32];
    unsigned long long lb_sum[B / 32];  // block look-back scratch
    int lb_flag[B / 32];
    unsigned long long prefix;
    int ok;
    int n, mbase;
    uint32_t claim;
};

template <int B>
__device__ void ploc_tile(const PlocParams& P, PlocSmem<B>& s, int tile, int tiles, int n, int mbase, int parity,
                          int ipt) {
    const int T = B * ipt;  // positions of this tile (ipt <= ploc_ipt_max(B))
    const int r = P.radius;
    const int s0 = tile * T;
    const int w0 = max(s0 - 2 * r, 0), w1 = min(s0 + T + 2 * r, n);
    // window: asynchronous 16-byte copies, all in flight at once (one memory round trip)
    for (int i = threadIdx.x; i < w1 - w0; i += B) {
        cp_async16(&s.lo[i], by_parity(P.lo, parity) + w0 + i);
        cp_async16(&s.hi[i], by_parity(P.hi, parity) + w0 + i);
        cp_async16(&s.info[i], by_parity(P.info, parity) + w0 + i);
    }
    cp_async_wait_all();
    __syncthreads();

    const int q0 = max(s0 - r, 0), q1 = min(s0 + T + r, n);
    nn_search_sym<B>(s.lo, s.hi, w0, n, q0, q1, r, s.nn, s.key);
    __syncthreads();

    // ---- merge decisions (blocked: ipt consecutive positions per thread) ---------------------------
    const int ib = s0 + threadIdx.x * ipt;
    uint32_t keep_bits = 0, merge_bits = 0;
#pragma unroll
    for (int k = 0; k < ploc_ipt_max(B); ++k) {
        int i = ib + k;
        if (k >= ipt || i >= n) break;
        int j = s.nn[i - q0];
        bool mutual = j >= 0 && s.nn[j - q0] == i;
        if (!(mutual && i > j)) keep_bits |= 1u << k;
        if (mutual && i < j) merge_bits |= 1u << k;
    }
    const uint32_t mine = (uint32_t)__popc(keep_bits) | ((uint32_t)__popc(merge_bits) << 16);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s.warp_sum[warp] = x;
    __syncthreads();
    uint32_t woff = 0, total = 0;
#pragma unroll
    for (int w = 0; w < B / 32; ++w) {
        uint32_t v = s.warp_sum[w];
        if (w < warp) woff += v;
        total += v;
    }
    const uint32_t excl = woff + x - mine;

    // ---- decoupled look-back over tiles: (kept, merged) prefixes (whole block) ----------------------
    {
        const unsigned long long agg = ((unsigned long long)(total & 0xFFFFu) << 31) | (total >> 16);
        unsigned long long* st = by_parity(P.status, parity);
        unsigned long long prefix = 0;
        bool ok = true;
        if (tile == 0) {  // block-uniform
            if (threadIdx.x == 0) st_release_u64(&st[0], (2ull << 62) | agg);
        } else {
            if (threadIdx.x == 0) st_release_u64(&st[tile], (1ull << 62) | agg);
            prefix = block_lookback<B>(st, tile, P.err, &ok, s.lb_sum, s.lb_flag);
            if (threadIdx.x == 0 && ok) st_release_u64(&st[tile], (2ull << 62) | (prefix + agg));
        }
        if (threadIdx.x == 0) {
            s.prefix = prefix;
            s.ok = ok ? 1 : 0;
            if (tile == tiles - 1 && ok) {
                unsigned long long inc = prefix + agg;
                P.ctrl->n[parity ^ 1] = (uint32_t)(inc >> 31);
                P.ctrl->merges[parity ^ 1] = (uint32_t)mbase + (uint32_t)(inc & 0x7FFFFFFFull);
            }
        }
    }
    __syncthreads();
    if (!s.ok) return;
    const uint32_t kept_before = (uint32_t)(s.prefix >> 31);
    const uint32_t merged_before = (uint32_t)(s.prefix & 0x7FFFFFFFull);

    // ---- write surviving clusters and new nodes ----------------------------------------------------
    float4* __restrict__ out_lo = by_parity(P.lo, parity ^ 1);
    float4* __restrict__ out_hi = by_parity(P.hi, parity ^ 1);
    int4* __restrict__ out_info = by_parity(P.info, parity ^ 1);
    uint32_t kpos = kept_before + (excl & 0xFFFFu);
    uint32_t mpos = (uint32_t)mbase + merged_before + (excl >> 16);
    const int max_internal = P.num_leaves - P.num_meshes;
#pragma unroll
    for (int k = 0; k < ploc_ipt_max(B); ++k) {
        if (!((keep_bits >> k) & 1u)) continue;  // also 0 for k >= ipt
        const int i = ib + k, ii = i - w0;
        float4 oa = s.lo[ii], ob = s.hi[ii];
        int4 oi = s.info[ii];
        if ((merge_bits >> k) & 1u) {
            const int ji = s.nn[i - q0] - w0;
            const int knew = (int)mpos++;
            if (knew >= max_internal) {
                atomicOr(P.err, kErrIterations);
                continue;
            }
            emit_node(P, knew, s.lo[ii], s.hi[ii], s.info[ii], s.lo[ji], s.hi[ji], s.info[ji], oa, ob, oi);
        }
        if (kpos < (uint32_t)P.num_leaves) {
            out_lo[kpos] = oa;
            out_hi[kpos] = ob;
            out_info[kpos] = oi;
        }
        ++kpos;
    }
}

// Every PLOC iteration while more than P.grid_stop clusters remain, in one cooperative launch. Iterations are
// separated by a grid barrier over the blocks that still have tiles.
template <int B>
__global__ void __launch_bounds__(B) ploc_kernel(PlocParams P) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    PlocSmem<B>& s = *reinterpret_cast<PlocSmem<B>*>(s_raw);
    uint32_t iter = 0;
    int active_prev = (int)gridDim.x;
    for (;;) {
        const int parity = iter & 1;
        if (threadIdx.x == 0) {
            s.n = (int)ld_acquire_u32(&P.ctrl->n[parity]);
            s.mbase = (int)ld_acquire_u32(&P.ctrl->merges[parity]);
            s.ok = ld_acquire_u32(P.err) == 0u;
        }
        __syncthreads();
        const int n = s.n, mbase = s.mbase;
        const bool ok = s.ok != 0;
        __syncthreads();
        if (!ok || n <= P.num_meshes || n <= P.grid_stop) break;
        if (iter >= P.max_iterations) {
            if (threadIdx.x == 0) atomicOr(P.err, kErrIterations);
            break;
        }
        // Items per thread shrink with the cluster count so that small iterations still spread over many
        // SMs; the same rule in every block.
        const long long cap = (long long)B * gridDim.x;
        const int ipt = min(ploc_ipt_max(B), n >= 4 * cap ? 4 : (n >= 2 * cap ? 2 : 1));
        const int T = B * ipt;
        const int tiles = (n + T - 1) / T;
        // The set of active blocks only shrinks: a block that leaves never comes back, and the barrier
        // waits for exactly the blocks still active (the same count in every block).
        const int active = min(active_prev, tiles);
        active_prev = active;
        if ((int)blockIdx.x >= active) break;
        // Clear the other parity's look-back words for the next iteration: it has at most n / B tiles.
        // Nobody reads that array during this iteration.
        const int next_words = (n + B - 1) / B;
        for (int t = blockIdx.x * B + threadIdx.x; t < next_words; t += active * B) by_parity(P.status, parity ^ 1)[t] = 0ull;
        if (blockIdx.x == 0 && threadIdx.x == 0) parity_slot(P.ctrl->tiles_taken, parity ^ 1) = 0u;
        // Tiles are claimed in order from a counter: a block that finishes early takes the next tile, and a
        // tile's look-back predecessors were claimed (and mostly finished) before it.
        for (;;) {
            if (threadIdx.x == 0) s.claim = atomicAdd(&parity_slot(P.ctrl->tiles_taken, parity), 1u);
            __syncthreads();
            const int t = (int)s.claim;
            if (t >= tiles) break;
            ploc_tile<B>(P, s, t, tiles, n, mbase, parity, ipt);
            __syncthreads();
        }
        if (active == 1) {
            __threadfence();
            __syncthreads();
        } else if (!grid_barrier(&P.ctrl->barrier, (uint32_t)active, P.err)) {
            break;
        }
        ++iter;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) P.ctrl->iterations = iter;
}

// Iterations between ctas * kMidSlice and kTailMax clusters in one thread-block cluster of 16 (or 8) CTAs of 1024
// threads.
// There ploc_kernel pays ~15 us per iteration for a chain of global round trips (tile claim, window load,
// look-back, grid barrier) while only a few blocks have tiles. Here the clusters stay in global memory (L2):
// CTA k takes positions [k * slice, (k + 1) * slice), loads them with a halo of r on each side into shared
// memory and finds the nearest neighbours of its slice and of the r positions on either side (same key as
// everywhere, each pair evaluated once), so the mutual test needs no other CTA; the slices' (kept, merged)
// counts are exchanged through distributed shared memory, so every CTA derives the same prefix, totals and
// next cluster count, and writes its kept clusters and new nodes in position order exactly as ploc_kernel
// numbers them. Every branch depends only on values that are identical in all CTAs, so all of them reach the
// same barriers.
constexpr int kMidCtasMax = 16;  // a non-portable cluster size; 8 where 16 cannot be scheduled
constexpr int kMidSlice = 2048;  // positions per CTA at most: the phase covers up to ctas * kMidSlice clusters
constexpr int kMidWindow = kMidSlice + 4 * kRadiusMax;  // the slice, its neighbours' positions and theirs
constexpr int kMidNear = kMidSlice + 2 * kRadiusMax;    // positions whose nearest neighbour the CTA computes

struct MidSmem {
    float4 lo[kMidWindow];
    float4 hi[kMidWindow];
    int4 info[kMidWindow];
    int nn[kMidNear];
    unsigned long long key[kMidNear];
    uint32_t warp_sum[kTailThreads / 32];
    uint32_t totals;  // kept | merged << 16 of this CTA's slice
};

__global__ void __launch_bounds__(kTailThreads) ploc_mid_kernel(PlocParams P) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    MidSmem& s = *reinterpret_cast<MidSmem*>(s_raw);
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const int ctas = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    constexpr int IPT = kMidSlice / kTailThreads;
    // every CTA reads the same control words: the decisions below are identical across the cluster
    const bool err0 = ld_acquire_u32(P.err) != 0u;
    uint32_t iter = P.ctrl->iterations;
    int n = (int)P.ctrl->n[iter & 1];
    int mbase = (int)P.ctrl->merges[iter & 1];
    if (err0 || n <= P.num_meshes || n <= kTailMax) return;
    if (n > ctas * kMidSlice) {  // cannot happen: ploc_kernel runs until n <= grid_stop
        if (rank == 0 && threadIdx.x == 0) atomicOr(P.err, kErrIterations);
        return;
    }
    const int r = P.radius;
    const int max_internal = P.num_leaves - P.num_meshes;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    bool failed = false;
    cluster.sync();  // all CTAs are running before anyone reads a peer's shared memory
    while (n > P.num_meshes && n > kTailMax) {
        if (iter >= P.max_iterations) {
            if (rank == 0 && threadIdx.x == 0) atomicOr(P.err, kErrIterations);
            failed = true;
            break;
        }
        const int par = (int)(iter & 1);
        const int slice = (n + ctas - 1) / ctas;
        const int q0 = min(n, rank * slice), q1 = min(n, q0 + slice);
        const int e0 = max(0, q0 - r), e1 = min(n, q1 + r);          // positions whose neighbour we need
        const int w0 = max(0, q0 - 2 * r), w1 = min(n, q1 + 2 * r);  // and their candidates
        const float4* __restrict__ glo = by_parity(P.lo, par);
        const float4* __restrict__ ghi = by_parity(P.hi, par);
        const int4* __restrict__ gin = by_parity(P.info, par);
        for (int i = threadIdx.x; i < w1 - w0; i += kTailThreads) {
            cp_async16(&s.lo[i], glo + w0 + i);
            cp_async16(&s.hi[i], ghi + w0 + i);
            cp_async16(&s.info[i], gin + w0 + i);
        }
        cp_async_wait_all();
        __syncthreads();
        nn_search_sym<kTailThreads>(s.lo, s.hi, w0, n, e0, e1, r, s.nn, s.key);
        __syncthreads();
        // ---- merge decisions for this slice ---------------------------------------------------------
        const int ib = q0 + (int)threadIdx.x * IPT;
        uint32_t keep_bits = 0, merge_bits = 0;
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const int i = ib + k;
            if (i >= q1) break;
            const int j = s.nn[i - e0];
            const bool mutual = j >= 0 && s.nn[j - e0] == i;  // j is within r of i: inside [e0, e1)
            if (!(mutual && i > j)) keep_bits |= 1u << k;
            if (mutual && i < j) merge_bits |= 1u << k;
        }
        const uint32_t mine = (uint32_t)__popc(keep_bits) | ((uint32_t)__popc(merge_bits) << 16);
        uint32_t x = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s.warp_sum[warp] = x;
        __syncthreads();
        const uint32_t ws = s.warp_sum[lane];
        uint32_t wx = ws;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, wx, o);
            if (lane >= o) wx += y;
        }
        const uint32_t local_total = __shfl_sync(0xffffffffu, wx, 31);
        const uint32_t woff = __shfl_sync(0xffffffffu, wx - ws, warp);
        const uint32_t excl = woff + x - mine;
        if (threadIdx.x == 0) s.totals = local_total;
        __syncthreads();
        cluster.sync();  // every slice's counts are published
        uint32_t before = 0, all = 0;
        for (int c = 0; c < ctas; ++c) {
            const uint32_t t = *cluster.map_shared_rank(&s.totals, c);
            if (c < rank) before += t;
            all += t;
        }
        // ---- kept clusters and new nodes, in position order ----------------------------------------
        float4* __restrict__ olo = by_parity(P.lo, par ^ 1);
        float4* __restrict__ ohi = by_parity(P.hi, par ^ 1);
        int4* __restrict__ oin = by_parity(P.info, par ^ 1);
        uint32_t kpos = (before & 0xFFFFu) + (excl & 0xFFFFu);
        uint32_t mpos = (uint32_t)mbase + (before >> 16) + (excl >> 16);
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            if (!((keep_bits >> k) & 1u)) continue;
            const int i = ib + k;
            float4 oa = s.lo[i - w0], ob = s.hi[i - w0];
            int4 oi = s.info[i - w0];
            if ((merge_bits >> k) & 1u) {
                const int j = s.nn[i - e0];
                const int knew = (int)mpos++;
                if (knew >= max_internal) {
                    atomicOr(P.err, kErrIterations);
                    continue;
                }
                emit_node(P, knew, s.lo[i - w0], s.hi[i - w0], s.info[i - w0], s.lo[j - w0], s.hi[j - w0],
                          s.info[j - w0], oa, ob, oi);
            }
            olo[kpos] = oa;
            ohi[kpos] = ob;
            oin[kpos] = oi;
            ++kpos;
        }
        const int kept = (int)(all & 0xFFFFu);
        __threadfence();
        __syncthreads();
        cluster.sync();  // this iteration's clusters are written; no peer reads the counts any more
        if (kept == n) {  // no progress: impossible under a strict total order on pairs
            if (rank == 0 && threadIdx.x == 0) atomicOr(P.err, kErrIterations);
            failed = true;
            break;
        }
        n = kept;
        mbase += (int)(all >> 16);
        ++iter;
    }
    if (!failed && rank == 0 && threadIdx.x == 0) {
        P.ctrl->n[iter & 1] = (uint32_t)n;
        P.ctrl->merges[iter & 1] = (uint32_t)mbase;
        P.ctrl->iterations = iter;
    }
}

// The last iterations (at most kTailMax clusters) in one thread-block cluster of kTailCtas CTAs of 1024 threads.
// Every CTA keeps all clusters in its shared memory (double-buffered); per iteration each CTA finds the nearest
// neighbours of its slice of positions, and after one cluster barrier reads the other slices from their
// owners' shared memory (distributed shared memory loads, all in flight at once); then every CTA runs the
// same merge and compaction over all positions, so all copies stay identical without exchanging them (only
// CTA 0 writes the new nodes). Once at most kTailSolo clusters remain, the other CTAs leave and CTA 0 finishes
// alone without a cluster barrier per iteration. Same rules as ploc_kernel, so the result still equals the
// oracle's loop.
constexpr int kTailCtasMax = 8;

struct TailSmem {
    float4 lo[2][kTailMax];
    float4 hi[2][kTailMax];
    int4 info[2][kTailMax];
    int nn[2][kTailMax];  // by iteration parity: peers read slice k while slice k+1 is being written
    uint32_t warp_sum[kTailThreads / 32];
};

__global__ void __launch_bounds__(kTailThreads) ploc_tail_kernel(PlocParams P) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    TailSmem& s = *reinterpret_cast<TailSmem*>(s_raw);
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const int ctas = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    constexpr int IPT = kTailMax / kTailThreads;
    // every CTA reads the same control words: the decisions below are identical across the cluster
    const bool err0 = ld_acquire_u32(P.err) != 0u;
    uint32_t iter = P.ctrl->iterations;
    int n = (int)P.ctrl->n[iter & 1];
    int mbase = (int)P.ctrl->merges[iter & 1];
    if (err0 || n <= P.num_meshes) return;
    if (n > kTailMax) {  // cannot happen: the grid kernel and the middle phase run until n <= kTailMax
        if (rank == 0 && threadIdx.x == 0) atomicOr(P.err, kErrIterations);
        return;
    }
    const uint32_t first_parity = iter & 1;
    for (int i = threadIdx.x; i < n; i += kTailThreads) {
        cp_async16(&s.lo[0][i], by_parity(P.lo, first_parity) + i);
        cp_async16(&s.hi[0][i], by_parity(P.hi, first_parity) + i);
        cp_async16(&s.info[0][i], by_parity(P.info, first_parity) + i);
    }
    cp_async_wait_all();
    __syncthreads();
    cluster.sync();  // all CTAs are running before anyone stores into a peer's shared memory
    const int r = P.radius;
    const int max_internal = P.num_leaves - P.num_meshes;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int cur = 0;
    uint32_t tail_iters = 0;
    bool failed = false;
    bool solo = ctas == 1;  // CTA 0 alone: the peers have left the cluster
    while (n > P.num_meshes) {
        if (iter + tail_iters >= P.max_iterations) {
            if (rank == 0 && threadIdx.x == 0) atomicOr(P.err, kErrIterations);
            failed = true;
            break;
        }
        if (!solo && n <= kTailSolo) {
            // few clusters: one CTA searches them all faster than the cluster exchanges slices
            cluster.sync();  // no peer reads this CTA's shared memory after this point
            if (rank != 0) return;
            solo = true;
        }
        const int par = (int)(tail_iters & 1);
        const float4* __restrict__ lo = s.lo[cur];
        const float4* __restrict__ hi = s.hi[cur];
        const int4* __restrict__ info = s.info[cur];
        // ---- neighbours of this CTA's slice; then every slice from its owner ---------------------------
        // (each position's candidates split over up to 16 threads: few positions, short searches)
        if (solo) {
            nn_search_split<kTailThreads>(lo, hi, n, 0, n, r, s.nn[par]);
            __syncthreads();
        } else {
            const int slice = (n + ctas - 1) / ctas;
            const int q0 = min(n, rank * slice), q1 = min(n, q0 + slice);
            nn_search_split<kTailThreads>(lo, hi, n, q0, q1, r, s.nn[par]);
            cluster.sync();  // release our slice, acquire the peers'
            // pull the other slices (all loads in flight at once; the owners do not write s.nn[par] again
            // before the next iteration's cluster barrier)
            int v[IPT];
#pragma unroll
            for (int k = 0; k < IPT; ++k) {
                const int q = (int)threadIdx.x + k * kTailThreads;
                const int owner = q < n ? q / slice : rank;
                v[k] = owner != rank ? cluster.map_shared_rank(s.nn[par], owner)[q] : 0;
            }
#pragma unroll
            for (int k = 0; k < IPT; ++k) {
                const int q = (int)threadIdx.x + k * kTailThreads;
                if (q < n && q / slice != rank) s.nn[par][q] = v[k];
            }
            __syncthreads();
        }
        const int* __restrict__ nn = s.nn[par];
        // ---- merge decisions and compaction over all positions (identical in every CTA) --------------
        const int ib = threadIdx.x * IPT;
        uint32_t keep_bits = 0, merge_bits = 0;
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const int i = ib + k;
            if (i >= n) break;
            const int j = nn[i];
            const bool mutual = j >= 0 && nn[j] == i;
            if (!(mutual && i > j)) keep_bits |= 1u << k;
            if (mutual && i < j) merge_bits |= 1u << k;
        }
        const uint32_t mine = (uint32_t)__popc(keep_bits) | ((uint32_t)__popc(merge_bits) << 16);
        uint32_t x = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s.warp_sum[warp] = x;
        __syncthreads();
        // scan of the 32 warp sums with shuffles (every warp, redundantly)
        const uint32_t ws = s.warp_sum[lane];
        uint32_t wx = ws;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, wx, o);
            if (lane >= o) wx += y;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, wx, 31);
        const uint32_t woff = __shfl_sync(0xffffffffu, wx - ws, warp);
        const uint32_t excl = woff + x - mine;
        uint32_t kpos = excl & 0xFFFFu;
        uint32_t mpos = (uint32_t)mbase + (excl >> 16);
        const int nxt = cur ^ 1;
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            if (!((keep_bits >> k) & 1u)) continue;
            const int i = ib + k;
            float4 oa = lo[i], ob = hi[i];
            int4 oi = info[i];
            if ((merge_bits >> k) & 1u) {
                const int j = nn[i];
                const int knew = (int)mpos++;
                if (knew >= max_internal) {
                    if (rank == 0) atomicOr(P.err, kErrIterations);
                    continue;
                }
                if (rank == 0) {
                    emit_node(P, knew, lo[i], hi[i], info[i], lo[j], hi[j], info[j], oa, ob, oi);
                } else {
                    const float4 ja = lo[j], jb = hi[j];
                    const int4 ji = info[j];
                    oa = make_float4(fminf(oa.x, ja.x), fminf(oa.y, ja.y), fminf(oa.z, ja.z),
                                     __int_as_float(P.num_leaves + knew));
                    ob = make_float4(fmaxf(ob.x, jb.x), fmaxf(ob.y, jb.y), fmaxf(ob.z, jb.z), ob.w);
                    oi = make_int4(oi.x + ji.x, min(oi.y, ji.y), max(oi.z, ji.z) + 1, 0);
                }
            }
            s.lo[nxt][kpos] = oa;
            s.hi[nxt][kpos] = ob;
            s.info[nxt][kpos] = oi;
            ++kpos;
        }
        const int kept = (int)(total & 0xFFFFu);
        mbase += (int)(total >> 16);
        __syncthreads();
        if (kept == n) {  // no progress: impossible under a strict total order on pairs
            if (rank == 0 && threadIdx.x == 0) atomicOr(P.err, kErrIterations);
            failed = true;
            break;
        }
        n = kept;
        cur = nxt;
        ++tail_iters;
    }
    if (!solo) cluster.sync();  // no CTA leaves while a peer may still read its shared memory
    if (failed || rank != 0) return;
    // final clusters (one per mesh) to the buffer of the final parity, for the root pass
    const uint32_t final_iter = iter + tail_iters;
    for (int i = threadIdx.x; i < n; i += kTailThreads) {
        by_parity(P.lo, final_iter & 1)[i] = s.lo[cur][i];
        by_parity(P.hi, final_iter & 1)[i] = s.hi[cur][i];
        by_parity(P.info, final_iter & 1)[i] = s.info[cur][i];
    }
    if (threadIdx.x == 0) P.ctrl->iterations = final_iter;
}

// ------------------------------------------------------------------------------------------------
// Hierarchical PLOC, after Benthin, Meister, Barczak, Mehalwal, Tsakok and Kensler, "H-PLOC" (HPG 2024): PLOC
// merging confined to the nodes of the binary radix tree of the sorted keys, bottom up in one launch, with no
// global iteration and no grid barrier.
//
// The radix tree (Apetrei 2014): split s lies between sorted positions s and s+1 with the order key
// (keys[s] ^ keys[s+1], s ^ (s+1), s), lexicographic; a node [l, r] joins the neighbour across the split with the
// smaller key (split r if l is its mesh's first position or r is not its mesh's last and key(r) < key(l-1), else
// split l-1). Mesh bits above the code make every split between meshes larger than any split inside one, so a
// mesh is a subtree. One thread starts at each leaf; at a split, the first child to arrive leaves its far boundary
// (atomic exchange) and stops, the second goes on with the union.
//
// Each node holds a list of clusters in position order, stored at its first position: a node of at most T
// positions (T = kHplocThreshold) is its leaves, untouched; a larger one is processed by the whole warp of the
// thread that reached it: the left child's list then the right child's, one cluster per lane, and PLOC
// iterations (nearest neighbour by the key of ploc_kernel over list indices within the radius, by warp shuffles;
// mutual pairs merge into the lower index; ballot compaction) until at most T clusters are left, or one at a
// mesh's root. Node ids are deterministic: split s of mesh k owns id N + s - k; a list of c clusters carries
// c - 1 ids not yet used, a node's pool is the left list's unused ids, its own split's id, the right list's;
// merges take ids from the front of the pool (iteration, then position order) and the rest go up with the list.
// oracle/dipl_oracle.c orc_hploc restates the whole procedure sequentially.
// ------------------------------------------------------------------------------------------------
constexpr int kHplocThreshold = 16;
constexpr int kHplocThreads = 256;
constexpr int kHplocMaxSteps = 192;  // tree levels: key bits (<= 64) + index bits (<= 32), with room to spare

struct HplocParams {
    const void* keys;           // sorted keys (uint32 or uint64)
    const long long* offsets;   // first sorted position of each mesh (+ the total)
    float4* lo;                 // cluster records by sorted position: min xyz, node id bits
    float4* hi;                 //                                     max xyz, mesh index bits
    int4* info;                 //                                     triangle count, first position, height, 0
    int4* child;                // internal node k: left, right, height, 0
    float4* node_lo;            // internal node k: min xyz, triangle count bits
    float4* node_hi;            // internal node k: max xyz, first sorted position bits
    int* parent;
    int* other;                 // per split: the first arriving child's far boundary (-1 before)
    int* cnt;                   // per first position of a processed node: the length of its list
    int* fid;                   // per position of a processed node's list: its unused node ids
    float4* root_lo;            // per mesh: the root cluster (the second cluster buffer)
    float4* root_hi;
    PlocCtrl* ctrl;
    uint32_t* err;
    int num_leaves;
    int num_inner;              // internal nodes of all meshes (num_leaves - num_meshes)
    int num_meshes;
    int radius;
    int max_node_iterations;    // iterations within one node before the build gives up (kErrIterations)
};

__device__ __forceinline__ int atomic_exch_acq_rel(int* p, int v) {
    int old;
    asm volatile("atom.acq_rel.gpu.global.exch.b32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

template <typename K>
__device__ __forceinline__ bool split_before(const K* __restrict__ keys, int a, int b) {
    const K xa = __ldg(keys + a) ^ __ldg(keys + a + 1), xb = __ldg(keys + b) ^ __ldg(keys + b + 1);
    if (xa != xb) return xa < xb;
    const unsigned ia = (unsigned)a ^ (unsigned)(a + 1), ib = (unsigned)b ^ (unsigned)(b + 1);
    if (ia != ib) return ia < ib;
    return a < b;
}

__device__ __forceinline__ float4 shfl4(float4 v, int src) {
    return make_float4(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src),
                       __shfl_sync(0xffffffffu, v.z, src), __shfl_sync(0xffffffffu, v.w, src));
}
__device__ __forceinline__ int4 shfl4(int4 v, int src) {
    return make_int4(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src),
                     __shfl_sync(0xffffffffu, v.z, src), __shfl_sync(0xffffffffu, v.w, src));
}

// One node [nl, nr] with split nm, processed by the whole warp (every lane calls this with the same arguments).
// Returns the PLOC iterations it ran.
__device__ __forceinline__ int hploc_node(const HplocParams& P, int nl, int nr, int nm, int id_base, bool whole) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int T = kHplocThreshold;
    const int lsize = nm - nl + 1, rsize = nr - nm;
    int cl = lsize > T ? __ldcg(P.cnt + nl) : lsize;
    int cr = rsize > T ? __ldcg(P.cnt + nm + 1) : rsize;
    if (cl < 1 || cl > T || cr < 1 || cr > T) {  // a processed child left 1..T clusters; never read past a list
        if (lane == 0) atomicOr(P.err, kErrIterations);
        cl = min(max(cl, 1), min(lsize, T));
        cr = min(max(cr, 1), min(rsize, T));
    }
    int c = cl + cr;
    const bool have = lane < c;
    const int p = lane < cl ? nl + lane : nm + 1 + (lane - cl);
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a;
    int4 inf = make_int4(0, 0, 0, 0);
    if (have) {
        a = __ldcg(P.lo + p);
        b = __ldcg(P.hi + p);
        inf = __ldcg(P.info + p);
    }
    int pool = -1;  // lane q holds the pool's entry q (c - 1 entries)
    if (lane < cl - 1) pool = lsize > T ? __ldcg(P.fid + nl + lane) : id_base + nl + lane;
    else if (lane == cl - 1) pool = id_base + nm;
    else if (lane < c - 1) {
        const int j = lane - cl;
        pool = rsize > T ? __ldcg(P.fid + nm + 1 + j) : id_base + nm + 1 + j;
    }
    const int target = whole ? 1 : T;
    const int R = min(P.radius, 31);
    int used = 0, iters = 0;
    while (c > target) {
        if (iters >= P.max_node_iterations) {
            if (lane == 0) atomicOr(P.err, kErrIterations);
            break;
        }
        float bestd = __int_as_float(0x7F800000);
        int bestj = -1;
        // candidates in the order of the key: gap d ascending; at one gap, the candidate with the even lower index
        // first, then the one below (the key's tie fields after the gap: parity of the lower index, side)
        auto consider = [&](int d, float df, float db, bool fwd_ok, bool back_ok) {
            if (((lane - d) & 1) <= (lane & 1)) {
                if (back_ok && (db < bestd || bestj < 0)) bestd = db, bestj = lane - d;
                if (fwd_ok && (df < bestd || bestj < 0)) bestd = df, bestj = lane + d;
            } else {
                if (fwd_ok && (df < bestd || bestj < 0)) bestd = df, bestj = lane + d;
                if (back_ok && (db < bestd || bestj < 0)) bestd = db, bestj = lane - d;
            }
        };
        const int dmax = min(R, c - 1);
        // two gaps per pass (independent shuffles and distances in flight together), folded in gap order
        for (int d = 1; d <= dmax; d += 2) {
            const int e = d + 1;  // the second gap (only when e <= dmax; e <= 32, and a shuffle by 32 is harmless)
            const float fx = __shfl_down_sync(full, a.x, d), fy = __shfl_down_sync(full, a.y, d);
            const float fz = __shfl_down_sync(full, a.z, d), gx = __shfl_down_sync(full, b.x, d);
            const float gy = __shfl_down_sync(full, b.y, d), gz = __shfl_down_sync(full, b.z, d);
            const float hx = __shfl_down_sync(full, a.x, e), hy = __shfl_down_sync(full, a.y, e);
            const float hz = __shfl_down_sync(full, a.z, e), kx = __shfl_down_sync(full, b.x, e);
            const float ky = __shfl_down_sync(full, b.y, e), kz = __shfl_down_sync(full, b.z, e);
            const bool fwd_d = lane + d < c, fwd_e = e <= dmax && lane + e < c;
            const float df = fwd_d ? ploc_distance(a.x, a.y, a.z, b.x, b.y, b.z, fx, fy, fz, gx, gy, gz)
                                   : __int_as_float(0x7F800000);
            const float de = fwd_e ? ploc_distance(a.x, a.y, a.z, b.x, b.y, b.z, hx, hy, hz, kx, ky, kz)
                                   : __int_as_float(0x7F800000);
            const float db = __shfl_up_sync(full, df, d);  // the pair (lane - d, lane), evaluated by lane - d
            const float dbe = __shfl_up_sync(full, de, e);
            consider(d, df, db, fwd_d, lane >= d && lane < c);
            if (e <= dmax) consider(e, de, dbe, fwd_e, lane >= e && lane < c);
        }
        const int partner = bestj >= 0 ? bestj : lane;
        const int nn_of_partner = __shfl_sync(full, bestj, partner);
        const bool valid = lane < c;
        const bool mutual = valid && bestj >= 0 && nn_of_partner == lane;
        const bool creator = mutual && lane < bestj;
        const float4 pa = shfl4(a, partner), pb = shfl4(b, partner);
        const int4 pi = shfl4(inf, partner);
        const unsigned cm = __ballot_sync(full, creator);
        const int t = __popc(cm & ((1u << lane) - 1u));
        const int id = __shfl_sync(full, pool, (used + t) & 31);
        const int k = id - P.num_leaves;
        const int left = __float_as_int(a.w), right = __float_as_int(pa.w);
        const bool in_range = k >= 0 && k < P.num_inner && left >= 0 && left < P.num_leaves + P.num_inner &&
                              right >= 0 && right < P.num_leaves + P.num_inner;
        if (creator && !in_range) atomicOr(P.err, kErrIterations);  // never write outside the node arrays
        if (creator && in_range) {
            const float3 lo = make_float3(fminf(a.x, pa.x), fminf(a.y, pa.y), fminf(a.z, pa.z));
            const float3 hi = make_float3(fmaxf(b.x, pb.x), fmaxf(b.y, pb.y), fmaxf(b.z, pb.z));
            const int count = inf.x + pi.x, pmin = min(inf.y, pi.y), height = max(inf.z, pi.z) + 1;
            P.child[k] = make_int4(left, right, height, 0);
            P.node_lo[k] = make_float4(lo.x, lo.y, lo.z, __int_as_float(count));
            P.node_hi[k] = make_float4(hi.x, hi.y, hi.z, __int_as_float(pmin));
            P.parent[left] = id;
            P.parent[right] = id;
            a = make_float4(lo.x, lo.y, lo.z, __int_as_float(id));
            b = make_float4(hi.x, hi.y, hi.z, b.w);
            inf = make_int4(count, pmin, height, 0);
        }
        used += __popc(cm);
        const bool keep = valid && !(mutual && lane > bestj);
        const unsigned km = __ballot_sync(full, keep);
        const int nc = __popc(km);
        ++iters;
        if (nc == c) {  // no pair merged: impossible under a strict order on pairs
            if (lane == 0) atomicOr(P.err, kErrIterations);
            break;
        }
        const int src = lane < nc ? (int)__fns(km, 0, lane + 1) : lane;
        a = shfl4(a, src);
        b = shfl4(b, src);
        inf = shfl4(inf, src);
        c = nc;
    }
    if (lane < c) {
        __stcg(P.lo + nl + lane, a);
        __stcg(P.hi + nl + lane, b);
        __stcg(P.info + nl + lane, inf);
    }
    const int f = __shfl_sync(full, pool, (used + lane) & 31);
    if (lane < c - 1) __stcg(P.fid + nl + lane, f);
    if (lane == 0) __stcg(P.cnt + nl, c);
    return iters;
}

template <typename K>
__global__ void __launch_bounds__(kHplocThreads) hploc_kernel(HplocParams P) {
    const unsigned full = 0xffffffffu;
    const K* __restrict__ keys = static_cast<const K*>(P.keys);
    const int N = P.num_leaves;
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    bool active = pos < N;
    int l = pos, r = pos, mesh = 0, mstart = 0, mend = N - 1;
    if (active && P.num_meshes > 1) {
        mesh = find_mesh(P.offsets, P.num_meshes, pos);
        mstart = (int)__ldg(P.offsets + mesh);
        mend = (int)__ldg(P.offsets + mesh + 1) - 1;
    }
    const int id_base = N - mesh;
    int iters = 0;
    for (int step = 0;; ++step) {
        bool todo = false;
        int split = -1;
        if (active) {
            if (l == mstart && r == mend) {
                // this mesh's root, processed by this warp in the previous step (its list is one cluster), or a
                // one-triangle mesh's leaf: the root goes to the second cluster buffer, where the layout reads it
                P.root_lo[mesh] = __ldcg(P.lo + mstart);
                P.root_hi[mesh] = __ldcg(P.hi + mstart);
                active = false;
            } else if (step >= kHplocMaxSteps) {
                active = false;
                atomicOr(P.err, kErrIterations);
            } else {
                const bool left_child = l == mstart || (r != mend && split_before(keys, r, l - 1));
                split = left_child ? r : l - 1;
                // release: this node's list, written by the lanes of this warp before the warp barrier that ended
                // the previous step, is visible before the arrival; acquire: so is the sibling's when we are second
                const int prev = atomic_exch_acq_rel(P.other + split, left_child ? l : r);
                if (prev < 0) {
                    active = false;  // first to arrive: the sibling's thread goes on
                } else {
                    if (left_child) r = prev;
                    else l = prev;
                    todo = (r - l + 1 > kHplocThreshold) || (l == mstart && r == mend);
                }
            }
        }
        __syncwarp();  // every lane's acquire before any lane of the warp loads a list
        unsigned pending = __ballot_sync(full, todo);
        while (pending) {
            const int src = __ffs(pending) - 1;
            pending &= pending - 1u;
            const int nl = __shfl_sync(full, l, src), nr = __shfl_sync(full, r, src);
            const int nm = __shfl_sync(full, split, src), nbase = __shfl_sync(full, id_base, src);
            const bool whole = __shfl_sync(full, (int)(l == mstart && r == mend), src) != 0;
            iters += hploc_node(P, nl, nr, nm, nbase, whole);
        }
        __syncwarp();  // every lane's part of the lists and nodes, before any lane's next (releasing) arrival
        if (!__any_sync(full, active)) break;
    }
    // every lane ran the same node iterations: one count per warp
    if ((threadIdx.x & 31) == 0 && iters) atomicAdd(&P.ctrl->iterations, (uint32_t)iters);
}

__global__ void ploc_init_kernel(const MeshDesc* __restrict__ meshes, const long long* __restrict__ offsets, int m,
                                 long long n, const uint32_t* __restrict__ perm, const float4* __restrict__ tbox,
                                 float4* __restrict__ lo, float4* __restrict__ hi, int4* __restrict__ info,
                                 int* __restrict__ parent) {
    long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p >= n) return;
    long long g = perm[p];
    int k = find_mesh(offsets, m, g);
    (void)meshes;
    const float4 a = __ldg(tbox + 2 * g), b = __ldg(tbox + 2 * g + 1);
    lo[p] = make_float4(a.x, a.y, a.z, __int_as_float((int)p));
    hi[p] = make_float4(b.x, b.y, b.z, __int_as_float(k));
    info[p] = make_int4(1, (int)p, 0, 0);
    parent[p] = -1;
}

__global__ void ploc_ctrl_init_kernel(PlocCtrl* ctrl, uint32_t n, uint32_t roots_second) {
    ctrl->n[0] = n;  // the rest was cleared by a memset
    ctrl->roots_second = roots_second;
}

__global__ void fill_int_kernel(int* p, long long n, int v) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// ------------------------------------------------------------------------------------------------
// Layout: a node with fewer than L triangles is a leaf (the reference's rule, sbvh.cc:273-276);
// inner nodes are numbered in reverse creation order (every root first, children after parents);
// each leaf's triangles go to one contiguous range, ranges ordered by the leaf's first sorted position.
// ------------------------------------------------------------------------------------------------
struct LayoutParams {
    const int4* child;
    const float4* node_lo;
    const float4* node_hi;
    const int* parent;
    int num_leaves;
    int num_inner;
    int L;
};

__device__ __forceinline__ int node_count(const LayoutParams& P, int id) {
    return id < P.num_leaves ? 1 : __float_as_int(P.node_lo[id - P.num_leaves].w);
}
__device__ __forceinline__ int node_pmin(const LayoutParams& P, int id) {
    return id < P.num_leaves ? id : __float_as_int(P.node_hi[id - P.num_leaves].w);
}

__global__ void inner_flags_kernel(LayoutParams P, uint32_t* __restrict__ rev_flags, const uint32_t* err) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= P.num_inner) return;
    uint32_t f = (*err == 0u) && __float_as_int(P.node_lo[k].w) >= P.L ? 1u : 0u;
    rev_flags[P.num_inner - 1 - k] = f;
}

// Inner-node numbering by height (hierarchical clustering): sort keys, then each inner node's traced index is its
// rank, stored where the reverse-order consumers read it (rev_index[num_inner - 1 - k]).
__global__ void height_keys_kernel(LayoutParams P, uint32_t* __restrict__ keys, const uint32_t* err) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= P.num_inner) return;
    const bool inner = (*err == 0u) && __float_as_int(P.node_lo[k].w) >= P.L;
    keys[k] = inner ? 254u - (uint32_t)min(max(P.child[k].z, 0), 254) : 255u;
}

__global__ void height_index_kernel(LayoutParams P, const uint32_t* __restrict__ order, uint32_t* __restrict__ rev_index,
                                    const uint32_t* err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.num_inner || *err != 0u) return;
    const int k = (int)order[i];
    if (__float_as_int(P.node_lo[k].w) >= P.L) rev_index[P.num_inner - 1 - k] = (uint32_t)i;  // inner nodes sort first
}

__global__ void leaf_owner_kernel(LayoutParams P, uint32_t* __restrict__ contrib, int* __restrict__ owner_leaf,
                                  const uint32_t* err) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P.num_leaves) return;
    if (*err != 0u) {
        contrib[p] = 0;
        owner_leaf[p] = -1;
        return;
    }
    int x = p;
    for (int guard = 0; guard < 64; ++guard) {
        int par = P.parent[x];
        if (par < 0 || node_count(P, par) >= P.L) break;
        x = par;
    }
    bool own = node_pmin(P, x) == p;
    contrib[p] = own ? (uint32_t)node_count(P, x) : 0u;
    owner_leaf[p] = own ? x : -1;
    (void)contrib;
}

__device__ __forceinline__ void write_tri(const MeshDesc* meshes, const long long* offsets, int m,
                                          const uint32_t* perm, const int* ref_tri, int pos, float4* tris, int slot) {
    long long g = perm[pos];
    if (ref_tri) g = ref_tri[g];  // a reference: its triangle
    int k = find_mesh(offsets, m, g);
    long long local = g - meshes[k].first;
    Tri t = load_tri(meshes[k], local);
    tris[3 * (long long)slot + 0] = make_float4(t.a.x, t.a.y, t.a.z, __int_as_float((int)local));
    tris[3 * (long long)slot + 1] = make_float4(t.b.x, t.b.y, t.b.z, 0.0f);
    tris[3 * (long long)slot + 2] = make_float4(t.c.x, t.c.y, t.c.z, 0.0f);
}

// One thread per sorted position: the position's leaf (the highest ancestor with fewer than L triangles) and
// its rank in the leaf's left-to-right order (the triangle counts of the left siblings met on the way up) give
// its slot directly, so every thread gathers and writes one triangle (no per-leaf loop).
__global__ void leaf_write_kernel(LayoutParams P, const MeshDesc* __restrict__ meshes,
                                  const long long* __restrict__ offsets, int m, const uint32_t* __restrict__ perm,
                                  const int* __restrict__ ref_tri, const uint32_t* __restrict__ starts, int* __restrict__ leaf_start_of,
                                  float4* __restrict__ tris, int* __restrict__ slot_pos, const uint32_t* err) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P.num_leaves || *err != 0u) return;
    int x = p, rank = 0;
    for (int guard = 0; guard < 64; ++guard) {
        const int par = P.parent[x];
        if (par < 0 || node_count(P, par) >= P.L) break;
        const int4 c = P.child[par - P.num_leaves];
        if (c.y == x) rank += node_count(P, c.x);
        x = par;
    }
    const int first = node_pmin(P, x);
    const int start = (int)starts[first];
    if (p == first) leaf_start_of[x] = start;
    if (slot_pos) slot_pos[start + rank] = p;
    write_tri(meshes, offsets, m, perm, ref_tri, p, tris, start + rank);
}

__device__ __forceinline__ float pad_down(float lo, float hi) {
    float m = fmaxf(fabsf(lo), fabsf(hi));
    return lo - (m * 9.5367431640625e-07f + 1e-30f);  // 2^-20 of the magnitude
}
__device__ __forceinline__ float pad_up(float lo, float hi) {
    float m = fmaxf(fabsf(lo), fabsf(hi));
    return hi + (m * 9.5367431640625e-07f + 1e-30f);
}

__device__ __forceinline__ double box_area(float3 lo, float3 hi) {
    double dx = (double)hi.x - lo.x, dy = (double)hi.y - lo.y, dz = (double)hi.z - lo.z;
    return 2.0 * (dx * dy + dy * dz + dz * dx);
}

__device__ __forceinline__ void child_box(const LayoutParams& P, const float4* tbox, const uint32_t* perm, int id,
                                          float3& lo, float3& hi) {
    if (id < P.num_leaves) {
        long long g = perm[id];
        const float4 a = __ldg(tbox + 2 * g), b = __ldg(tbox + 2 * g + 1);
        lo = make_float3(a.x, a.y, a.z);
        hi = make_float3(b.x, b.y, b.z);
    } else {
        float4 a = P.node_lo[id - P.num_leaves], b = P.node_hi[id - P.num_leaves];
        lo = make_float3(a.x, a.y, a.z);
        hi = make_float3(b.x, b.y, b.z);
    }
}

__device__ __forceinline__ void node_write_one(const LayoutParams& P, const float4* __restrict__ tbox,
                                               const long long* __restrict__ offsets, int m,
                                               const uint32_t* __restrict__ perm,
                                               const uint32_t* __restrict__ rev_index,
                                               const int* __restrict__ leaf_start_of, BNode* __restrict__ nodes,
                                               double* __restrict__ sah, const uint32_t* err, double& local_sum,
                                               double& local_count, int& mesh_out) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= P.num_inner || *err != 0u) return;
    if (__float_as_int(P.node_lo[k].w) < P.L) return;
    const int f = (int)rev_index[P.num_inner - 1 - k];
    const int4 c = P.child[k];
    float3 lo[2], hi[2];
    int ref[2];
    double acc = box_area(make_float3(P.node_lo[k].x, P.node_lo[k].y, P.node_lo[k].z),
                          make_float3(P.node_hi[k].x, P.node_hi[k].y, P.node_hi[k].z));
    for (int s = 0; s < 2; ++s) {
        int id = s == 0 ? c.x : c.y;
        child_box(P, tbox, perm, id, lo[s], hi[s]);
        int cnt = node_count(P, id);
        if (cnt >= P.L) {
            ref[s] = (int)rev_index[P.num_inner - 1 - (id - P.num_leaves)];
        } else {
            ref[s] = make_leaf_ref(leaf_start_of[id], cnt);
            acc += box_area(lo[s], hi[s]) * cnt;
        }
    }
    BNode nd;
    nd.a = make_float4(pad_down(lo[0].x, hi[0].x), pad_up(lo[0].x, hi[0].x), pad_down(lo[0].y, hi[0].y),
                       pad_up(lo[0].y, hi[0].y));
    nd.b = make_float4(pad_down(lo[1].x, hi[1].x), pad_up(lo[1].x, hi[1].x), pad_down(lo[1].y, hi[1].y),
                       pad_up(lo[1].y, hi[1].y));
    nd.c = make_float4(pad_down(lo[0].z, hi[0].z), pad_up(lo[0].z, hi[0].z), pad_down(lo[1].z, hi[1].z),
                       pad_up(lo[1].z, hi[1].z));
    nd.d = make_int4(ref[0], ref[1], 0, 0);
    nodes[f] = nd;
    local_sum = acc;
    local_count = 1.0;
    mesh_out = m == 1 ? 0 : find_mesh(offsets, m, (long long)perm[__float_as_int(P.node_hi[k].w)]);
}

// Single-mesh builds: one FP64 atomic pair per block instead of one per node.
__global__ void node_write_kernel(LayoutParams P, const float4* __restrict__ tbox,
                                  const long long* __restrict__ offsets, int m, const uint32_t* __restrict__ perm,
                                  const uint32_t* __restrict__ rev_index, const int* __restrict__ leaf_start_of,
                                  BNode* __restrict__ nodes, double* __restrict__ sah, const uint32_t* err) {
    double local_sum = 0.0, local_count = 0.0;
    int mesh = -1;  // this thread's node's mesh, -1 without a node
    node_write_one(P, tbox, offsets, m, perm, rev_index, leaf_start_of, nodes, sah, err, local_sum, local_count, mesh);
    if (m != 1) {
        // Nodes are numbered in position order, so a warp's nodes nearly always belong to one mesh: one FP64 atomic
        // pair per warp then, instead of 32 on the same two addresses (the 256-mesh batch spent 91 ms in this kernel
        // with one pair per node). Lanes of a warp that spans meshes add their own.
        const unsigned full = 0xffffffffu;
        const int lead = __ffs(__ballot_sync(full, mesh >= 0)) - 1;
        const int m0 = lead >= 0 ? __shfl_sync(full, mesh, lead) : -1;
        if (__all_sync(full, mesh < 0 || mesh == m0)) {
            for (int o = 16; o > 0; o >>= 1) {
                local_sum += __shfl_xor_sync(full, local_sum, o);
                local_count += __shfl_xor_sync(full, local_count, o);
            }
            if ((threadIdx.x & 31) == 0 && m0 >= 0) {
                atomicAdd(&sah[2 * m0], local_sum);
                atomicAdd(&sah[2 * m0 + 1], local_count);
            }
        } else if (mesh >= 0) {
            atomicAdd(&sah[2 * mesh], local_sum);
            atomicAdd(&sah[2 * mesh + 1], local_count);
        }
        return;
    }
    __shared__ double s_sum[32], s_cnt[32];
    for (int o = 16; o > 0; o >>= 1) {
        local_sum += __shfl_xor_sync(0xffffffffu, local_sum, o);
        local_count += __shfl_xor_sync(0xffffffffu, local_count, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_sum[warp] = local_sum, s_cnt[warp] = local_count;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, c = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a += s_sum[w], c += s_cnt[w];
        if (c > 0.0) {
            atomicAdd(&sah[0], a);
            atomicAdd(&sah[1], c);
        }
    }
}

// Roots of every mesh: the final clusters (one per mesh, in mesh order).
struct RootInfo {
    int root_ref;
    int depth;
    int num_leaves;  // triangles under the root
    int root_id;     // PLOC node id of the root
    double root_area;
    double leaf_cost;  // SAH cost contribution when the root itself is a leaf
};

__global__ void roots_kernel(LayoutParams P, const float4* __restrict__ lo0, const float4* __restrict__ hi0,
                             const float4* __restrict__ lo1, const float4* __restrict__ hi1, const PlocCtrl* ctrl,
                             int m, const uint32_t* __restrict__ rev_index, const int* __restrict__ leaf_start_of,
                             RootInfo* __restrict__ roots, const uint32_t* err) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    RootInfo ri{};
    if (*err != 0u) {
        roots[k] = ri;
        return;
    }
    const bool odd = ctrl->roots_second != 0u || (ctrl->iterations & 1u) != 0u;
    const float4* final_lo = odd ? lo1 : lo0;
    const float4* final_hi = odd ? hi1 : hi0;
    int id = __float_as_int(final_lo[k].w);
    int cnt = node_count(P, id);
    float3 lo = make_float3(final_lo[k].x, final_lo[k].y, final_lo[k].z);
    float3 hi = make_float3(final_hi[k].x, final_hi[k].y, final_hi[k].z);
    ri.root_area = box_area(lo, hi);
    if (cnt >= P.L) {
        ri.root_ref = (int)rev_index[P.num_inner - 1 - (id - P.num_leaves)];
        ri.depth = P.child[id - P.num_leaves].z;
    } else {
        ri.root_ref = make_leaf_ref(leaf_start_of[id], cnt);
        ri.depth = id < P.num_leaves ? 0 : P.child[id - P.num_leaves].z;
        ri.leaf_cost = ri.root_area * cnt;
    }
    ri.num_leaves = cnt;
    ri.root_id = id;
    roots[k] = ri;
}

// Automatic choice by size: 512 threads x up to 2 positions below 2M triangles (1M sphere: 1.58 ms against 1.65
// ms with 256 x 4), 256 x up to 4 above (16M EMC60 soup: 16.3 ms against 18.9 ms with 512 x 2).
int ploc_block_for(int requested, int64_t n) {
    if (requested == 128 || requested == 256 || requested == 512) return requested;
    return n < (int64_t(1) << 21) ? 512 : 256;
}

template <int B>
dipl_status launch_ploc(const PlocParams& P, int initial_tiles, cudaStream_t stream) {
    const size_t smem = sizeof(PlocSmem<B>);
    DIPL_CUDA(cudaFuncSetAttribute(ploc_kernel<B>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, sms = 0, per_sm = 0;
    DIPL_CUDA(cudaGetDevice(&dev));
    DIPL_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    DIPL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ploc_kernel<B>, B, smem));
    if (per_sm < 1) {
        set_last_error("PLOC kernel cannot be resident");
        return DIPL_ERR_CUDA;
    }
    int grid = std::max(1, std::min(initial_tiles, sms * per_sm));
    // cooperative launch (all blocks co-resident, required by the grid barrier); capturable into a graph
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.gridDim = dim3(grid), cfg.blockDim = dim3(B), cfg.dynamicSmemBytes = smem, cfg.stream = stream;
    cfg.attrs = attr, cfg.numAttrs = 1;
    DIPL_CUDA(cudaLaunchKernelEx(&cfg, ploc_kernel<B>, P));
    note_launches();
    return DIPL_OK;
}

// CTAs of the middle phase: the largest cluster of 16 or 8 CTAs the device schedules with its shared memory, 0
// without one (then ploc_kernel runs down to kTailMax clusters).
int ploc_mid_ctas_probe() {
    int ctas = 0;
    const size_t smem = sizeof(MidSmem);
    if (cudaFuncSetAttribute(ploc_mid_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess &&
        cudaFuncSetAttribute(ploc_mid_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
        for (int c = kMidCtasMax; c >= 8 && ctas == 0; c /= 2) {
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = c, attr[0].val.clusterDim.y = 1, attr[0].val.clusterDim.z = 1;
            cfg.gridDim = dim3(c), cfg.blockDim = dim3(kTailThreads), cfg.dynamicSmemBytes = smem;
            cfg.attrs = attr, cfg.numAttrs = 1;
            int clusters = 0;
            if (cudaOccupancyMaxActiveClusters(&clusters, ploc_mid_kernel, &cfg) == cudaSuccess && clusters > 0)
                ctas = c;
        }
    }
    (void)cudaGetLastError();
    return ctas;
}

DeviceProbe g_mid_ctas;
int ploc_mid_ctas() { return probe_per_device(g_mid_ctas, ploc_mid_ctas_probe); }

dipl_status launch_ploc_mid(const PlocParams& P, int ctas, cudaStream_t stream) {
    const size_t smem = sizeof(MidSmem);
    DIPL_CUDA(cudaFuncSetAttribute(ploc_mid_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    DIPL_CUDA(cudaFuncSetAttribute(ploc_mid_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = ctas, attr[0].val.clusterDim.y = 1, attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(ctas), cfg.blockDim = dim3(kTailThreads), cfg.dynamicSmemBytes = smem, cfg.stream = stream;
    cfg.attrs = attr, cfg.numAttrs = 1;
    DIPL_CUDA(cudaLaunchKernelEx(&cfg, ploc_mid_kernel, P));
    note_launches();
    return DIPL_OK;
}

DeviceProbe g_tail_ctas;

dipl_status launch_ploc_tail(const PlocParams& P, cudaStream_t stream) {
    const size_t smem = sizeof(TailSmem);
    DIPL_CUDA(cudaFuncSetAttribute(ploc_tail_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // the largest cluster size the device can schedule with this footprint
    const int ctas = probe_per_device(g_tail_ctas, [smem] {
        for (int c = kTailCtasMax; c >= 1; c /= 2) {
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = c, attr[0].val.clusterDim.y = 1, attr[0].val.clusterDim.z = 1;
            cfg.gridDim = dim3(c), cfg.blockDim = dim3(kTailThreads), cfg.dynamicSmemBytes = smem;
            cfg.attrs = attr, cfg.numAttrs = 1;
            int clusters = 0;
            if (cudaOccupancyMaxActiveClusters(&clusters, ploc_tail_kernel, &cfg) == cudaSuccess && clusters > 0)
                return c;
            (void)cudaGetLastError();
        }
        return 1;
    });
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = ctas, attr[0].val.clusterDim.y = 1, attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(ctas), cfg.blockDim = dim3(kTailThreads), cfg.dynamicSmemBytes = smem, cfg.stream = stream;
    cfg.attrs = attr, cfg.numAttrs = 1;
    DIPL_CUDA(cudaLaunchKernelEx(&cfg, ploc_tail_kernel, P));
    note_launches();
    return DIPL_OK;
}

inline unsigned blocks_for(long long n, int threads) { return (unsigned)std::max<long long>(1, (n + threads - 1) / threads); }

}  // namespace

// ------------------------------------------------------------------------------------------------
// Host orchestration.
// ------------------------------------------------------------------------------------------------
static dipl_status validate_desc(const dipl_build_desc& d) {
    DIPL_CHECK_ARG(d.num_triangles >= 0 && d.num_triangles < (1ll << 27), "num_triangles must be in [0, 2^27)");
    DIPL_CHECK_ARG(d.num_triangles == 0 || (d.d_v0 && d.d_v1 && d.d_v2), "vertex arrays must be non-NULL");
    DIPL_CHECK_ARG(d.code_type == DIPL_CODE_MORTON30 || d.code_type == DIPL_CODE_EMC60, "bad code_type");
    DIPL_CHECK_ARG(d.bv_type == DIPL_BV_AABB || d.bv_type == DIPL_BV_SOBB, "bad bv_type");
    DIPL_CHECK_ARG(d.layout == DIPL_LAYOUT_BINARY || d.layout == DIPL_LAYOUT_WIDE8_Q8, "bad layout");
    DIPL_CHECK_ARG(d.max_triangles_per_leaf >= 2 && d.max_triangles_per_leaf <= 8,
                   "max_triangles_per_leaf must be in [2, 8]");
    DIPL_CHECK_ARG(d.nn_search_radius >= 1 && d.nn_search_radius <= kRadiusMax, "nn_search_radius must be in [1, 32]");
    DIPL_CHECK_ARG(d.kdop_size >= 6 && d.kdop_size <= 32 && d.kdop_size % 2 == 0, "kdop_size must be even, 6..32");
    DIPL_CHECK_ARG(d.ploc_block_size == 0 || d.ploc_block_size == 128 || d.ploc_block_size == 256 ||
                       d.ploc_block_size == 512,
                   "ploc_block_size must be 0, 128, 256 or 512");
    DIPL_CHECK_ARG(d.bv_type == DIPL_BV_AABB || d.layout == DIPL_LAYOUT_BINARY,
                   "SOBB bounding volumes use the binary layout");
    DIPL_CHECK_ARG(d.layout != DIPL_LAYOUT_WIDE8_Q8 || d.max_triangles_per_leaf <= 5,
                   "the 8-wide layout needs max_triangles_per_leaf <= 5 (at most 32 leaf triangles per node)");
    DIPL_CHECK_ARG(d.sort_digit_bits == 0 || d.sort_digit_bits == 6 || d.sort_digit_bits == 7 ||
                       d.sort_digit_bits == 8 || d.sort_digit_bits == 10,
                   "sort_digit_bits must be 0, 6, 7, 8 or 10");
    DIPL_CHECK_ARG(d.clustering == DIPL_CLUSTER_HPLOC || d.clustering == DIPL_CLUSTER_PLOC,
                   "clustering must be DIPL_CLUSTER_HPLOC or DIPL_CLUSTER_PLOC");
    DIPL_CHECK_ARG(d.split_budget >= 0 && d.split_budget <= 100, "split_budget must be 0..100");
    return DIPL_OK;
}

// ------------------------------------------------------------------------------------------------
// A build in three phases: prepare (validation, every allocation, uploads), enqueue (only kernels, memsets
// and device copies on the stream, ending with one copy of the per-mesh summary to pinned host memory:
// capturable into a CUDA graph) and finish (read the summary after the stream synchronised, make handles).
// ------------------------------------------------------------------------------------------------
struct BuildPlan {
    std::vector<dipl_build_desc> descs;
    std::vector<int> mesh_of_desc;
    std::vector<MeshDesc> meshes;
    std::vector<long long> offsets;   // first triangle of every mesh (+ the total): vertex access
    std::vector<long long> coffsets;  // first cluster leaf (reference) of every mesh (+ the total)
    dipl_build_desc d0{};
    int count = 0, m = 0, L = 4;
    long long T = 0;                  // triangles of the batch
    long long N = 0, K = 0, Kalloc = 1;  // cluster leaves (references; = T without pre-splitting), internal nodes
    bool split = false;               // pre-splitting of large triangles
    int code_bits = 30, mesh_bits = 0, key_bits = 30, code_shift = 0, mesh_shift = 0, key_bytes = 4;
    int digit_bits = 8, B = 256, tiles0 = 1, tiles_max = 1;
    cudaStream_t stream = nullptr;
    std::shared_ptr<Storage> out;   // arrays the handles keep
    std::shared_ptr<Storage> work;  // scratch of the pipeline
    uint32_t* d_err = nullptr;
    MeshDesc* d_meshes = nullptr;
    long long* d_offsets = nullptr;
    long long* d_coffsets = nullptr;  // = d_offsets without pre-splitting
    uint32_t *pieces = nullptr, *piece_first = nullptr;  // per triangle: references, first reference
    unsigned long long* mesh_wsum = nullptr;
    int* ref_tri = nullptr;           // per reference: its triangle (global index); NULL without pre-splitting
    Bounds* d_bounds = nullptr;
    CodeParams* d_params = nullptr;
    void *keys = nullptr, *keys_sorted = nullptr, *keys_alt = nullptr;
    uint32_t *perm = nullptr, *perm_alt = nullptr;
    float4* tbox = nullptr;  // per triangle (input order): box lo, box hi (32 bytes)
    unsigned char* sort_scratch = nullptr;
    PlocCtrl* d_ctrl = nullptr;
    int4* child = nullptr;
    float4 *nlo = nullptr, *nhi = nullptr;
    int* parent = nullptr;
    unsigned long long* status = nullptr;
    float4 *c_lo[2] = {nullptr, nullptr}, *c_hi[2] = {nullptr, nullptr};
    int4* c_in[2] = {nullptr, nullptr};
    int *hp_other = nullptr, *hp_cnt = nullptr, *hp_fid = nullptr;  // hierarchical clustering
    uint32_t *rev_flags = nullptr, *contrib = nullptr, *d_counts = nullptr;
    int *owner_leaf = nullptr, *leaf_start_of = nullptr;
    int* slot_pos = nullptr;  // pre-split SOBB builds: per slot of the leaf triangle array, its sorted position
    unsigned char* scan_scratch = nullptr;
    BNode* nodes = nullptr;
    float4* tris = nullptr;
    double* d_sah = nullptr;
    RootInfo* d_roots = nullptr;
    SobbScratch sobb{};
    SNode* snodes = nullptr;
    unsigned char* h_summary = nullptr;  // pinned
    bool owns_summary = false;
    size_t summary_bytes = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int graph_kernels = 0;
    ~BuildPlan() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        if (h_summary && owns_summary) cudaFreeHost(h_summary);
    }
};

static dipl_status enqueue_bounds_and_params(BuildPlan& P, cudaStream_t stream);

static dipl_status plan_prepare(BuildPlan& P, const dipl_build_desc* descs, int count, cudaStream_t stream,
                                bool own_summary) {
    DIPL_CHECK_ARG(descs && count >= 1, "descs must be non-NULL and count >= 1");
    for (int i = 0; i < count; ++i) {
        dipl_status st = validate_desc(descs[i]);
        if (st != DIPL_OK) return st;
    }
    const dipl_build_desc& d0 = descs[0];
    for (int i = 1; i < count; ++i) {
        DIPL_CHECK_ARG(descs[i].code_type == d0.code_type && descs[i].bv_type == d0.bv_type &&
                           descs[i].layout == d0.layout && descs[i].max_triangles_per_leaf == d0.max_triangles_per_leaf &&
                           descs[i].nn_search_radius == d0.nn_search_radius && descs[i].kdop_size == d0.kdop_size &&
                           descs[i].ploc_block_size == d0.ploc_block_size &&
                           descs[i].sort_digit_bits == d0.sort_digit_bits && descs[i].clustering == d0.clustering &&
                           descs[i].split_budget == d0.split_budget,
                       "batched builds need one set of build options");
    }
    P.descs.assign(descs, descs + count);
    P.count = count;
    P.d0 = d0;
    P.stream = stream;
    P.mesh_of_desc.assign(count, -1);
    long long total = 0;
    for (int i = 0; i < count; ++i) {
        if (descs[i].num_triangles == 0) continue;
        P.mesh_of_desc[i] = (int)P.meshes.size();
        P.meshes.push_back(MeshDesc{descs[i].d_v0, descs[i].d_v1, descs[i].d_v2, total, descs[i].num_triangles});
        P.offsets.push_back(total);
        total += descs[i].num_triangles;
    }
    DIPL_CHECK_ARG(total < (1ll << 27), "total triangles of a build must be < 2^27");
    P.m = (int)P.meshes.size();
    P.offsets.push_back(total);
    P.T = total;
    P.N = total;
    P.coffsets = P.offsets;
    P.split = d0.split_budget > 0;
    P.L = d0.max_triangles_per_leaf;
    P.out = std::make_shared<Storage>();
    P.out->stream = stream;
    P.work = std::make_shared<Storage>();
    P.work->stream = stream;
    dipl_status st;
    if ((st = P.out->alloc(&P.d_err, 4)) != DIPL_OK) return st;
    P.K = P.N - P.m;
    P.Kalloc = std::max<long long>(P.K, 1);
    if (P.m == 0) return DIPL_OK;
    const int m = P.m;
    Storage& W = *P.work;
    Storage& O = *P.out;
    if ((st = W.alloc(&P.d_meshes, m)) != DIPL_OK || (st = W.alloc(&P.d_offsets, m + 1)) != DIPL_OK ||
        (st = W.alloc(&P.d_bounds, m)) != DIPL_OK || (st = W.alloc(&P.d_params, m)) != DIPL_OK)
        return st;
    DIPL_CUDA(cudaMemcpyAsync(P.d_meshes, P.meshes.data(), sizeof(MeshDesc) * m, cudaMemcpyHostToDevice, stream));
    DIPL_CUDA(cudaMemcpyAsync(P.d_offsets, P.offsets.data(), sizeof(long long) * (m + 1), cudaMemcpyHostToDevice,
                              stream));
    P.d_coffsets = P.d_offsets;
    if (P.split) {
        // bounds and code parameters first (they are the triangles'), then the piece counts, their scan and every
        // mesh's first reference; the reference count sizes everything after, so it is read back here
        const long long T = P.T;
        uint32_t* d_total = nullptr;
        if ((st = W.alloc(&P.pieces, T)) != DIPL_OK || (st = W.alloc(&P.piece_first, T)) != DIPL_OK ||
            (st = W.alloc(&P.mesh_wsum, m)) != DIPL_OK || (st = W.alloc(&P.d_coffsets, m + 1)) != DIPL_OK ||
            (st = W.alloc(&d_total, 4)) != DIPL_OK)
            return st;
        unsigned char* scan_tmp = nullptr;
        if ((st = W.alloc(&scan_tmp, scan_scratch_bytes(T))) != DIPL_OK) return st;
        if ((st = enqueue_bounds_and_params(P, stream)) != DIPL_OK) return st;
        DIPL_CUDA(cudaMemsetAsync(P.mesh_wsum, 0, sizeof(unsigned long long) * m, stream));
        split_weight_kernel<<<blocks_for(T, 256), 256, 0, stream>>>(P.d_meshes, P.d_offsets, m, T, P.d_bounds,
                                                                    P.mesh_wsum);
        note_launches();
        split_count_kernel<<<blocks_for(T, 256), 256, 0, stream>>>(P.d_meshes, P.d_offsets, m, T, P.d_bounds,
                                                                   P.mesh_wsum, d0.split_budget, P.pieces);
        note_launches();
        DIPL_CUDA(cudaGetLastError());
        if ((st = exclusive_scan_u32(P.pieces, P.piece_first, T, d_total, scan_tmp, stream, P.d_err)) != DIPL_OK)
            return st;
        mesh_ref_offsets_kernel<<<blocks_for(m + 1, 64), 64, 0, stream>>>(P.d_offsets, m, P.piece_first, d_total,
                                                                          P.d_coffsets);
        note_launches();
        DIPL_CUDA(cudaGetLastError());
        P.coffsets.assign(m + 1, 0);
        DIPL_CUDA(cudaMemcpyAsync(P.coffsets.data(), P.d_coffsets, sizeof(long long) * (m + 1), cudaMemcpyDeviceToHost,
                                  stream));
        uint32_t err = 0;
        DIPL_CUDA(cudaMemcpyAsync(&err, P.d_err, 4, cudaMemcpyDeviceToHost, stream));
        DIPL_CUDA(cudaStreamSynchronize(stream));
        if (err != 0u) {
            set_last_error("build: a bounded device wait timed out while counting the pieces of large triangles");
            return DIPL_ERR_TIMEOUT;
        }
        P.N = P.coffsets[m];
        DIPL_CHECK_ARG(P.N < (1ll << 27), "references of a build (triangles and their pieces) must be < 2^27");
        P.K = P.N - m;
        P.Kalloc = std::max<long long>(P.K, 1);
        if ((st = O.alloc(&P.ref_tri, P.N)) != DIPL_OK) return st;
    }
    const long long N = P.N, K = P.K, Kalloc = P.Kalloc;
    P.code_bits = d0.code_type == DIPL_CODE_MORTON30 ? 30 : 60;
    while ((1ll << P.mesh_bits) < m) ++P.mesh_bits;
    P.key_bits = P.code_bits + P.mesh_bits;
    if (P.key_bits > 64) {
        P.code_shift = P.key_bits - 64;
        P.key_bits = 64;
    }
    P.mesh_shift = P.mesh_bits > 0 ? P.code_bits - P.code_shift : 0;
    P.key_bytes = P.key_bits <= 32 ? 4 : 8;
    P.digit_bits = d0.sort_digit_bits > 0 ? d0.sort_digit_bits : 8;
    if ((st = W.alloc((unsigned char**)&P.keys, N * P.key_bytes)) != DIPL_OK ||
        (st = W.alloc((unsigned char**)&P.keys_sorted, N * P.key_bytes)) != DIPL_OK ||
        (st = W.alloc((unsigned char**)&P.keys_alt, N * P.key_bytes)) != DIPL_OK ||
        (st = O.alloc(&P.perm, N)) != DIPL_OK || (st = W.alloc(&P.perm_alt, N)) != DIPL_OK ||
        (st = W.alloc(&P.tbox, 2 * N)) != DIPL_OK ||
        (st = W.alloc(&P.sort_scratch, radix_sort_scratch_bytes(N, 0, P.key_bits, P.digit_bits))) != DIPL_OK)
        return st;
    P.B = ploc_block_for(d0.ploc_block_size, (int64_t)N);
    P.tiles0 = (int)((N + P.B * ploc_ipt_max(P.B) - 1) / (P.B * ploc_ipt_max(P.B)));
    P.tiles_max = (int)((N + P.B - 1) / P.B);
    if ((st = W.alloc(&P.d_ctrl, 1)) != DIPL_OK || (st = O.alloc(&P.child, Kalloc)) != DIPL_OK ||
        (st = O.alloc(&P.nlo, Kalloc)) != DIPL_OK || (st = O.alloc(&P.nhi, Kalloc)) != DIPL_OK ||
        (st = W.alloc(&P.parent, N + Kalloc)) != DIPL_OK || (st = W.alloc(&P.status, 2 * P.tiles_max + 2)) != DIPL_OK)
        return st;
    for (int k = 0; k < 2; ++k)
        if ((st = W.alloc(&P.c_lo[k], N)) != DIPL_OK || (st = W.alloc(&P.c_hi[k], N)) != DIPL_OK ||
            (st = W.alloc(&P.c_in[k], N)) != DIPL_OK)
            return st;
    if (d0.clustering == DIPL_CLUSTER_HPLOC &&
        ((st = W.alloc(&P.hp_other, N)) != DIPL_OK || (st = W.alloc(&P.hp_cnt, N)) != DIPL_OK ||
         (st = W.alloc(&P.hp_fid, N)) != DIPL_OK))
        return st;
    if ((st = W.alloc(&P.rev_flags, Kalloc)) != DIPL_OK || (st = W.alloc(&P.contrib, N)) != DIPL_OK ||
        (st = W.alloc(&P.owner_leaf, N)) != DIPL_OK || (st = W.alloc(&P.leaf_start_of, N + Kalloc)) != DIPL_OK ||
        (st = W.alloc(&P.scan_scratch, scan_scratch_bytes(std::max(N, Kalloc)))) != DIPL_OK ||
        (st = W.alloc(&P.d_counts, 4)) != DIPL_OK || (st = O.alloc(&P.nodes, Kalloc)) != DIPL_OK ||
        (st = O.alloc(&P.tris, 3 * N)) != DIPL_OK || (st = W.alloc(&P.d_sah, 2 * m)) != DIPL_OK ||
        (st = W.alloc(&P.d_roots, m)) != DIPL_OK)
        return st;
    if (d0.bv_type == DIPL_BV_SOBB) {
        if ((st = sobb_prepare(N, K, W, O, &P.sobb, &P.snodes)) != DIPL_OK) return st;
        if (P.split && (st = W.alloc(&P.slot_pos, N)) != DIPL_OK) return st;
    }
    P.summary_bytes = sizeof(RootInfo) * m + sizeof(double) * 2 * m + 16;
    if (own_summary) {  // a plan replays into its own pinned buffer
        if (cudaMallocHost(&P.h_summary, P.summary_bytes) != cudaSuccess) {
            P.h_summary = nullptr;
            set_last_error("pinned host allocation failed");
            return DIPL_ERR_OUT_OF_MEMORY;
        }
        P.owns_summary = true;
    } else {  // a one-shot build reads it back right away: the calling thread's staging buffer
        P.h_summary = pinned_host_buffer(P.summary_bytes);
        if (!P.h_summary) {
            set_last_error("pinned host allocation failed");
            return DIPL_ERR_OUT_OF_MEMORY;
        }
    }
    return DIPL_OK;
}

template <int B>
static dipl_status launch_ploc_any(const PlocParams& p, int tiles0, cudaStream_t s) {
    return launch_ploc<B>(p, tiles0, s);
}

// Everything on the stream, nothing else: no allocation, no host copy from pageable memory, no synchronisation.
// Scene bounds and code parameters of every mesh (from its triangles).
static dipl_status enqueue_bounds_and_params(BuildPlan& P, cudaStream_t stream) {
    const int m = P.m;
    const long long T = P.T;
    DIPL_CUDA(cudaMemsetAsync(P.d_err, 0, 4, stream));
    bounds_init_kernel<<<blocks_for(m, 128), 128, 0, stream>>>(P.d_bounds, m);
    note_launches();
    {
        long long grid = std::max<long long>(1, std::min<long long>((T + 1023) / 1024, 148 * 16));
        long long chunk = (T + grid - 1) / grid;
        bounds_kernel<<<(unsigned)grid, 256, 0, stream>>>(P.d_meshes, P.d_offsets, m, T, chunk, P.d_bounds);
        note_launches();
    }
    code_params_kernel<<<blocks_for(m, 64), 64, 0, stream>>>(P.d_bounds, m, P.d0.code_type, P.d_params);
    note_launches();
    if (P.d0.code_type == DIPL_CODE_EMC60) {
        emc_tables_kernel<<<(unsigned)m, 256, 0, stream>>>(P.d_params);
        note_launches();
    }
    DIPL_CUDA(cudaGetLastError());
    return DIPL_OK;
}

static dipl_status plan_enqueue(BuildPlan& P, cudaStream_t stream) {
    if (P.m == 0) {
        DIPL_CUDA(cudaMemsetAsync(P.d_err, 0, 4, stream));
        return DIPL_OK;
    }
    const int m = P.m;
    const long long N = P.N, K = P.K;
    const dipl_build_desc& d0 = P.d0;
    dipl_status st;
    if (P.split) {
        // bounds and parameters were enqueued with the piece counts (plan_prepare): the references and their codes
        ref_tri_kernel<<<blocks_for(P.T, 256), 256, 0, stream>>>(P.T, P.pieces, P.piece_first, P.ref_tri);
        note_launches();
        if (P.key_bytes == 4)
            split_refs_kernel<uint32_t><<<blocks_for(N, kSplitThreads), kSplitThreads, 0, stream>>>(
                P.d_meshes, P.d_offsets, m, N, P.ref_tri, P.pieces, P.piece_first, P.d_params, d0.code_type,
                P.code_shift, P.mesh_shift, P.tbox, (uint32_t*)P.keys);
        else
            split_refs_kernel<unsigned long long><<<blocks_for(N, kSplitThreads), kSplitThreads, 0, stream>>>(
                P.d_meshes, P.d_offsets, m, N, P.ref_tri, P.pieces, P.piece_first, P.d_params, d0.code_type,
                P.code_shift, P.mesh_shift, P.tbox, (unsigned long long*)P.keys);
        note_launches();
    } else if ((st = enqueue_bounds_and_params(P, stream)) != DIPL_OK) {
        return st;
    }
    if (!P.split) {  // (the references' codes are written above)
        if (P.key_bytes == 4)
            codes_kernel<uint32_t><<<blocks_for(N, 256), 256, 0, stream>>>(P.d_meshes, P.d_offsets, m, N, P.d_params,
                                                                           d0.code_type, P.code_shift, P.mesh_shift,
                                                                           (uint32_t*)P.keys, P.tbox);
        else
            codes_kernel<unsigned long long><<<blocks_for(N, 256), 256, 0, stream>>>(
                P.d_meshes, P.d_offsets, m, N, P.d_params, d0.code_type, P.code_shift, P.mesh_shift,
                (unsigned long long*)P.keys, P.tbox);
        note_launches();
    }
    DIPL_CUDA(cudaGetLastError());
    st = radix_sort_pairs(P.keys, nullptr, P.keys_sorted, P.perm, P.keys_alt, P.perm_alt, N, P.key_bytes, 0,
                          P.key_bits, P.digit_bits, P.sort_scratch, stream, P.d_err);
    if (st != DIPL_OK) return st;

    // ---- PLOC ------------------------------------------------------------------------------------------
    PlocParams pp{};
    DIPL_CUDA(cudaMemsetAsync(P.d_ctrl, 0, sizeof(PlocCtrl), stream));
    const bool hier = d0.clustering == DIPL_CLUSTER_HPLOC;
    ploc_ctrl_init_kernel<<<1, 1, 0, stream>>>(P.d_ctrl, (uint32_t)N, hier ? 1u : 0u);
    note_launches();
    if (!hier)
        DIPL_CUDA(cudaMemsetAsync(P.status, 0, sizeof(unsigned long long) * (2 * P.tiles_max + 2), stream));
    fill_int_kernel<<<blocks_for(N + K, 256), 256, 0, stream>>>(P.parent, N + K, -1);
    note_launches();
    ploc_init_kernel<<<blocks_for(N, 256), 256, 0, stream>>>(P.d_meshes, P.d_coffsets, m, N, P.perm, P.tbox,
                                                             P.c_lo[0], P.c_hi[0], P.c_in[0], P.parent);
    note_launches();
    DIPL_CUDA(cudaGetLastError());
    if (hier) {
        DIPL_CUDA(cudaMemsetAsync(P.hp_other, 0xFF, sizeof(int) * N, stream));
        HplocParams hp{};
        hp.keys = P.keys_sorted, hp.offsets = P.d_coffsets;
        hp.lo = P.c_lo[0], hp.hi = P.c_hi[0], hp.info = P.c_in[0];
        hp.child = P.child, hp.node_lo = P.nlo, hp.node_hi = P.nhi, hp.parent = P.parent;
        hp.other = P.hp_other, hp.cnt = P.hp_cnt, hp.fid = P.hp_fid;
        hp.root_lo = P.c_lo[1], hp.root_hi = P.c_hi[1];
        hp.ctrl = P.d_ctrl, hp.err = P.d_err;
        hp.num_leaves = (int)N, hp.num_inner = (int)K, hp.num_meshes = m, hp.radius = d0.nn_search_radius;
        hp.max_node_iterations = clustering_iteration_limit() ? (int)clustering_iteration_limit() : 64;
        const unsigned grid = blocks_for(N, kHplocThreads);
        if (P.key_bytes == 4) hploc_kernel<uint32_t><<<grid, kHplocThreads, 0, stream>>>(hp);
        else hploc_kernel<unsigned long long><<<grid, kHplocThreads, 0, stream>>>(hp);
        note_launches();
        DIPL_CUDA(cudaGetLastError());
    }
    pp.lo[0] = P.c_lo[0], pp.hi[0] = P.c_hi[0], pp.lo[1] = P.c_lo[1], pp.hi[1] = P.c_hi[1];
    pp.info[0] = P.c_in[0], pp.info[1] = P.c_in[1];
    pp.child = P.child, pp.node_lo = P.nlo, pp.node_hi = P.nhi, pp.parent = P.parent;
    pp.status[0] = P.status, pp.status[1] = P.status + P.tiles_max + 1;
    pp.ctrl = P.d_ctrl, pp.err = P.d_err;
    pp.num_leaves = (int)N, pp.num_meshes = m, pp.radius = d0.nn_search_radius;
    pp.max_iterations = clustering_iteration_limit() ? clustering_iteration_limit() : kMaxPlocIterations;
    const int mid_ctas = hier ? 0 : ploc_mid_ctas();
    pp.grid_stop = mid_ctas > 0 ? mid_ctas * kMidSlice : kTailMax;
    if (!hier && N > m && N > pp.grid_stop) {
        switch (P.B) {
            case 128: st = launch_ploc_any<128>(pp, P.tiles0, stream); break;
            case 512: st = launch_ploc_any<512>(pp, P.tiles0, stream); break;
            default: st = launch_ploc_any<256>(pp, P.tiles0, stream); break;
        }
        if (st != DIPL_OK) return st;
    }
    if (!hier && N > m && N > kTailMax && mid_ctas > 0 && (st = launch_ploc_mid(pp, mid_ctas, stream)) != DIPL_OK)
        return st;
    if (!hier && N > m && (st = launch_ploc_tail(pp, stream)) != DIPL_OK) return st;

    // ---- layout -------------------------------------------------------------------------------------
    LayoutParams LP{P.child, P.nlo, P.nhi, P.parent, (int)N, (int)K, P.L};
    DIPL_CUDA(cudaMemsetAsync(P.d_sah, 0, sizeof(double) * 2 * m, stream));
    DIPL_CUDA(cudaMemsetAsync(P.d_counts, 0, 16, stream));
    if (K > 0) {
        inner_flags_kernel<<<blocks_for(K, 256), 256, 0, stream>>>(LP, P.rev_flags, P.d_err);
        note_launches();
        if ((st = exclusive_scan_u32(P.rev_flags, P.rev_flags, K, P.d_counts, P.scan_scratch, stream, P.d_err)) !=
            DIPL_OK)
            return st;
        if (hier) {
            // Hierarchical ids follow split positions, so reverse id order would scatter the tree's top levels over
            // the whole node array. Number the inner nodes by height instead, the tallest (the roots) first, ties
            // by id: the top levels every ray visits sit together at the front, as with the global loop's reverse
            // creation order. A one-pass stable sort of 8-bit keys (255 - height; 255 for nodes inside leaves).
            uint32_t* hkeys = reinterpret_cast<uint32_t*>(P.keys);
            uint32_t* hsorted = reinterpret_cast<uint32_t*>(P.keys_sorted);
            height_keys_kernel<<<blocks_for(K, 256), 256, 0, stream>>>(LP, hkeys, P.d_err);
            note_launches();
            DIPL_CUDA(cudaGetLastError());
            if ((st = radix_sort_pairs(hkeys, nullptr, hsorted, P.perm_alt, P.keys_alt, P.contrib, K, 4, 0, 8, 8,
                                       P.sort_scratch, stream, P.d_err)) != DIPL_OK)
                return st;
            height_index_kernel<<<blocks_for(K, 256), 256, 0, stream>>>(LP, P.perm_alt, P.rev_flags, P.d_err);
            note_launches();
        }
    }
    leaf_owner_kernel<<<blocks_for(N, 256), 256, 0, stream>>>(LP, P.contrib, P.owner_leaf, P.d_err);
    note_launches();
    if ((st = exclusive_scan_u32(P.contrib, P.contrib, N, nullptr, P.scan_scratch, stream, P.d_err)) != DIPL_OK)
        return st;
    leaf_write_kernel<<<blocks_for(N, 256), 256, 0, stream>>>(LP, P.d_meshes, P.d_offsets, m, P.perm, P.ref_tri,
                                                               P.contrib, P.leaf_start_of, P.tris, P.slot_pos, P.d_err);
    note_launches();
    if (K > 0) {
        node_write_kernel<<<blocks_for(K, 256), 256, 0, stream>>>(LP, P.tbox, P.d_coffsets, m, P.perm, P.rev_flags,
                                                                   P.leaf_start_of, P.nodes, P.d_sah, P.d_err);
        note_launches();
    }
    roots_kernel<<<blocks_for(m, 64), 64, 0, stream>>>(LP, P.c_lo[0], P.c_hi[0], P.c_lo[1], P.c_hi[1], P.d_ctrl, m,
                                                       P.rev_flags, P.leaf_start_of, P.d_roots, P.d_err);
    note_launches();
    DIPL_CUDA(cudaGetLastError());
    if (d0.bv_type == DIPL_BV_SOBB) {
        SobbRefs refs;
        if (P.split) refs = SobbRefs{P.slot_pos, P.perm, P.tbox};
        st = sobb_enqueue(P.child, P.nlo, P.nhi, P.parent, P.leaf_start_of, P.owner_leaf, P.tris, P.nodes, P.rev_flags,
                          (int)N, (int)K, P.L, d0.kdop_size, P.sobb, refs, P.snodes, stream, P.d_err);
        if (st != DIPL_OK) return st;
    }
    // ---- the per-mesh summary to pinned host memory --------------------------------------------------
    RootInfo* h_roots = reinterpret_cast<RootInfo*>(P.h_summary);
    double* h_sah = reinterpret_cast<double*>(P.h_summary + sizeof(RootInfo) * m);
    uint32_t* h_tail = reinterpret_cast<uint32_t*>(P.h_summary + sizeof(RootInfo) * m + sizeof(double) * 2 * m);
    DIPL_CUDA(cudaMemcpyAsync(h_roots, P.d_roots, sizeof(RootInfo) * m, cudaMemcpyDeviceToHost, stream));
    DIPL_CUDA(cudaMemcpyAsync(h_sah, P.d_sah, sizeof(double) * 2 * m, cudaMemcpyDeviceToHost, stream));
    DIPL_CUDA(cudaMemcpyAsync(h_tail, P.d_counts, 4, cudaMemcpyDeviceToHost, stream));
    DIPL_CUDA(cudaMemcpyAsync(h_tail + 1, &P.d_ctrl->iterations, 4, cudaMemcpyDeviceToHost, stream));
    DIPL_CUDA(cudaMemcpyAsync(h_tail + 2, P.d_err, 4, cudaMemcpyDeviceToHost, stream));
    return DIPL_OK;
}

// After the stream synchronised: check the error word, build the 8-wide layout if asked, make the handles.
static dipl_status plan_finish(BuildPlan& P, dipl_bvh** out, bool allow_wide) {
    const int m = P.m;
    const dipl_build_desc& d0 = P.d0;
    auto make_handle = [&](int i) {
        auto* h = new dipl_bvh();
        h->storage = P.out;
        h->num_triangles = P.descs[i].num_triangles;
        h->code_type = P.descs[i].code_type;
        h->bv_type = P.descs[i].bv_type;
        h->layout = P.descs[i].layout;
        h->max_leaf = P.descs[i].max_triangles_per_leaf;
        h->radius = P.descs[i].nn_search_radius;
        h->kdop = P.descs[i].kdop_size;
        h->clustering = P.descs[i].clustering;
        h->d_err = P.d_err;
        h->root = 0;
        return h;
    };
    if (m == 0) {
        for (int i = 0; i < P.count; ++i) out[i] = make_handle(i);
        return DIPL_OK;
    }
    const RootInfo* h_roots = reinterpret_cast<const RootInfo*>(P.h_summary);
    const double* h_sah = reinterpret_cast<const double*>(P.h_summary + sizeof(RootInfo) * m);
    const uint32_t* h_tail =
        reinterpret_cast<const uint32_t*>(P.h_summary + sizeof(RootInfo) * m + sizeof(double) * 2 * m);
    const uint32_t err = h_tail[2];
    if (err != 0u) {
        set_last_error(err & kErrTimeout ? "build: a bounded device wait timed out"
                                         : "build: clustering did not converge");
        return (err & kErrTimeout) ? DIPL_ERR_TIMEOUT : DIPL_ERR_INTERNAL;
    }
    const int64_t inner_total = (int64_t)h_tail[0];
    const int iterations = (int)h_tail[1];
    WNode* wnodes = nullptr;
    float4* wtris = nullptr;
    int64_t wcount = 0;
    std::vector<int> wroots, wlevels;
    if (d0.layout == DIPL_LAYOUT_WIDE8_Q8) {
        if (!allow_wide) {
            set_last_error("the 8-wide layout cannot be captured in a build plan (it reads level sizes back)");
            return DIPL_ERR_UNSUPPORTED;
        }
        std::vector<int> root_ids(m), root_counts(m);
        for (int k = 0; k < m; ++k) root_ids[k] = h_roots[k].root_id, root_counts[k] = h_roots[k].num_leaves;
        dipl_status st = build_wide(P.child, P.nlo, P.nhi, P.leaf_start_of, P.tris, (int)P.N, P.L, root_ids,
                                    root_counts, *P.out, P.stream, P.d_err, &wnodes, &wtris, &wcount, wroots, wlevels);
        if (st != DIPL_OK) return st;
    }
    for (int i = 0; i < P.count; ++i) {
        dipl_bvh* h = make_handle(i);
        h->nodes = d0.bv_type == DIPL_BV_SOBB ? static_cast<void*>(P.snodes) : static_cast<void*>(P.nodes);
        h->tris = P.tris;
        h->perm = reinterpret_cast<int32_t*>(P.perm);
        h->children = P.child;
        h->node_lo = P.nlo;
        h->node_hi = P.nhi;
        h->batch_leaves = P.N;
        h->batched = P.m > 1;
        h->ref_tri = P.ref_tri;
        h->node_capacity = inner_total;
        h->ploc_iterations = iterations;
        const int k = P.mesh_of_desc[i];
        if (k >= 0) {
            const RootInfo& ri = h_roots[k];
            h->root = ri.root_ref;
            h->depth = ri.depth;
            h->leaf_base = P.coffsets[k];
            h->num_refs = P.coffsets[k + 1] - P.coffsets[k];
            h->num_nodes = (int64_t)h_sah[2 * k + 1];
            h->sah_area = ri.root_area;
            h->sah_sum = h_sah[2 * k] + ri.leaf_cost;
            if (d0.layout == DIPL_LAYOUT_WIDE8_Q8) {
                h->root = wroots[k];
                h->depth = wlevels[k];
            }
        }
        if (d0.layout == DIPL_LAYOUT_WIDE8_Q8) {
            h->nodes = wnodes;
            h->tris = wtris;
            h->node_size = sizeof(WNode);
            h->node_capacity = wcount;
            h->num_nodes = wcount;
        }
        out[i] = h;
    }
    return DIPL_OK;
}

dipl_status build_batched(const dipl_build_desc* descs, int count, dipl_bvh** out, cudaStream_t stream) {
    DIPL_CHECK_ARG(descs && out && count >= 1, "descs/out must be non-NULL and count >= 1");
    for (int i = 0; i < count; ++i) out[i] = nullptr;
    BuildPlan P;
    dipl_status st = plan_prepare(P, descs, count, stream, false);
    if (st != DIPL_OK) return st;
    if ((st = plan_enqueue(P, stream)) != DIPL_OK) return st;
    if (P.m > 0) DIPL_CUDA(cudaStreamSynchronize(stream));  // the build's one host synchronisation
    return plan_finish(P, out, true);
}

}  // namespace dipl

// ---- build plans: a batch captured once into a CUDA graph and replayed ---------------------------------
struct dipl_build_plan {
    dipl::BuildPlan plan;
};

namespace dipl {

dipl_status plan_create(const dipl_build_desc* descs, int count, dipl_build_plan** out, cudaStream_t stream) {
    DIPL_CHECK_ARG(out != nullptr, "out must be non-NULL");
    *out = nullptr;
    auto holder = std::make_unique<dipl_build_plan>();
    BuildPlan& P = holder->plan;
    for (int i = 0; i < count && descs; ++i)
        if (descs[i].split_budget != 0) {
            // the pieces depend on the vertex positions, which a plan's replays may change
            set_last_error("pre-splitting (split_budget > 0) cannot be captured in a build plan");
            return DIPL_ERR_UNSUPPORTED;
        }
    dipl_status st = plan_prepare(P, descs, count, stream, true);
    if (st != DIPL_OK) return st;
    if (P.d0.layout == DIPL_LAYOUT_WIDE8_Q8) {
        set_last_error("the 8-wide layout cannot be captured in a build plan (it reads level sizes back)");
        return DIPL_ERR_UNSUPPORTED;
    }
    // run once eagerly (sets kernel attributes, validates), then capture the same sequence
    if ((st = plan_enqueue(P, stream)) != DIPL_OK) return st;
    DIPL_CUDA(cudaStreamSynchronize(stream));
    cudaStream_t cap;
    DIPL_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        st = plan_enqueue(P, cap);
        cudaGraph_t g = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(cap, &g);
        if (st == DIPL_OK && e2 != cudaSuccess) st = cuda_status(e2, "cudaStreamEndCapture");
        if (st == DIPL_OK) {
            P.graph = g;
            e2 = cudaGraphInstantiate(&P.graph_exec, g, 0);
            if (e2 != cudaSuccess) st = cuda_status(e2, "cudaGraphInstantiate");
            size_t nn = 0;
            if (st == DIPL_OK && cudaGraphGetNodes(g, nullptr, &nn) == cudaSuccess && nn > 0) {
                std::vector<cudaGraphNode_t> nodes_(nn);
                if (cudaGraphGetNodes(g, nodes_.data(), &nn) == cudaSuccess)
                    for (auto nd : nodes_) {
                        cudaGraphNodeType t;
                        if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++P.graph_kernels;
                    }
            }
        } else if (g) {
            cudaGraphDestroy(g);
        }
    } else {
        st = cuda_status(e, "cudaStreamBeginCapture");
    }
    cudaStreamDestroy(cap);
    if (st != DIPL_OK) return st;
    *out = holder.release();
    return DIPL_OK;
}

dipl_status plan_launch(dipl_build_plan* plan, cudaStream_t stream) {
    DIPL_CHECK_ARG(plan != nullptr, "plan must be non-NULL");
    if (plan->plan.m == 0) return DIPL_OK;
    DIPL_CUDA(cudaGraphLaunch(plan->plan.graph_exec, stream));
    note_launches(plan->plan.graph_kernels);
    return DIPL_OK;
}

dipl_status plan_get_bvhs(dipl_build_plan* plan, dipl_bvh** out, cudaStream_t stream) {
    DIPL_CHECK_ARG(plan && out, "plan/out must be non-NULL");
    DIPL_CUDA(cudaStreamSynchronize(stream));
    return plan_finish(plan->plan, out, false);
}

void plan_destroy(dipl_build_plan* plan) { delete plan; }

}  // namespace dipl

namespace dipl {

// Codes of one mesh, as the build computes them (without mesh bits).
dipl_status compute_codes(const dipl_build_desc* desc, void* d_codes, cudaStream_t stream) {
    DIPL_CHECK_ARG(desc != nullptr, "desc must be non-NULL");
    dipl_status st = validate_desc(*desc);
    if (st != DIPL_OK) return st;
    const long long N = desc->num_triangles;
    if (N == 0) return DIPL_OK;
    DIPL_CHECK_ARG(d_codes != nullptr, "codes must be non-NULL");
    ScratchArena scratch(stream);
    MeshDesc md{desc->d_v0, desc->d_v1, desc->d_v2, 0, N};
    long long offs[2] = {0, N};
    MeshDesc* d_meshes;
    long long* d_offsets;
    Bounds* d_bounds;
    CodeParams* d_params;
    if ((st = scratch.alloc(&d_meshes, 1)) != DIPL_OK || (st = scratch.alloc(&d_offsets, 2)) != DIPL_OK ||
        (st = scratch.alloc(&d_bounds, 1)) != DIPL_OK || (st = scratch.alloc(&d_params, 1)) != DIPL_OK)
        return st;
    DIPL_CUDA(cudaMemcpyAsync(d_meshes, &md, sizeof(md), cudaMemcpyHostToDevice, stream));
    DIPL_CUDA(cudaMemcpyAsync(d_offsets, offs, sizeof(offs), cudaMemcpyHostToDevice, stream));
    bounds_init_kernel<<<1, 32, 0, stream>>>(d_bounds, 1); note_launches();
    long long grid = std::max<long long>(1, std::min<long long>((N + 1023) / 1024, 148 * 16));
    long long chunk = (N + grid - 1) / grid;
    bounds_kernel<<<(unsigned)grid, 256, 0, stream>>>(d_meshes, d_offsets, 1, N, chunk, d_bounds); note_launches();
    code_params_kernel<<<1, 32, 0, stream>>>(d_bounds, 1, desc->code_type, d_params); note_launches();
    if (desc->code_type == DIPL_CODE_EMC60) {
        emc_tables_kernel<<<1, 256, 0, stream>>>(d_params);
        note_launches();
    }
    if (desc->code_type == DIPL_CODE_MORTON30)
        codes_kernel<uint32_t><<<blocks_for(N, 256), 256, 0, stream>>>(d_meshes, d_offsets, 1, N, d_params,
                                                                       desc->code_type, 0, 0, (uint32_t*)d_codes,
                                                                       nullptr);
    else
        codes_kernel<unsigned long long><<<blocks_for(N, 256), 256, 0, stream>>>(
            d_meshes, d_offsets, 1, N, d_params, desc->code_type, 0, 0, (unsigned long long*)d_codes, nullptr);
    note_launches();
    DIPL_CUDA(cudaGetLastError());
    // keep the scratch alive until the kernels ran (frees are stream-ordered)
    return DIPL_OK;
}

}  // namespace dipl
