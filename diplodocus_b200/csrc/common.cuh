// Shared device/host helpers of the B200 BVH engine (sm_100a only).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "dipl_bvh.h"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "libdipl_bvh is built for sm_100a (B200) only"
#endif

namespace dipl {

// ------------------------------------------------------------------------------------------------
// Constants of the reference's intersection arithmetic (src/util/util.h:15-16).
// ------------------------------------------------------------------------------------------------
constexpr float kEpsilon = 1e-6f;
constexpr float kInfinity = 3.40282346638528859812e+38f;  // FLT_MAX, the reference's "miss" t

// Bounded spins: every device-side wait gives up after this many polls (with __nanosleep back-off,
// well over a second), records an error word and lets the kernel return.
constexpr uint32_t kSpinLimit = 1u << 24;

// Device error word bits (host maps them to dipl_status).
constexpr uint32_t kErrTimeout = 1u;
constexpr uint32_t kErrStack = 2u;
constexpr uint32_t kErrIterations = 4u;

// Leaf references inside nodes: ref >= 0 is a node index; ref < 0 is ~((first_tri << 3) | count).
constexpr int kLeafCountBits = 3;
__host__ __device__ __forceinline__ int make_leaf_ref(int first, int count) {
    return ~((first << kLeafCountBits) | count);
}
__host__ __device__ __forceinline__ int leaf_first(int ref) { return (~ref) >> kLeafCountBits; }
__host__ __device__ __forceinline__ int leaf_count(int ref) { return (~ref) & ((1 << kLeafCountBits) - 1); }

// Binary FP32 node: both child boxes + references (64 bytes, four 16-byte loads).
struct __align__(16) BNode {
    float4 a;  // left  lo.x hi.x lo.y hi.y
    float4 b;  // right lo.x hi.x lo.y hi.y
    float4 c;  // left lo.z hi.z, right lo.z hi.z
    int4 d;    // left ref, right ref, unused, unused
};
static_assert(sizeof(BNode) == 64, "BNode must be 64 bytes");

// Binary SOBB node (64 bytes): per child three slab directions (indices into the direction table)
// and the slab intervals along them.
struct __align__(16) SNode {
    float4 a;  // left  lo0 hi0 lo1 hi1
    float4 b;  // left  lo2 hi2, right lo0 hi0
    float4 c;  // right lo1 hi1 lo2 hi2
    int4 d;    // left ref, right ref, left axes (3 x 8 bits), right axes (3 x 8 bits)
};
static_assert(sizeof(SNode) == 64, "SNode must be 64 bytes");

// 8-wide node with 8-bit quantised child bounds (80 bytes), after Ylitie, Karras & Laine (HPG 2017).
struct __align__(16) WNode {
    float px, py, pz;          // quantisation origin
    unsigned char ex, ey, ez;  // power-of-two scale exponents (biased by 127, like float exponents)
    unsigned char imask;       // bit i: child slot i is an inner node
    int child_base;            // index of the first inner child node
    int tri_base;              // index of the first triangle of the node's leaves
    unsigned char meta[8];     // per slot: 0 = empty; inner: 0b001 << 5 | (24 + rank); leaf: unary count << 5 | tri offset
    unsigned char qlox[8], qloy[8], qloz[8];
    unsigned char qhix[8], qhiy[8], qhiz[8];
};
static_assert(sizeof(WNode) == 80, "WNode must be 80 bytes");

// ------------------------------------------------------------------------------------------------
// Device helpers.
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ int float_to_ordered(float f) {
    int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float ordered_to_float(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7FFFFFFF); }

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Grid-wide barrier for co-resident (cooperatively launched) blocks: sense by generation count,
// bounded spin. Returns false (and sets *err) if it gave up.
struct GridBarrier {
    uint32_t count;
    uint32_t generation;
};

// `expected` = number of blocks taking part (the same value in every participating block).
__device__ __forceinline__ bool grid_barrier(GridBarrier* bar, uint32_t expected, uint32_t* err,
                                             uint32_t spin_limit = kSpinLimit) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        uint32_t gen = ld_acquire_u32(&bar->generation);
        __threadfence();
        uint32_t arrived = atomicAdd(&bar->count, 1u);
        if (arrived == expected - 1) {
            atomicExch(&bar->count, 0u);
            __threadfence();
            st_release_u32(&bar->generation, gen + 1u);
        } else {
            uint32_t spins = 0;
            while (ld_acquire_u32(&bar->generation) == gen) {
                if (++spins > spin_limit || ld_acquire_u32(err) != 0u) {
                    atomicOr(err, kErrTimeout);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

// Warp-parallel decoupled look-back (call with all 32 lanes of one warp). `status[j]` holds a 64-bit word:
// state in the top two bits (0 = not ready, 1 = aggregate of tile j, 2 = inclusive prefix through tile j)
// and a value in the low 62 bits; values add without carries between packed fields. Returns the exclusive
// prefix of `tile`, reading 32 predecessors per round trip. Bounded: on timeout sets *err and *ok = false.
__device__ __forceinline__ unsigned long long warp_lookback(const unsigned long long* status, long long tile,
                                                            uint32_t* err, bool* ok,
                                                            uint32_t spin_limit = kSpinLimit) {
    constexpr unsigned long long kVal = (1ull << 62) - 1ull;
    const int lane = threadIdx.x & 31;
    unsigned long long prefix = 0;
    long long j = tile - 1;
    uint32_t spins = 0;
    *ok = true;
    while (j >= 0) {
        const long long idx = j - lane;
        const unsigned long long w = idx >= 0 ? ld_acquire_u64(status + idx) : (2ull << 62);
        const unsigned long long state = w >> 62;
        const uint32_t inc = __ballot_sync(0xffffffffu, state == 2ull);
        const uint32_t zero = __ballot_sync(0xffffffffu, state == 0ull);
        const int lim = inc ? __ffs(inc) - 1 : 31;
        const uint32_t upto = lim == 31 ? 0xffffffffu : ((2u << lim) - 1u);
        if (zero & upto) {
            if (++spins > spin_limit) {
                if (lane == 0) atomicOr(err, kErrTimeout);
                *ok = false;
                return 0ull;
            }
            __nanosleep(20);
            continue;
        }
        unsigned long long v = lane <= lim ? (w & kVal) : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        prefix += v;
        if (inc) break;
        j -= 32;
    }
    return prefix;
}

// Block-wide decoupled look-back (call with every thread of the block; same status layout as warp_lookback).
// Thread t polls predecessor `tile - 1 - t`, so one round trip covers B predecessors: when all tiles of a
// round run at once, the inclusive-prefix frontier then advances B tiles per round trip instead of 32.
// `wsum` / `wflag` are shared scratch of B/32 entries. Returns the same value in every thread.
template <int B>
__device__ __forceinline__ unsigned long long block_lookback(const unsigned long long* status, long long tile,
                                                             uint32_t* err, bool* ok, unsigned long long* wsum,
                                                             int* wflag, uint32_t spin_limit = kSpinLimit) {
    constexpr unsigned long long kVal = (1ull << 62) - 1ull;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long prefix = 0;
    long long j = tile - 1;
    uint32_t spins = 0;
    *ok = true;
    for (;;) {
        const long long idx = j - (long long)threadIdx.x;
        // positions before tile 0 read as an inclusive prefix of zero
        const unsigned long long w = idx >= 0 ? ld_acquire_u64(status + idx) : (2ull << 62);
        const unsigned long long state = w >> 62;
        const uint32_t inc = __ballot_sync(0xffffffffu, state == 2ull);
        const uint32_t zero = __ballot_sync(0xffffffffu, state == 0ull);
        const int lim = inc ? __ffs(inc) - 1 : 31;
        const uint32_t upto = lim == 31 ? 0xffffffffu : ((2u << lim) - 1u);
        unsigned long long v = lane <= lim ? (w & kVal) : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) {
            wsum[warp] = v;
            wflag[warp] = (zero & upto) ? 2 : (inc ? 1 : 0);  // 2: not ready, 1: reached an inclusive prefix
        }
        __syncthreads();
        // every thread combines the warps nearest first (same result everywhere, no second pass)
        unsigned long long s = 0;
        int code = 0;
#pragma unroll
        for (int wi = 0; wi < B / 32; ++wi) {
            const int f = wflag[wi];
            if (f == 2) {
                code = 2;
                break;
            }
            s += wsum[wi];
            if (f == 1) {
                code = 1;
                break;
            }
        }
        __syncthreads();  // scratch is rewritten by the next round
        if (code == 2) {
            if (++spins > spin_limit) {
                if (threadIdx.x == 0) atomicOr(err, kErrTimeout);
                *ok = false;
                return 0ull;
            }
            __nanosleep(20);
            continue;
        }
        prefix += s;
        if (code == 1) break;
        j -= B;
    }
    return prefix;
}

// Surface-area-like distance of PLOC: half the area of the union box, evaluated with fixed FMAs so
// the host restatement (oracle/dipl_oracle.c ploc_key) rounds identically. NaN counts as +inf.
__device__ __forceinline__ float ploc_distance(float lx0, float ly0, float lz0, float hx0, float hy0, float hz0,
                                               float lx1, float ly1, float lz1, float hx1, float hy1, float hz1) {
    float dx = __fsub_rn(fmaxf(hx0, hx1), fminf(lx0, lx1));
    float dy = __fsub_rn(fmaxf(hy0, hy1), fminf(ly0, ly1));
    float dz = __fsub_rn(fmaxf(hz0, hz1), fminf(lz0, lz1));
    float d = __fmaf_rn(dx, dy, __fmaf_rn(dy, dz, __fmul_rn(dz, dx)));
    return (d != d) ? __int_as_float(0x7F800000) : d;
}

}  // namespace dipl

// ------------------------------------------------------------------------------------------------
// Host-side error plumbing (thread-local last error).
// ------------------------------------------------------------------------------------------------
namespace dipl {
void set_last_error(const std::string& msg);
dipl_status cuda_status(cudaError_t e, const char* what);
}  // namespace dipl

#define DIPL_CUDA(call)                                                        \
    do {                                                                       \
        cudaError_t _e = (call);                                               \
        if (_e != cudaSuccess) return ::dipl::cuda_status(_e, #call);          \
    } while (0)

#define DIPL_CHECK_ARG(cond, msg)                                              \
    do {                                                                       \
        if (!(cond)) {                                                         \
            ::dipl::set_last_error(msg);                                       \
            return DIPL_ERR_INVALID_ARGUMENT;                                  \
        }                                                                      \
    } while (0)
