// Single-pass exclusive prefix sum of uint32 (decoupled look-back across 2048-element tiles,
// bounded spin). Used by the BVH layout to number nodes and place leaf triangle ranges.
#include "internal.h"

namespace dipl {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr unsigned long long kAgg = 1ull << 62;
constexpr unsigned long long kInc = 2ull << 62;

__global__ void __launch_bounds__(kScanThreads) scan_kernel(const uint32_t* in, uint32_t* out,
                                                            int64_t n, unsigned long long* __restrict__ status,
                                                            uint32_t* __restrict__ tile_counter, uint32_t* d_total,
                                                            uint32_t* __restrict__ err) {
    __shared__ uint32_t s_tile;
    __shared__ unsigned long long s_warp[kScanThreads / 32];
    __shared__ unsigned long long s_prefix;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const int64_t base = (int64_t)tile * kScanTile + (int64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    unsigned long long local = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        int64_t i = base + k;
        v[k] = i < n ? in[i] : 0u;
        local += v[k];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long x = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    unsigned long long woff = 0, total = 0;
    for (int w = 0; w < kScanThreads / 32; ++w) {
        unsigned long long t = s_warp[w];
        if (w < warp) woff += t;
        total += t;
    }
    if (threadIdx.x < 32) {
        unsigned long long prefix = 0;
        bool ok = true;
        if (tile == 0) {
            if (threadIdx.x == 0) st_release_u64(&status[0], kInc | total);
        } else {
            if (threadIdx.x == 0) st_release_u64(&status[tile], kAgg | total);
            prefix = warp_lookback(status, tile, err, &ok);
            if (threadIdx.x == 0 && ok) st_release_u64(&status[tile], kInc | (prefix + total));
        }
        if (threadIdx.x == 0) {
            s_prefix = ok ? prefix : 0ull;
            if (d_total && (int64_t)(tile + 1) * kScanTile >= n) *d_total = (uint32_t)(prefix + total);
        }
    }
    __syncthreads();
    unsigned long long run = s_prefix + woff + (x - local);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        int64_t i = base + k;
        if (i < n) out[i] = (uint32_t)run;
        run += v[k];
    }
}

}  // namespace

size_t scan_scratch_bytes(int64_t n) {
    int64_t tiles = (n + kScanTile - 1) / kScanTile;
    return (size_t)tiles * 8 + 64;
}

dipl_status exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* d_total, void* scratch,
                               cudaStream_t stream, uint32_t* d_err) {
    if (n <= 0) {
        if (d_total) DIPL_CUDA(cudaMemsetAsync(d_total, 0, 4, stream));
        return DIPL_OK;
    }
    int64_t tiles = (n + kScanTile - 1) / kScanTile;
    auto* counter = static_cast<uint32_t*>(scratch);
    auto* status = reinterpret_cast<unsigned long long*>(static_cast<unsigned char*>(scratch) + 64);
    DIPL_CUDA(cudaMemsetAsync(scratch, 0, scan_scratch_bytes(n), stream));
    scan_kernel<<<(unsigned)tiles, kScanThreads, 0, stream>>>(in, out, n, status, counter, d_total, d_err); note_launches();
    DIPL_CUDA(cudaGetLastError());
    return DIPL_OK;
}

}  // namespace dipl
