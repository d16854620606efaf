// Stable LSD radix sort of (key, uint32 value) pairs, one kernel per digit (onesweep scheme of
// Adinets & Merrill 2022): an up-front histogram kernel counts every digit of every pass in one read
// of the keys; each pass kernel then ranks a 4096-key tile with warp-level match_any multisplit,
// resolves its global digit offsets by decoupled look-back over earlier tiles (bounded spin), and
// scatters through shared memory so the global writes come out in digit runs.
#include "internal.h"

namespace dipl {
namespace {

// 512 threads x 8 keys: few registers per thread (at most 64, so 3 tiles of 16 warps share an SM) keep
// enough loads in flight to hide memory latency.
constexpr int kSortThreads = 512;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 keys
constexpr int kMaxPasses = 11;

// Look-back word: 2-bit state in the top bits, 30-bit count below.
constexpr uint32_t kLbAggregate = 1u << 30;
constexpr uint32_t kLbInclusive = 2u << 30;
constexpr uint32_t kLbCountMask = (1u << 30) - 1u;

template <typename K>
__device__ __forceinline__ uint32_t digit_of(K key, int shift, uint32_t mask) {
    return static_cast<uint32_t>(key >> shift) & mask;
}

template <typename K, int BITS>
__global__ void __launch_bounds__(256) histogram_kernel(const K* __restrict__ keys, int64_t n, int begin_bit,
                                                        int end_bit, int passes, uint32_t* __restrict__ hist) {
    constexpr int BINS = 1 << BITS;
    extern __shared__ uint32_t s_hist[];  // [passes][BINS]
    for (int i = threadIdx.x; i < passes * BINS; i += blockDim.x) s_hist[i] = 0u;
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        K key = keys[i];
        for (int p = 0; p < passes; ++p) {
            int shift = begin_bit + p * BITS;
            int width = min(BITS, end_bit - shift);
            uint32_t d = digit_of(key, shift, (1u << width) - 1u);
            atomicAdd(&s_hist[p * BINS + d], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * BINS; i += blockDim.x) {
        uint32_t c = s_hist[i];
        if (c) atomicAdd(&hist[i], c);
    }
}

// Block-wide exclusive scan of `count` values in shared memory (count <= 1025), in place; returns total.
__device__ uint32_t block_exclusive_scan_smem(uint32_t* vals, int count) {
    __shared__ uint32_t s_warp[kSortWarps];
    const int per = (count + kSortThreads - 1) / kSortThreads;
    const int beg = threadIdx.x * per;
    uint32_t local = 0;
    for (int i = 0; i < per; ++i)
        if (beg + i < count) local += vals[beg + i];
    // warp inclusive scan of local
    uint32_t x = local;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    uint32_t warp_off = 0, total = 0;
    for (int w = 0; w < kSortWarps; ++w) {
        uint32_t v = s_warp[w];
        if (w < warp) warp_off += v;
        total += v;
    }
    uint32_t run = warp_off + x - local;
    __syncthreads();
    for (int i = 0; i < per; ++i) {
        if (beg + i < count) {
            uint32_t v = vals[beg + i];
            vals[beg + i] = run;
            run += v;
        }
    }
    __syncthreads();
    return total;
}

template <typename K, int BITS>
struct SortSmem {
    static constexpr int BINS = 1 << BITS;
    K keys[kSortTile];
    uint32_t vals[kSortTile];
    uint32_t whist[kSortWarps][BINS + 1];
    uint32_t dtotal[BINS + 1];
    uint32_t gexcl[BINS];
    int32_t gofs[BINS];
    uint32_t tile;
};

template <typename K, int BITS>
__global__ void __launch_bounds__(kSortThreads, 2) onesweep_kernel(
    const K* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, K* __restrict__ keys_out,
    uint32_t* __restrict__ vals_out, int64_t n, int shift, int width, const uint32_t* __restrict__ pass_hist,
    uint32_t* __restrict__ lookback, uint32_t* __restrict__ tile_counter, uint32_t* __restrict__ err) {
    constexpr int BINS = 1 << BITS;
    extern __shared__ __align__(16) unsigned char s_raw[];
    SortSmem<K, BITS>& s = *reinterpret_cast<SortSmem<K, BITS>*>(s_raw);
    const uint32_t mask = (1u << width) - 1u;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    if (threadIdx.x == 0) s.tile = atomicAdd(tile_counter, 1u);
    for (int i = threadIdx.x; i < kSortWarps * (BINS + 1); i += kSortThreads) (&s.whist[0][0])[i] = 0u;
    for (int d = threadIdx.x; d < BINS; d += kSortThreads) s.gexcl[d] = pass_hist[d];
    __syncthreads();
    block_exclusive_scan_smem(s.gexcl, BINS);  // global exclusive digit starts of this pass
    const uint32_t tile = s.tile;
    const int64_t base = (int64_t)tile * kSortTile;

    // ---- load (warp-striped: coalesced) and rank within the warp --------------------------------
    K key[kSortItems];
    uint32_t val[kSortItems];
    uint32_t dig[kSortItems];
    uint32_t rank[kSortItems];
    const int64_t wbase = base + (int64_t)warp * 32 * kSortItems;
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        int64_t idx = wbase + k * 32 + lane;
        bool valid = idx < n;
        key[k] = valid ? keys_in[idx] : K(0);
        val[k] = valid ? (vals_in ? vals_in[idx] : static_cast<uint32_t>(idx)) : 0u;
        dig[k] = valid ? digit_of(key[k], shift, mask) : static_cast<uint32_t>(BINS);
    }
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        uint32_t peers = __match_any_sync(0xffffffffu, dig[k]);
        int leader = __ffs(peers) - 1;
        uint32_t prev = 0;
        if (lane == leader) {
            prev = s.whist[warp][dig[k]];
            s.whist[warp][dig[k]] = prev + __popc(peers);
        }
        __syncwarp();
        prev = __shfl_sync(0xffffffffu, prev, leader);
        rank[k] = prev + __popc(peers & lt);
    }
    __syncthreads();

    // ---- per-digit: exclusive offsets across warps, tile totals --------------------------------
    for (int d = threadIdx.x; d <= BINS; d += kSortThreads) {
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            uint32_t c = s.whist[w][d];
            s.whist[w][d] = run;
            run += c;
        }
        s.dtotal[d] = run;
    }
    __syncthreads();

    // ---- publish this tile's digit counts first, so later tiles can sum past it while it scatters ----------
    constexpr int kDigitsPerThread = (BINS + kSortThreads - 1) / kSortThreads;
    uint32_t* my = lookback + (size_t)tile * BINS;
    uint32_t tot[kDigitsPerThread];
#pragma unroll
    for (int q = 0; q < kDigitsPerThread; ++q) {
        const int d = (int)threadIdx.x + q * kSortThreads;
        tot[q] = d < BINS ? s.dtotal[d] : 0u;
        if (d < BINS) st_release_u32(&my[d], (tile == 0 ? kLbInclusive : kLbAggregate) | tot[q]);
    }
    __syncthreads();
    block_exclusive_scan_smem(s.dtotal, BINS + 1);  // dtotal[d] := local start of digit d in the tile

    // ---- scatter into shared memory in digit order --------------------------------------------------------
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        uint32_t pos = s.dtotal[dig[k]] + s.whist[warp][dig[k]] + rank[k];
        s.keys[pos] = key[k];
        s.vals[pos] = val[k];
    }

    // ---- decoupled look-back per digit (bounded spin), overlapping the other threads' scatter ---------------
#pragma unroll
    for (int q = 0; q < kDigitsPerThread; ++q) {
        const int d = (int)threadIdx.x + q * kSortThreads;
        if (d >= BINS) break;
        uint32_t prefix = 0;
        if (tile != 0) {
            int64_t j = (int64_t)tile - 1;
            uint32_t spins = 0;
            while (j >= 0) {
                uint32_t w = ld_acquire_u32(lookback + (size_t)j * BINS + d);
                uint32_t state = w & ~kLbCountMask;
                if (state == 0u) {
                    if (++spins > kSpinLimit) {
                        atomicOr(err, kErrTimeout);
                        break;
                    }
                    __nanosleep(32);
                    continue;
                }
                prefix += w & kLbCountMask;
                if (state == kLbInclusive) break;
                --j;
            }
            st_release_u32(&my[d], kLbInclusive | ((prefix + tot[q]) & kLbCountMask));
        }
        s.gofs[d] = static_cast<int32_t>(s.gexcl[d] + prefix) - static_cast<int32_t>(s.dtotal[d]);
    }
    __syncthreads();

    // ---- out to global in digit runs --------------------------------------------------------------------------
    const int valid_count = static_cast<int>(s.dtotal[BINS]);
    for (int i = threadIdx.x; i < valid_count; i += kSortThreads) {
        K k = s.keys[i];
        uint32_t d = digit_of(k, shift, mask);
        int64_t out = (int64_t)s.gofs[d] + i;
        keys_out[out] = k;
        vals_out[out] = s.vals[i];
    }
}

template <typename K, int BITS>
dipl_status sort_impl(const K* kin, const uint32_t* vin, K* kout, uint32_t* vout, K* kalt, uint32_t* valt, int64_t n,
                      int begin_bit, int end_bit, unsigned char* scratch, cudaStream_t stream, uint32_t* d_err) {
    constexpr int BINS = 1 << BITS;
    const int passes = (end_bit - begin_bit + BITS - 1) / BITS;
    const int64_t tiles = (n + kSortTile - 1) / kSortTile;
    uint32_t* hist = reinterpret_cast<uint32_t*>(scratch);
    uint32_t* counters = hist + kMaxPasses * 1024;
    uint32_t* lookback = counters + 64;
    size_t clear = (size_t)(kMaxPasses * 1024 + 64) * 4 + (size_t)passes * tiles * BINS * 4;
    DIPL_CUDA(cudaMemsetAsync(scratch, 0, clear, stream));

    const size_t hsmem = (size_t)passes * BINS * 4;
    int hblocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
    if (hblocks < 1) hblocks = 1;
    if (hsmem > 48 * 1024)
        DIPL_CUDA(cudaFuncSetAttribute(histogram_kernel<K, BITS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)hsmem));
    histogram_kernel<K, BITS><<<hblocks, 256, hsmem, stream>>>(kin, n, begin_bit, end_bit, passes, hist); note_launches();
    DIPL_CUDA(cudaGetLastError());

    const size_t smem = sizeof(SortSmem<K, BITS>);
    DIPL_CUDA(cudaFuncSetAttribute(onesweep_kernel<K, BITS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // Ping-pong so that the last pass lands in (kout, vout); the input is never written.
    const K* src_k = kin;
    const uint32_t* src_v = vin;
    for (int p = 0; p < passes; ++p) {
        bool to_out = ((passes - 1 - p) % 2) == 0;
        K* dk = to_out ? kout : kalt;
        uint32_t* dv = to_out ? vout : valt;
        int shift = begin_bit + p * BITS;
        int width = std::min(BITS, end_bit - shift);
        onesweep_kernel<K, BITS><<<(unsigned)tiles, kSortThreads, smem, stream>>>(
            src_k, src_v, dk, dv, n, shift, width, hist + p * BINS, lookback + (size_t)p * tiles * BINS,
            counters + p, d_err); note_launches();
        DIPL_CUDA(cudaGetLastError());
        src_k = dk;
        src_v = dv;
    }
    return DIPL_OK;
}

template <typename K>
dipl_status sort_dispatch(const K* kin, const uint32_t* vin, K* kout, uint32_t* vout, K* kalt, uint32_t* valt,
                          int64_t n, int begin_bit, int end_bit, int bits, unsigned char* scratch, cudaStream_t s,
                          uint32_t* err) {
    switch (bits) {
        case 6: return sort_impl<K, 6>(kin, vin, kout, vout, kalt, valt, n, begin_bit, end_bit, scratch, s, err);
        case 7: return sort_impl<K, 7>(kin, vin, kout, vout, kalt, valt, n, begin_bit, end_bit, scratch, s, err);
        case 8: return sort_impl<K, 8>(kin, vin, kout, vout, kalt, valt, n, begin_bit, end_bit, scratch, s, err);
        case 10: return sort_impl<K, 10>(kin, vin, kout, vout, kalt, valt, n, begin_bit, end_bit, scratch, s, err);
        default: set_last_error("sort digit width must be 6, 7, 8 or 10"); return DIPL_ERR_INVALID_ARGUMENT;
    }
}

}  // namespace

size_t radix_sort_scratch_bytes(int64_t n, int begin_bit, int end_bit, int digit_bits) {
    int bits = digit_bits > 0 ? digit_bits : 8;
    int passes = (end_bit - begin_bit + bits - 1) / bits;
    int64_t tiles = (n + kSortTile - 1) / kSortTile;
    return (size_t)(kMaxPasses * 1024 + 64) * 4 + (size_t)passes * tiles * (size_t(1) << bits) * 4 + 256;
}

bool radix_sort_bits_ok(int begin_bit, int end_bit, int digit_bits) {
    int bits = digit_bits > 0 ? digit_bits : 8;
    if (bits != 6 && bits != 7 && bits != 8 && bits != 10) return false;
    int passes = (end_bit - begin_bit + bits - 1) / bits;
    return passes >= 1 && passes <= kMaxPasses;
}

dipl_status radix_sort_pairs(const void* kin, const uint32_t* vin, void* kout, uint32_t* vout, void* kalt,
                             uint32_t* valt, int64_t n, int key_bytes, int begin_bit, int end_bit, int digit_bits,
                             void* scratch, cudaStream_t stream, uint32_t* d_err) {
    if (n <= 0) return DIPL_OK;
    int bits = digit_bits > 0 ? digit_bits : 8;
    auto* sc = static_cast<unsigned char*>(scratch);
    if (key_bytes == 4)
        return sort_dispatch<uint32_t>(static_cast<const uint32_t*>(kin), vin, static_cast<uint32_t*>(kout), vout,
                                       static_cast<uint32_t*>(kalt), valt, n, begin_bit, end_bit, bits, sc, stream,
                                       d_err);
    return sort_dispatch<unsigned long long>(static_cast<const unsigned long long*>(kin), vin,
                                             static_cast<unsigned long long*>(kout), vout,
                                             static_cast<unsigned long long*>(kalt), valt, n, begin_bit, end_bit,
                                             bits, sc, stream, d_err);
}

}  // namespace dipl
