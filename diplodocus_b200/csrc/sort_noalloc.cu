// A radix-sort entry point that allocates no device memory.
//
// Some callers cannot allocate: a host application that reserves the whole GPU heap up front and hands
// plug-ins fixed buffers (renderers and game engines commonly do), or a latency-bound loop in which a
// cudaMalloc could synchronise the device and stall it. For them this entry point takes its scratch from
// one array in device global memory that is part of the library image: every GPU that loads the library
// holds it (kNoAllocScratchBytes, about 5 MB) until the process exits, and no allocation happens per call.
//
// Limits and rules of use:
//  - at most kNoAllocMaxKeys (2^18 = 262,144) pairs per call; larger sorts are rejected;
//  - the first call in a CUDA context looks up the array's device address (cudaGetSymbolAddress) with that
//    context current and caches it under the context's id, so make that first call before any stream capture.
//    Each context loads the library's device image anew, so after a device reset, or when another context is
//    made current, the array may sit at another address: a call from a context the cache has not seen looks it
//    up again (context ids are never reused within a process, so a stale address is never handed out);
//  - every call on a device uses the same array, which keeps whatever the last call left in it; the parts
//    that must start at zero (digit histograms, look-back words, the error word) are cleared by each call,
//    but two calls whose work overlaps on the GPU (different streams, no ordering between them) race on it
//    and give wrong results: order them;
//  - like dipl_radix_sort_pairs, the call synchronises `stream` once at the end to report device errors.
#include <mutex>

#include <cuda.h>  // CUcontext and CUresult types only: the two driver calls are resolved at run time

#include "internal.h"

namespace dipl {
namespace {

constexpr int64_t kNoAllocMaxKeys = int64_t(1) << 18;
constexpr size_t kErrBytes = 256;
constexpr size_t kAltKeyBytes = size_t(kNoAllocMaxKeys) * 8;  // room for 64-bit keys
constexpr size_t kAltValBytes = size_t(kNoAllocMaxKeys) * 4;
// Histograms + look-back words of the widest choice: 10-bit digits over 64-bit keys (7 passes), counted
// for 3840-key tiles, which bounds the tile count of the sort's larger tiles (radix_sort_scratch_bytes is
// checked against this size on every call).
constexpr size_t kSortTilesMax = (size_t(kNoAllocMaxKeys) + 3839) / 3840;
constexpr size_t kSortScratchBytes = (11 * 1024 + 64) * 4 + 7 * kSortTilesMax * 1024 * 4 + 256;
constexpr size_t kNoAllocScratchBytes = kErrBytes + kAltKeyBytes + kAltValBytes + kSortScratchBytes;

// The scratch array. In host code this name is only a stand-in for the device object: its device address
// comes from cudaGetSymbolAddress below, never from taking the address of the name.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Identity of the calling thread's current context, through the driver's cuCtxGetCurrent / cuCtxGetId (resolved
// at run time through the runtime, so the library needs no link-time dependency on the driver library). 0 when no
// context is current yet.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

dipl_status current_context_id(unsigned long long* id) {
    static std::once_flag once;
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(f);
        (void)cudaGetLastError();
    });
    if (!get_current || !get_id) {
        set_last_error("dipl_radix_sort_pairs_noalloc: cuCtxGetCurrent / cuCtxGetId unavailable from the driver");
        return DIPL_ERR_CUDA;
    }
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS) {
        set_last_error("dipl_radix_sort_pairs_noalloc: cuCtxGetCurrent failed");
        return DIPL_ERR_CUDA;
    }
    *id = 0;
    if (ctx && get_id(ctx, id) != CUDA_SUCCESS) {
        set_last_error("dipl_radix_sort_pairs_noalloc: cuCtxGetId failed");
        return DIPL_ERR_CUDA;
    }
    return DIPL_OK;
}

constexpr int kMaxDevices = 64;
struct ScratchAddress {
    unsigned long long context_id = 0;  // 0: nothing cached
    void* ptr = nullptr;
};
std::mutex g_scratch_mu;
ScratchAddress g_scratch[kMaxDevices];

// Device address of the scratch array in the current context (looked up once per context).
dipl_status scratch_for_current_context(unsigned char** out) {
    int dev = 0;
    DIPL_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_last_error("dipl_radix_sort_pairs_noalloc: device ordinal out of range");
        return DIPL_ERR_UNSUPPORTED;
    }
    unsigned long long id = 0;
    dipl_status st = current_context_id(&id);
    if (st != DIPL_OK) return st;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (id == 0 || g_scratch[dev].context_id != id || !g_scratch[dev].ptr) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);  // binds the device's context if none was
        if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        if ((st = current_context_id(&id)) != DIPL_OK) return st;
        g_scratch[dev].context_id = id;
        g_scratch[dev].ptr = p;
    }
    *out = static_cast<unsigned char*>(g_scratch[dev].ptr);
    return DIPL_OK;
}

}  // namespace
}  // namespace dipl

using namespace dipl;

extern "C" dipl_status dipl_radix_sort_pairs_noalloc(const void* d_keys_in, const uint32_t* d_vals_in,
                                                     void* d_keys_out, uint32_t* d_vals_out, int64_t n,
                                                     int32_t key_bytes, int32_t begin_bit, int32_t end_bit,
                                                     int32_t digit_bits, void* stream) {
    if (n < 0 || (key_bytes != 4 && key_bytes != 8) || begin_bit < 0 || end_bit <= begin_bit ||
        end_bit > 8 * key_bytes || !radix_sort_bits_ok(begin_bit, end_bit, digit_bits)) {
        set_last_error("dipl_radix_sort_pairs_noalloc: bad size, key width, bit range or digit width");
        return DIPL_ERR_INVALID_ARGUMENT;
    }
    if (n > kNoAllocMaxKeys) {
        set_last_error("dipl_radix_sort_pairs_noalloc: n = " + std::to_string(n) + " exceeds the limit of " +
                       std::to_string(kNoAllocMaxKeys) + " pairs of the fixed scratch; use dipl_radix_sort_pairs");
        return DIPL_ERR_INVALID_ARGUMENT;
    }
    if (n == 0) return DIPL_OK;
    if (!d_keys_in || !d_keys_out || !d_vals_out) {
        set_last_error("dipl_radix_sort_pairs_noalloc: key/value arrays must be non-NULL");
        return DIPL_ERR_INVALID_ARGUMENT;
    }
    if (radix_sort_scratch_bytes(n, begin_bit, end_bit, digit_bits) > kSortScratchBytes) {
        set_last_error("dipl_radix_sort_pairs_noalloc: scratch layout too small (internal)");
        return DIPL_ERR_INTERNAL;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned char* base = nullptr;
    dipl_status st = scratch_for_current_context(&base);
    if (st != DIPL_OK) return st;
    uint32_t* err = reinterpret_cast<uint32_t*>(base);
    void* kalt = base + kErrBytes;
    uint32_t* valt = reinterpret_cast<uint32_t*>(base + kErrBytes + kAltKeyBytes);
    unsigned char* sort_scratch = base + kErrBytes + kAltKeyBytes + kAltValBytes;
    DIPL_CUDA(cudaMemsetAsync(err, 0, 4, s));  // the array keeps the previous call's contents
    st = radix_sort_pairs(d_keys_in, d_vals_in, d_keys_out, d_vals_out, kalt, valt, n, key_bytes, begin_bit, end_bit,
                          digit_bits, sort_scratch, s, err);
    if (st != DIPL_OK) return st;
    return check_device_error(err, s, "dipl_radix_sort_pairs_noalloc");
}
