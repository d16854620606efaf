// Self-test of the bounded device-side waits (failure detection without a GPU fault).
//
// Every wait of the engine on another block's progress — the warp and block decoupled look-backs of the sort
// and the clustering, and the grid barrier between clustering iterations — gives up after a bounded number of
// polls, records kErrTimeout in an error word and lets the kernel return, so the host gets DIPL_ERR_TIMEOUT and
// the CUDA context stays usable. This entry point runs those same wait primitives on a status word that no
// tile ever publishes and on a barrier with one participant that never arrives, with a small poll limit, then
// launches one more kernel to show that the context still works.
#include "internal.h"

namespace dipl {
namespace {

constexpr int kSelftestThreads = 128;

struct SelftestScratch {
    unsigned long long status[64];  // look-back words of tiles 0..63: all "not ready" (0)
    GridBarrier bar;
    uint32_t err[3];                // warp look-back, block look-back, grid barrier
    uint32_t sentinel;
};

__global__ void __launch_bounds__(kSelftestThreads) selftest_waits_kernel(SelftestScratch* S, uint32_t spin_limit) {
    __shared__ unsigned long long wsum[kSelftestThreads / 32];
    __shared__ int wflag[kSelftestThreads / 32];
    bool ok = true;
    if (blockIdx.x == 0) {
        if (threadIdx.x < 32) warp_lookback(S->status, 1, &S->err[0], &ok, spin_limit);  // tile 0 never publishes
    } else {
        block_lookback<kSelftestThreads>(S->status, 1, &S->err[1], &ok, wsum, wflag, spin_limit);
    }
    grid_barrier(&S->bar, gridDim.x + 1u, &S->err[2], spin_limit);  // one participant never arrives
}

__global__ void selftest_after_kernel(SelftestScratch* S) {
    if (threadIdx.x == 0 && blockIdx.x == 0) S->sentinel = 0x5E1F7E57u;
}

}  // namespace
}  // namespace dipl

using namespace dipl;

extern "C" dipl_status dipl_selftest_bounded_waits(uint32_t spin_limit, uint32_t* out_flags, void* stream) {
    DIPL_CHECK_ARG(out_flags, "out_flags must be non-NULL");
    DIPL_CHECK_ARG(spin_limit >= 1 && spin_limit <= (1u << 20), "spin_limit must be in [1, 2^20]");
    *out_flags = 0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    void* raw = nullptr;
    dipl_status st = device_alloc(&raw, sizeof(SelftestScratch), s);
    if (st != DIPL_OK) return st;
    SelftestScratch* S = static_cast<SelftestScratch*>(raw);
    SelftestScratch h{};
    cudaError_t e = cudaMemsetAsync(S, 0, sizeof(SelftestScratch), s);
    if (e == cudaSuccess) {
        selftest_waits_kernel<<<2, kSelftestThreads, 0, s>>>(S, spin_limit);
        note_launches();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        selftest_after_kernel<<<1, 32, 0, s>>>(S);
        note_launches();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, S, sizeof(SelftestScratch), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    device_free(S, s);
    if (e != cudaSuccess) return cuda_status(e, "dipl_selftest_bounded_waits");
    uint32_t flags = 0;
    if (h.err[0] & kErrTimeout) flags |= 1u;
    if (h.err[1] & kErrTimeout) flags |= 2u;
    if (h.err[2] & kErrTimeout) flags |= 4u;
    if (h.sentinel == 0x5E1F7E57u) flags |= 8u;
    *out_flags = flags;
    if (flags == 15u) {
        set_last_error("dipl_selftest_bounded_waits: every wait gave up as expected; the context is usable");
        return DIPL_ERR_TIMEOUT;
    }
    set_last_error("dipl_selftest_bounded_waits: a wait did not give up, or the context failed (flags " +
                   std::to_string(flags) + ")");
    return DIPL_ERR_INTERNAL;
}
