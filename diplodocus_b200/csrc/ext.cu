// Dispatch of the traversals that are not the binary FP32-AABB one.
#include "internal.h"

namespace dipl {

dipl_status trace_closest_ext(const dipl_bvh* b, const dipl_ray* rays, int64_t n, dipl_hit* hits, int leaf_test,
                              uint32_t flags, unsigned long long* counters, cudaStream_t s) {
    if (b->layout == DIPL_LAYOUT_WIDE8_Q8) return trace_wide(b, rays, n, hits, nullptr, leaf_test, flags, counters, false, s);
    if (b->bv_type == DIPL_BV_SOBB) return trace_sobb(b, rays, n, hits, nullptr, leaf_test, flags, counters, false, s);
    set_last_error("trace: no traversal for this combination of layout and bounding volume");
    return DIPL_ERR_UNSUPPORTED;
}

dipl_status trace_any_ext(const dipl_bvh* b, const dipl_ray* rays, int64_t n, uint8_t* occluded, int leaf_test,
                          uint32_t flags, cudaStream_t s) {
    if (b->layout == DIPL_LAYOUT_WIDE8_Q8) return trace_wide(b, rays, n, nullptr, occluded, leaf_test, flags, nullptr, true, s);
    if (b->bv_type == DIPL_BV_SOBB) return trace_sobb(b, rays, n, nullptr, occluded, leaf_test, flags, nullptr, true, s);
    set_last_error("trace: no traversal for this combination of layout and bounding volume");
    return DIPL_ERR_UNSUPPORTED;
}

}  // namespace dipl
