// Traversal of the SOBB and 8-wide quantised layouts (filled in by sobb.cu / wide.cu when built).
#include "internal.h"

namespace dipl {

dipl_status trace_closest_ext(const dipl_bvh*, const dipl_ray*, int64_t, dipl_hit*, int, uint32_t,
                              unsigned long long*, cudaStream_t) {
    set_last_error("this layout is not available in this build");
    return DIPL_ERR_UNSUPPORTED;
}

dipl_status trace_any_ext(const dipl_bvh*, const dipl_ray*, int64_t, uint8_t*, int, uint32_t, cudaStream_t) {
    set_last_error("this layout is not available in this build");
    return DIPL_ERR_UNSUPPORTED;
}

}  // namespace dipl
