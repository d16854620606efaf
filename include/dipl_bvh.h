/*
 * dipl_bvh.h — C ABI of the B200 BVH build-and-trace engine (libdipl_bvh.so, sm_100a).
 *
 * The engine stands behind the reference's acceleration-structure boundary:
 *   AccelerationStructure::Build(config, stats, span<const Triangle>)   src/acceleration/acceleration_structure.h:15-16
 *   AccelerationStructure::Intersect(stats, ray, ray_hit, backface)     src/acceleration/acceleration_structure.h:17
 *   AccelerationStructure::IntersectAny(stats, ray, backface)           src/acceleration/acceleration_structure.h:18
 * and replaces the brute-force device loops DummyIntersect / DummyIntersectAny
 * (src/gpu/renderer/gpu_renderer_util.h:29-94) behind the GPU frontend. The reference's GPU side has no
 * C ABI (namespace diplodocus::cuda_kernels, src/gpu/renderer/gpu_renderer_api.h:8-11); this header is
 * the batch-oriented C replacement: a scene in, a BVH handle out; a ray batch in, hit records out.
 *
 * Conventions
 *  - Every pointer argument named d_* or documented as "device" is a CUDA device pointer; the rest are
 *    host pointers. `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *  - Every call returns a dipl_status; nothing aborts. dipl_last_error() gives a message for the
 *    calling thread's most recent failure. There is no CPU fallback: without a usable sm_100 device
 *    every entry point that touches the GPU returns DIPL_ERR_CUDA.
 *  - Calls are asynchronous on `stream` unless documented otherwise. A BVH handle is immutable after
 *    its build completes, so concurrent traces on one handle (any streams) are safe once the build
 *    has been ordered before them.
 */
#ifndef DIPL_BVH_H_
#define DIPL_BVH_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DIPL_ABI_VERSION 2

#if defined(__GNUC__)
#define DIPL_API __attribute__((visibility("default")))
#else
#define DIPL_API
#endif

typedef enum dipl_status {
    DIPL_OK = 0,
    DIPL_ERR_INVALID_ARGUMENT = 1, /* bad pointer, size or enum value */
    DIPL_ERR_CUDA = 2,             /* a CUDA runtime call failed (no device, launch failure, ...) */
    DIPL_ERR_OUT_OF_MEMORY = 3,    /* a device allocation failed */
    DIPL_ERR_TIMEOUT = 4,          /* a bounded device-side wait (look-back, grid barrier) gave up */
    DIPL_ERR_INTERNAL = 5,         /* a device-side consistency check failed (e.g. traversal stack) */
    DIPL_ERR_UNSUPPORTED = 6,      /* a valid option the library does not provide */
    DIPL_ERR_IO = 7                /* a scene file could not be read or parsed */
} dipl_status;

/* Code used to order primitives before clustering.
 * Mirrors MortonType (src/gpu/config/gpu_acceleration_structure_config.h:5). */
typedef enum dipl_code_type { DIPL_CODE_MORTON30 = 0, DIPL_CODE_EMC60 = 1 } dipl_code_type;

/* Bounding volume of the nodes. Mirrors BoundingVolumeType (gpu_acceleration_structure_config.h:7). */
typedef enum dipl_bv_type { DIPL_BV_AABB = 0, DIPL_BV_SOBB = 1 } dipl_bv_type;

/* Clustering of the build. HPLOC (default): PLOC merging confined to the nodes of the binary radix tree of the
 * sorted codes, bottom up in one launch (hierarchical PLOC, Benthin et al. 2024); PLOC: the global PLOC loop
 * (Meister & Bittner 2017), every iteration over all clusters of the scene. Both merge by the same distance and
 * tie rule; HPLOC's trees have about the same SAH cost (within 1% on the 1M sphere and the soup) and build in a
 * fraction of the time. The reference names PLOC as its planned builder (README.md:156-161). */
typedef enum dipl_clustering { DIPL_CLUSTER_HPLOC = 0, DIPL_CLUSTER_PLOC = 1 } dipl_clustering;

/* Node layout used by traces. BINARY: two FP32 child boxes per 64-byte node (80 bytes with SOBB).
 * WIDE8_Q8: 8-wide nodes with 8-bit conservatively quantised child bounds (80 bytes), FP32 leaf re-test. */
typedef enum dipl_layout { DIPL_LAYOUT_BINARY = 0, DIPL_LAYOUT_WIDE8_Q8 = 1 } dipl_layout;

/* Leaf test. REF_MT reproduces Triangle::IntersectRay (src/scene/triangle.cc:10-43) bit for bit
 * (|det| < 1e-6 cull, no FMA, IEEE divide). WATERTIGHT is Woop, Benthin & Wald (2013). */
typedef enum dipl_leaf_test { DIPL_LEAF_REF_MT = 0, DIPL_LEAF_WATERTIGHT = 1 } dipl_leaf_test;

/* Trace flags. BACKFACE_CULLING has the reference's meaning (triangle.cc:18-21): with it, a triangle
 * is hit only when e1 . (dir x e2) > 0. */
#define DIPL_TRACE_BACKFACE_CULLING 1u
/* Trace a batch of 2^20 rays or more in the order of a key of each ray's origin cell and direction octant
 * (computed and sorted on the device inside the call), so that the rays of a warp start close together and head
 * the same way; each record still goes to its ray's index and the records are the same either way. Without it
 * the rays are traced in the order given. On a B200 it pays for incoherent batches (16M random rays in a
 * pre-split 16M-triangle soup: 163 ms against 211 ms) but not for camera-like rays that already come in order
 * (4M rays on a 1M-triangle sphere: the sort costs more than it saves), so it is an option of the call. */
#define DIPL_TRACE_COHERENT_ORDER 2u

/* Build description. The three vertex arrays are the reference GPU scene's SoA positions
 * tri_v0_pos / tri_v1_pos / tri_v2_pos (src/gpu/scene/gpu_scene.h:18-20): float3 per triangle,
 * i.e. 3 floats with a 12-byte stride, DEVICE memory. The engine keeps no pointer to them after the
 * build returns (it copies what traces need), unlike SBvh, which keeps a span (sbvh.h:33). */
typedef struct dipl_build_desc {
    const float* d_v0;
    const float* d_v1;
    const float* d_v2;
    int64_t num_triangles;
    int32_t code_type;              /* dipl_code_type */
    int32_t bv_type;                /* dipl_bv_type */
    int32_t layout;                 /* dipl_layout */
    int32_t max_triangles_per_leaf; /* a node with fewer triangles than this is a leaf (reference
                                       meaning, sbvh.cc:273-276); 2..8, default 4 */
    int32_t nn_search_radius;       /* PLOC radius r, 1..32 (GpuAccelerationStructureConfig::nn_search_radius) */
    int32_t kdop_size;              /* SOBB direction set: kdop_size/2 directions, 6..32 (kdop_size) */
    int32_t ploc_block_size;        /* clustering threads per block: 0 = auto, else 128, 256 or 512 */
    int32_t sort_digit_bits;        /* radix sort digit width: 0 = auto (8), else 6, 7, 8 or 10 */
    int32_t clustering;             /* dipl_clustering (ABI version 2) */
    int32_t split_budget;           /* pre-splitting of large triangles (ABI version 2): at most this percentage
                                       more clustering leaves than triangles, 0..100; 0 = none (the default). A
                                       triangle whose box is large against its mesh's others enters the clustering
                                       as pieces (the boxes of its parts in halves of its box); leaves still hold
                                       the whole triangle, so hits are the same and rays meet fewer empty boxes.
                                       One-shot builds only (not in build plans). */
} dipl_build_desc;

/* A ray: origin, hit interval lower bound, direction, upper bound (32 bytes). A hit needs
 * tmin < t < tmax. The reference's Ray (src/scene/ray.h:7-11) has origin, dir and t_max and always
 * uses tmin = kEpsilon = 1e-6 (sbvh.cc:85); pass tmin = 1e-6f to reproduce it. */
typedef struct dipl_ray {
    float ox, oy, oz, tmin;
    float dx, dy, dz, tmax;
} dipl_ray;

/* A closest-hit record (16 bytes): the reference RayHit's triangle_id, t, b1 and b2
 * (src/scene/ray_hit.h:8-17; b0 = 1 - u - v). A miss is prim = -1, t = +inf, u = v = 0. */
typedef struct dipl_hit {
    int32_t prim;
    float t, u, v;
} dipl_hit;

typedef struct dipl_bvh dipl_bvh; /* opaque, owns its device memory */

typedef struct dipl_bvh_info {
    int64_t num_triangles;
    int64_t num_inner_nodes;     /* nodes of the traced layout */
    int64_t num_leaves;          /* clustering leaves: the triangles, and their pieces with pre-splitting */
    int64_t node_bytes;          /* bytes of the traced node array */
    int64_t triangle_bytes;      /* bytes of the leaf triangle array (one record per clustering leaf) */
    int32_t depth;               /* levels of the clustering tree (bounds the traversal stack) */
    int32_t ploc_iterations;     /* PLOC: global iterations; HPLOC: iterations of all tree nodes, summed */
    int32_t code_type, bv_type, layout, max_triangles_per_leaf, nn_search_radius, kdop_size;
    int32_t clustering, reserved; /* dipl_clustering (ABI version 2) */
} dipl_bvh_info;

/* Fills a description with the defaults (Morton30, AABB, binary, leaves < 4, r = 16, 32-DOP, auto, HPLOC, no
 * pre-splitting). */
DIPL_API void dipl_build_desc_init(dipl_build_desc* desc);

/* Builds a BVH over desc->num_triangles triangles (0 is allowed: every ray misses).
 * Replaces AccelerationStructure::Build (acceleration_structure.h:15-16) / SBvh::Build (sbvh.cc:17-58).
 * The work is queued on `stream`; the call returns once the BVH is complete (it reads back the roots,
 * depth and SAH sums, the build's one host synchronisation), so, like SBvh::Build, the result is ready
 * when it returns. Device memory is released in stream order on `stream` by dipl_bvh_destroy, so that
 * stream must outlive the handle. */
DIPL_API dipl_status dipl_bvh_build(const dipl_build_desc* desc, dipl_bvh** out, void* stream);

/* Builds `count` independent BVHs in one pipeline: one persistent clustering launch for all meshes
 * (their clusters never merge across meshes). out[i] is an ordinary handle for descs[i]; all descs must
 * share the build options. Returns when complete, like dipl_bvh_build. */
DIPL_API dipl_status dipl_bvh_build_batched(const dipl_build_desc* descs, int32_t count, dipl_bvh** out, void* stream);

/* Build plans (batching form). A plan fixes a batch of meshes (their vertex pointers and sizes and one set
 * of options), allocates everything once, runs the build once and captures the whole pipeline (bounds, codes,
 * sort, the persistent clustering launch, layout) into one CUDA graph. dipl_build_plan_launch replays it,
 * rebuilding every BVH from the current contents of the vertex arrays (e.g. after a deformation), with no
 * allocation and no host synchronisation; dipl_build_plan_get_bvhs waits for the stream and returns one
 * handle per mesh for the latest build (valid until the next launch; destroy them with dipl_bvh_destroy).
 * The 8-wide layout is not available in plans (its build reads level sizes back). */
typedef struct dipl_build_plan dipl_build_plan;
DIPL_API dipl_status dipl_build_plan_create(const dipl_build_desc* descs, int32_t count, dipl_build_plan** out,
                                            void* stream);
DIPL_API dipl_status dipl_build_plan_launch(dipl_build_plan* plan, void* stream);
DIPL_API dipl_status dipl_build_plan_get_bvhs(dipl_build_plan* plan, dipl_bvh** out, void* stream);
DIPL_API dipl_status dipl_build_plan_destroy(dipl_build_plan* plan);

/* Autotuner of the build knobs (clustering, PLOC radius, PLOC block size, sort digit width) for a batch: times
 * real builds of these meshes and keeps the fastest setting whose SAH cost is within 2% of the radius-16 default
 * with the requested clustering; the winner is cached per (code, bounding volume, layout, leaf size, requested
 * clustering, size bucket floor(log2 total triangles)) in
 * `cache_path` (one JSON object per line; NULL = no cache). tuned[i] = descs[i] with the chosen knobs;
 * *from_cache (may be NULL) tells whether the cache answered. Synchronises `stream` (it builds). */
DIPL_API dipl_status dipl_autotune_build(const dipl_build_desc* descs, int32_t count, const char* cache_path,
                                         dipl_build_desc* tuned, int32_t* from_cache, void* stream);

/* Closest hit for n rays (device arrays of dipl_ray / dipl_hit). Replaces
 * AccelerationStructure::Intersect (acceleration_structure.h:17; SBvh::Intersect sbvh.cc:60-145) and the
 * device brute force DummyIntersect (gpu_renderer_util.h:29-72). Exact-t ties resolve to the lowest
 * primitive id, like DummyAccelerationStucture::Intersect (dummy_acceleration_structure.cc:21-64). */
DIPL_API dipl_status dipl_bvh_trace_closest(const dipl_bvh* bvh, const dipl_ray* d_rays, int64_t n, dipl_hit* d_hits,
                                   int32_t leaf_test, uint32_t flags, void* stream);

/* As dipl_bvh_trace_closest, also adding the node visits and triangle tests of the batch to
 * d_counters[0] and d_counters[1] (device, 2 x uint64). The counts mirror AccelerationStats'
 * traversal_count / intersection_count (src/stats/acceleration_stats.h:14-16) in 64 bits. */
DIPL_API dipl_status dipl_bvh_trace_closest_counted(const dipl_bvh* bvh, const dipl_ray* d_rays, int64_t n, dipl_hit* d_hits,
                                           int32_t leaf_test, uint32_t flags, uint64_t* d_counters, void* stream);

/* Any hit (occlusion) for n rays: d_occluded[i] = 1 if some triangle has tmin < t < tmax.
 * Replaces AccelerationStructure::IntersectAny (acceleration_structure.h:18; SBvh::IntersectAny
 * sbvh.cc:147-191) and DummyIntersectAny (gpu_renderer_util.h:74-94). */
DIPL_API dipl_status dipl_bvh_trace_any(const dipl_bvh* bvh, const dipl_ray* d_rays, int64_t n, uint8_t* d_occluded,
                               int32_t leaf_test, uint32_t flags, void* stream);

/* SAH cost C = [sum over inner nodes SA(n) + sum over leaves SA(n) |n|] / SA(root), C_t = C_i = 1,
 * summed in FP64 on the device over the traced layout. Synchronises `stream`. */
DIPL_API dipl_status dipl_bvh_sah_cost(const dipl_bvh* bvh, double* cost, void* stream);

DIPL_API dipl_status dipl_bvh_get_info(const dipl_bvh* bvh, dipl_bvh_info* info);

/* Copies the clustering result to HOST buffers (any may be NULL); n = num_leaves of dipl_bvh_get_info (the
 * triangle count without pre-splitting): h_perm[n] = triangle id at each sorted-code position (leaf node id =
 * position; a split triangle appears once per piece); h_children[2*(n-1)] = left/right node
 * ids of internal node k (id num_triangles + k; PLOC numbers nodes in creation order, HPLOC gives node k the
 * id of radix-tree split k or of a split below it); h_boxes[6*(n-1)] = its box
 * (lo xyz, hi xyz). Synchronises `stream`. For checking and debugging. */
DIPL_API dipl_status dipl_bvh_download_topology(const dipl_bvh* bvh, int32_t* h_perm, int32_t* h_children, float* h_boxes,
                                       void* stream);

/* Copies the traced node array and leaf triangle array to HOST memory (sizes from dipl_bvh_info),
 * and the root reference (>= 0: node index; < 0: ~(first_triangle << 3 | count) leaf). Synchronises. */
DIPL_API dipl_status dipl_bvh_download_layout(const dipl_bvh* bvh, void* h_nodes, void* h_triangles, int32_t* h_root,
                                     void* stream);

/* Synchronises `stream` and reports device-side failures recorded by earlier traces on this handle
 * (a traversal stack or step limit hit: DIPL_ERR_INTERNAL), then clears them. Traces never fault on
 * such a failure; they finish the ray with what they have and record it here. */
DIPL_API dipl_status dipl_bvh_check_errors(const dipl_bvh* bvh, void* stream);

/* Releases the handle's device memory in stream order on its build stream. NULL is a no-op. */
DIPL_API dipl_status dipl_bvh_destroy(dipl_bvh* bvh);

/* ---- building blocks exported for tests and callers that need them on their own ---------------- */

/* Codes of the build (Morton30 in the low 30 bits of uint32, or EMC60 in the low 60 bits of uint64)
 * for the triangles of desc (uses d_v0/d_v1/d_v2, num_triangles, code_type). d_codes is device memory
 * of num_triangles uint32 (MORTON30) or uint64 (EMC60). */
DIPL_API dipl_status dipl_compute_codes(const dipl_build_desc* desc, void* d_codes, void* stream);

/* Stable LSD radix sort of (key, value) pairs on bits [begin_bit, end_bit) of the keys. Keys are uint32
 * (key_bytes = 4) or uint64 (key_bytes = 8); values uint32. d_vals_in may be NULL (values 0..n-1).
 * Input and output arrays must not overlap. */
DIPL_API dipl_status dipl_radix_sort_pairs(const void* d_keys_in, const uint32_t* d_vals_in, void* d_keys_out,
                                  uint32_t* d_vals_out, int64_t n, int32_t key_bytes, int32_t begin_bit,
                                  int32_t end_bit, int32_t digit_bits, void* stream);

/* No counterpart in the reference. The same sort as dipl_radix_sort_pairs for callers that may not
 * allocate device memory (a host application that owns the whole GPU heap and gives plug-ins fixed
 * buffers, or a loop that must not stall on cudaMalloc). Its scratch is one fixed array in the library's
 * device image (about 5 MB on every GPU that loads the library, held until the process exits); no memory is
 * allocated per call. At most 262,144 pairs (larger n: DIPL_ERR_INVALID_ARGUMENT). The first call in each
 * CUDA context looks up the array's address in that context (a context made current later, or the one after a
 * device reset, gets its own lookup), so make it before any stream capture. All calls on a device share
 * the array: the call clears what must start at zero, but calls whose GPU work overlaps race on it, so
 * order them. Synchronises `stream` at the end, like dipl_radix_sort_pairs. */
DIPL_API dipl_status dipl_radix_sort_pairs_noalloc(const void* d_keys_in, const uint32_t* d_vals_in, void* d_keys_out,
                                                   uint32_t* d_vals_out, int64_t n, int32_t key_bytes,
                                                   int32_t begin_bit, int32_t end_bit, int32_t digit_bits,
                                                   void* stream);

/* FP64 oracle re-intersection (checking only): for each hit, t/u/v of the ray against triangle `prim`
 * of the original vertex arrays, in double precision (d_tuv: 3 doubles per ray; misses give +inf,0,0). */
DIPL_API dipl_status dipl_reintersect_f64(const float* d_v0, const float* d_v1, const float* d_v2, const dipl_ray* d_rays,
                                 const dipl_hit* d_hits, int64_t n, double* d_tuv, void* stream);

/* Adjoint of the closest-hit t/u/v (differentiation form). Given the forward hits and upstream
 * gradients d_dtuv (3 floats per ray: dL/dt, dL/du, dL/dv), ADDS dL/dvertex into d_dv0/d_dv1/d_dv2
 * (float3 per triangle, like the vertex arrays; atomically) and WRITES dL/dorigin and dL/ddirection
 * (float3 per ray) into d_dorig / d_ddir (either may be NULL). Hit ids are held fixed (visibility is
 * discrete); misses contribute nothing. */
DIPL_API dipl_status dipl_trace_adjoint(const float* d_v0, const float* d_v1, const float* d_v2, const dipl_ray* d_rays,
                               const dipl_hit* d_hits, const float* d_dtuv, int64_t n, float* d_dv0, float* d_dv1,
                               float* d_dv2, float* d_dorig, float* d_ddir, void* stream);

/* ---- GPU frontend: wavefront ray generation (generate -> trace -> bounce -> trace) ------------------------ */

/* Pinhole camera of the reference scene (Camera: pos, dir, up, fov in radians; far = the primary rays' t_max). */
typedef struct dipl_camera {
    float pos[3];
    float dir[3];
    float up[3];
    float fov;
    float far_t;
} dipl_camera;

/* One primary ray per pixel, row-major from the top-left pixel, into d_rays (width * height records).
 * Replaces the per-pixel ray set-up of the reference renderers: the camera basis of
 * CpuRaytracer::StartRender / GpuRenderer::StartRender (src/renderer/cpu_raytracer.cc:64-70,
 * src/renderer/gpu_renderer.cc:25-35) and the direction of RaytracingBounceKernel
 * (src/gpu/renderer/gpu_renderer_api.cu:43-53): dir = normalize(p00 + qw*x + qh*y), with the CPU build's
 * Normalize (src/util/vec3.h:111-117) in FP32 without FMA; origin = pos, tmin = 1e-6, tmax = far_t. */
DIPL_API dipl_status dipl_generate_pinhole_rays(const dipl_camera* camera, int32_t width, int32_t height,
                                                dipl_ray* d_rays, void* stream);

/* One cosine-weighted bounce ray per hit (the renderer's next path segment, TracePath in
 * src/gpu/renderer/gpu_pathtracer.cu:12). For hit i: the hit point o + d*t, the triangle's geometric normal
 * (from the vertex arrays, facing the incoming ray), a direction drawn from the cosine-weighted hemisphere
 * about it with the reference's counter-based hash (HashU32 / U01FromU32, src/util/util.h:24-37; seed, ray
 * index), and the origin offset along the normal by RayEpsilon (src/scene/ray.h:15-24) like OffsetRayOrigin
 * (src/renderer/cpu_raytracer.cc:41-46); tmax = FLT_MAX. Misses give a ray that hits nothing (tmax = 0).
 * All arithmetic is IEEE add/mul/div/sqrt in FP32 in a fixed order, so the records are reproducible bit for
 * bit on the host. d_out may not alias d_rays. */
DIPL_API dipl_status dipl_generate_bounce_rays(const float* d_v0, const float* d_v1, const float* d_v2,
                                               const dipl_ray* d_rays, const dipl_hit* d_hits, int64_t n,
                                               uint32_t seed, dipl_ray* d_out, void* stream);

/* Shadow rays of the renderer's local illumination, one per (hit, light sample), for dipl_bvh_trace_any.
 * Replaces the shadow-ray set-up of IsShadowed (src/renderer/cpu_raytracer.cc:222-237,
 * src/gpu/renderer/gpu_renderer_util.h:96-108) around the hit record the reference makes (Ray::At(t), RayEpsilon,
 * the triangle's geometric normal): dir = (light - pos) / |light - pos|, origin offset by RayEpsilon along the
 * normal on dir's side (OffsetRayOrigin), tmax = |light - pos| (1 - RayEpsilon). Lights, in the reference's order:
 * num_area_lights area lights (triangle ids of the vertex arrays) with `samples` samples each, drawn as
 * LocalIlluminationAreaLights does (cpu_raytracer.cc:165-186: RandomAreaLightSample01(seed, x, y, light, sample, dim)
 * over ray i's pixel x = i % width, y = i / width, then Triangle::SampleSurface; the reference's seed is 42), then
 * num_point_lights point lights (d_point_lights: xyz per light). Output: d_out[i * per_hit + j] with
 * per_hit = num_area_lights * samples + num_point_lights. A ray that casts no shadow ray for a light gets a null ray
 * (tmax = 0, never occluded): a miss; a hit on an area light's own triangle (the reference returns the light's
 * colour and casts no more area-light rays for that hit); a light within kEpsilon of the hit point.
 * FP32 IEEE arithmetic in the reference's order, so the records are reproducible bit for bit on the host. */
DIPL_API dipl_status dipl_generate_shadow_rays(const float* d_v0, const float* d_v1, const float* d_v2,
                                               const dipl_ray* d_rays, const dipl_hit* d_hits, int64_t n, int32_t width,
                                               const int32_t* d_area_light_triangles, int32_t num_area_lights,
                                               int32_t samples, const float* d_point_lights, int32_t num_point_lights,
                                               uint32_t seed, dipl_ray* d_out, void* stream);

/* No counterpart in the reference. Failure-detection self-test: runs the library's bounded device waits (the
 * warp and block decoupled look-backs of the sort and the clustering, and the grid barrier between clustering
 * iterations) on a status word that no tile publishes and on a barrier with one participant that never
 * arrives, each giving up after spin_limit polls (1..2^20), then launches one more kernel on the same context.
 * *out_flags gets bit 0/1/2 when the warp look-back / block look-back / grid barrier gave up and bit 3 when
 * the follow-up kernel ran. Returns DIPL_ERR_TIMEOUT when all four bits are set (the expected outcome),
 * DIPL_ERR_INTERNAL otherwise. Synchronises `stream`. */
DIPL_API dipl_status dipl_selftest_bounded_waits(uint32_t spin_limit, uint32_t* out_flags, void* stream);

/* ---- OBJ scenes: the reference's scene files into the engine (host side) --------------------------------- */

/* A loaded scene: triangles in file order with the reference Scene's float bits, materials, lights, camera. */
typedef struct dipl_obj_scene dipl_obj_scene;

typedef struct dipl_obj_scene_info {
    int64_t num_triangles;
    int64_t num_materials;
    int64_t num_area_lights;
    int64_t num_point_lights;
    float camera[11]; /* pos[3], dir[3], up[3], fov, far (the .meta camera) */
} dipl_obj_scene_info;

/* Replaces ObjSceneLoader::Load (src/io/scene/obj_scene_loader.cc:189-205): reads <dirpath>/<name>.meta
 * (camera, point lights; LoadMetadata, :120-187) then <name>.obj and the MTL files it names (LoadObj, :20-118,
 * with its vendored tinyobjloader's quad split, ear clipping and index rules). DIPL_ERR_IO (message in
 * dipl_last_error) where the reference returns std::nullopt; also when a vertex or normal index is out of
 * range. Host only: no device is needed. Free with dipl_obj_scene_destroy. */
DIPL_API dipl_status dipl_obj_scene_load(const char* dirpath, const char* name, dipl_obj_scene** out);
DIPL_API dipl_status dipl_obj_scene_get_info(const dipl_obj_scene* scene, dipl_obj_scene_info* info);
/* Host copies (any pointer may be NULL): positions and normals 9 floats per triangle (v0, v1, v2; normals 0
 * where the triangle has none), geometric normals 3 floats (Normalize(Cross(v1 - v0, v2 - v0)), scene.cc:18-21),
 * material ids (-1 = none), has_vertex_normals 1 byte per triangle. */
DIPL_API dipl_status dipl_obj_scene_get_triangles(const dipl_obj_scene* scene, float* positions, float* normals,
                                                  float* geom_normals, int32_t* material_ids,
                                                  uint8_t* has_vertex_normals);
/* The three vertex arrays (float3 each, host memory) in the SoA layout dipl_build_desc takes after upload. */
DIPL_API dipl_status dipl_obj_scene_get_soa(const dipl_obj_scene* scene, float* v0, float* v1, float* v2);
/* values: 19 floats per material (ambient, diffuse, specular, transmittance, emission, shininess, ior, r_ior,
 * dissolve: src/scene/material.h); names: 64 bytes per material, NUL-terminated. Either may be NULL. */
DIPL_API dipl_status dipl_obj_scene_get_materials(const dipl_obj_scene* scene, float* values, char* names);
/* Area lights (one per emissive triangle: triangle id, emission colour (3 floats), surface area) and point
 * lights (7 floats each: pos, color, power). Any pointer may be NULL. */
DIPL_API dipl_status dipl_obj_scene_get_lights(const dipl_obj_scene* scene, int32_t* area_triangle_ids,
                                               float* area_colors, float* area_surface_areas, float* point_lights);
DIPL_API void dipl_obj_scene_destroy(dipl_obj_scene* scene);

/* ---- limits -------------------------------------------------------------------------------------------------- */

/* No counterpart in the reference, which has no limits and aborts on any CUDA error (CUDA_CHECK -> abort,
 * src/gpu/cuda_utils.h:12-18). Process-wide limits of this library (every device and thread), for callers that
 * share the GPU with other work and for exercising the failure paths without a GPU fault:
 *   device_memory_bytes    device memory the library may hold at once (all live allocations of builds, handles and
 *                          traces); an allocation beyond it fails like a failed cudaMallocAsync, with
 *                          DIPL_ERR_OUT_OF_MEMORY, and the call releases what it had taken. 0 = no limit.
 *   clustering_iterations  iterations the clustering may take before the build gives up with DIPL_ERR_INTERNAL:
 *                          global iterations (PLOC) or iterations within one radix-tree node (HPLOC). 0 = the
 *                          built-in bounds (65536, 64). Read when a build is enqueued: a build plan keeps the value
 *                          of its capture.
 *   trace_steps            traversal steps (inner nodes and leaves) one ray may take; a ray that needs more is
 *                          finished with what it has and DIPL_ERR_INTERNAL is recorded for dipl_bvh_check_errors.
 *                          0 = the built-in bound (twice the node count, plus 64).
 * dipl_get_limits also reports the device memory the library holds now (may be NULL). */
typedef struct dipl_limits {
    uint64_t device_memory_bytes;
    uint32_t clustering_iterations;
    uint32_t trace_steps;
} dipl_limits;
DIPL_API dipl_status dipl_set_limits(const dipl_limits* limits);
DIPL_API dipl_status dipl_get_limits(dipl_limits* limits, uint64_t* device_memory_in_use);

DIPL_API const char* dipl_status_string(dipl_status status);
/* Message of the calling thread's most recent failure ("" if none). */
DIPL_API const char* dipl_last_error(void);
DIPL_API int32_t dipl_abi_version(void);
/* Number of CUDA kernels this library has launched in the process so far (all entry points). */
DIPL_API uint64_t dipl_kernel_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* DIPL_BVH_H_ */
