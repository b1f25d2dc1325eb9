/*
 * yrcuda.h — C ABI of libyrcuda, the B200 (sm_100a) backend for YaoRay.
 *
 * Every entry point takes plain pointers and sizes and returns a yrc_status;
 * no C++ exception and no CUDA or torch type crosses this boundary. On error
 * the message of the failing call is available from yrc_last_error() on the
 * calling thread. The library owns all device memory it allocates; the caller
 * owns every host buffer it passes in.
 *
 * Reference interfaces replaced or mirrored (paths inside QiuRuhai/YaoRay):
 *   RenderBvhNode / RenderBvhPrimitive / RenderBvh   include/yaoray/accel/bvh.hpp:34-81
 *   BuildBvh                                         include/yaoray/accel/bvh.hpp:102, src/accel/bvh_builder.cpp:269-286
 *   BuildRenderAcceleration / BuildTwoLevelBvh       include/yaoray/accel/acceleration.hpp:138, two_level_bvh.hpp:55
 *   IntersectBvh / IntersectAcceleration             include/yaoray/accel/bvh.hpp:107-114, acceleration.hpp:143-150
 *   IntersectTwoLevelBvh                             include/yaoray/accel/two_level_bvh.hpp:77-84
 *   IntersectAccelerationProbe                       include/yaoray/accel/acceleration.hpp:152-161
 *   RenderBackend::Prepare / Render (CUDA stub)      include/yaoray/runtime/backend.hpp:90-98,
 *                                                    src/runtime/cuda_stub_backend.cpp:20-37
 */
#ifndef YRCUDA_H
#define YRCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */

typedef enum yrc_status {
    YRC_OK = 0,
    YRC_ERR_INVALID_ARGUMENT = 1, /* bad pointer, size or scene data            */
    YRC_ERR_CUDA = 2,             /* a CUDA runtime call failed                  */
    YRC_ERR_OUT_OF_MEMORY = 3,    /* device allocation or the admission budget   */
    YRC_ERR_CANCELLED = 4,        /* a render was cancelled between passes       */
    YRC_ERR_UNSUPPORTED = 5,      /* scene feature outside what the kernels run  */
    YRC_ERR_DEVICE_FAULT = 6,     /* a kernel reported an error status word      */
    YRC_ERR_BUILD = 7             /* BVH build error (reference error strings)   */
} yrc_status;

/* Message of the last failing call on this thread ("" if none). */
const char* yrc_last_error(void);
/* Library version string, e.g. "0.1.0". */
const char* yrc_version(void);
/* 1 when a CUDA device is usable by the library, else 0 (never faults). */
int yrc_device_available(void);

/* ---------------------------------------------------------------- geometry */

/* RenderPrimitive (include/yaoray/scene/geometry.hpp:20-27). */
typedef struct yrc_primitive {
    uint32_t first_index;
    uint32_t index_count;
    int32_t material_index;
    uint32_t flags; /* bit0 has_normals, bit1 has_uvs, bit2 has_tangents */
} yrc_primitive;

/* RenderSphere (geometry.hpp:29-35). */
typedef struct yrc_sphere {
    float center[3];
    float radius;
    int32_t material_index;
    int32_t area_light_index;
    int32_t flip_normals;
    int32_t reserved;
} yrc_sphere;

/* RenderInstance (geometry.hpp:39-42): column-major Mat4f. */
typedef struct yrc_instance {
    int32_t primitive;
    float object_to_world[16];
} yrc_instance;

/*
 * GeometryView (geometry.hpp:44-71). `positions` points at the first vertex
 * position; consecutive vertices are `vertex_stride` bytes apart (12 for a
 * packed xyz array, 48 for an array of RenderVertex).
 */
typedef struct yrc_geometry {
    const float* positions;
    int64_t vertex_count;
    int64_t vertex_stride;
    const uint32_t* indices;
    int64_t index_count;
    const yrc_primitive* primitives;
    int32_t primitive_count;
    const yrc_sphere* spheres;
    int32_t sphere_count;
    const yrc_instance* instances;
    int32_t instance_count;
} yrc_geometry;

/* --------------------------------------------------------------------- BVH */

/* RenderBvhNode (bvh.hpp:34-47), byte-identical, 32 bytes. */
typedef struct yrc_bvh_node {
    float bounds_min[3];
    float bounds_max[3];
    int32_t payload_offset;  /* leaf: first primitive slot; interior: right child */
    int32_t primitive_count; /* > 0: leaf */
} yrc_bvh_node;

/* RenderBvhPrimitive (bvh.hpp:49-55). kind: 0 triangle, 1 sphere. */
typedef struct yrc_bvh_primitive {
    int32_t kind;
    int32_t mesh_primitive;
    int32_t sphere;
    int32_t local_triangle;
    int32_t flat_triangle_index;
} yrc_bvh_primitive;

/* BvhBuildOptions (bvh.hpp:17-32). split_method: 0 SAH buckets, 1 median. */
typedef struct yrc_bvh_options {
    int32_t split_method;
    int32_t max_leaf_triangles;        /* default 4 */
    int32_t thread_count;              /* 0 = all hardware threads */
    int32_t parallel_min_subtree_size; /* default 1024 */
} yrc_bvh_options;

/* Read-only view of a RenderBvh's arrays (the reference's, or yrc_bvh_*'s). */
typedef struct yrc_bvh_view {
    const yrc_bvh_node* nodes;
    int64_t node_count;
    const int32_t* primitive_indices;
    int64_t primitive_index_count;
    const yrc_bvh_primitive* primitives;
    int64_t primitive_count;
    int32_t max_depth;
} yrc_bvh_view;

typedef struct yrc_bvh yrc_bvh; /* host-side built BVH (owned by the library) */

/* Fill `options` with BvhBuildOptions' defaults. */
void yrc_bvh_options_default(yrc_bvh_options* options);

/*
 * BuildBvh (src/accel/bvh_builder.cpp:269-286) on the host, multi-threaded,
 * producing the same nodes, primitive_indices and primitives, byte for byte,
 * as the reference builder for the same geometry and options. Returns
 * YRC_ERR_BUILD with the reference's error string for invalid geometry.
 */
yrc_status yrc_bvh_build(const yrc_geometry* geometry, const yrc_bvh_options* options, yrc_bvh** out);
/*
 * The same build with the hierarchy built on the current CUDA device: the
 * same nodes, primitive_indices and primitives, byte for byte. Where the
 * reference splits a range at the median (std::nth_element, used only when
 * every centroid extent of a range is below 1e-8 or its box has no area),
 * the host's own std::nth_element permutes that range (a subtree of at most
 * 64 refs that meets one is built by the host's serial builder) and the
 * device builds the rest. The median-split option is built on the host;
 * *built_on_device (optional) is 1 when the device built the hierarchy.
 * Synchronous. No counterpart in the reference (its builder is CPU-only).
 */
yrc_status yrc_bvh_build_device(const yrc_geometry* geometry, const yrc_bvh_options* options, yrc_bvh** out,
                                int32_t* built_on_device);
/* View of a built BVH; valid until yrc_bvh_destroy. */
yrc_status yrc_bvh_get_view(const yrc_bvh* bvh, yrc_bvh_view* view);
void yrc_bvh_destroy(yrc_bvh* bvh);

/* --------------------------------------------------------- two-level input */

/* One BLAS (RenderBlas, two_level_bvh.hpp:14-18). */
typedef struct yrc_blas_view {
    int32_t mesh_primitive;
    float object_bounds_min[3];
    float object_bounds_max[3];
    yrc_bvh_view bvh;
} yrc_blas_view;

/* PreparedMeshInstance (two_level_bvh.hpp:20-26). */
typedef struct yrc_prepared_instance {
    int32_t primitive;
    int32_t blas_index;
    float object_to_world[16];
    float world_to_object[16];
    float world_bounds_min[3];
    float world_bounds_max[3];
} yrc_prepared_instance;

/* RenderTlasPrimitive (two_level_bvh.hpp:28-33). kind: 0 instance, 1 sphere. */
typedef struct yrc_tlas_primitive {
    int32_t kind;
    int32_t instance;
    int32_t sphere;
    float world_bounds_min[3];
    float world_bounds_max[3];
} yrc_tlas_primitive;

/* TwoLevelBvh (two_level_bvh.hpp:42-46) as plain arrays. */
typedef struct yrc_two_level_view {
    const yrc_blas_view* blases;
    int32_t blas_count;
    const yrc_prepared_instance* instances;
    int32_t instance_count;
    const yrc_bvh_node* tlas_nodes;
    int64_t tlas_node_count;
    const int32_t* tlas_primitive_indices;
    int64_t tlas_primitive_index_count;
    const yrc_tlas_primitive* tlas_primitives;
    int64_t tlas_primitive_count;
    int32_t tlas_max_depth;
} yrc_two_level_view;

typedef struct yrc_two_level yrc_two_level; /* host-side built two-level BVH */

/* BuildTwoLevelBvh (src/accel/two_level_bvh.cpp:257-331) on the host. */
yrc_status yrc_two_level_build(const yrc_geometry* geometry, const yrc_bvh_options* options, yrc_two_level** out);
/* The same build with every BLAS built by yrc_bvh_build_device's device
 * path (byte-identical); the TLAS over the instances stays on the host.
 * *device_blases (optional) counts the BLASes the device built. No
 * counterpart in the reference. */
yrc_status yrc_two_level_build_device(const yrc_geometry* geometry, const yrc_bvh_options* options,
                                      yrc_two_level** out, int32_t* device_blases);
yrc_status yrc_two_level_get_view(const yrc_two_level* two_level, yrc_two_level_view* view);
void yrc_two_level_destroy(yrc_two_level* two_level);

/* ------------------------------------------------------ device accelerator */

typedef struct yrc_accel yrc_accel; /* geometry + BVH resident in HBM */

/*
 * Upload a flat BVH (the reference's RenderBvh arrays or yrc_bvh_build's) and
 * the triangles/spheres it references to the current CUDA device, in the
 * traversal layout the kernels read. The result of tracing is defined as the
 * result of IntersectBvh on the same geometry and BVH.
 */
yrc_status yrc_accel_create_flat(const yrc_geometry* geometry, const yrc_bvh_view* bvh, yrc_accel** out);
/* Same for a two-level BVH: the result is IntersectTwoLevelBvh's. */
yrc_status yrc_accel_create_two_level(const yrc_geometry* geometry, const yrc_two_level_view* two_level,
                                      yrc_accel** out);
void yrc_accel_destroy(yrc_accel* accel);

/* Bytes of device memory the accelerator holds. */
int64_t yrc_accel_device_bytes(const yrc_accel* accel);

/* ------------------------------------------------------------------- rays */

/* Ray3f + [t_min, t_max] (ray.hpp:7-23, bvh.hpp:107-114). 32 bytes. */
typedef struct yrc_ray {
    float origin[3];
    float t_min;
    float direction[3];
    float t_max;
} yrc_ray;

/*
 * BvhHit (bvh.hpp:89-98), compacted to 16 bytes. `id` >= 0 is the hit's
 * flat_triangle_index; -1 is a miss; id <= -2 is a hit on sphere (-2 - id).
 * On a miss t = the ray's t_max and u = v = 0, as IntersectBvh returns.
 */
typedef struct yrc_hit {
    float t;
    int32_t id;
    float u;
    float v;
} yrc_hit;

enum {
    YRC_TRACE_CLOSEST = 0, /* closest hit -> yrc_hit                               */
    YRC_TRACE_ANY = 1,     /* occlusion only -> uint8 per ray: IntersectBvh().hit    */
    YRC_TRACE_STATS = 2    /* also count node/triangle/sphere tests (BvhTraceStats) */
};

/* Per-ray work counters (BvhTraceStats, bvh.hpp:83-87), when requested. */
typedef struct yrc_trace_stats {
    uint64_t node_tests;
    uint64_t triangle_tests;
    uint64_t sphere_tests;
    uint64_t rays;
} yrc_trace_stats;

/*
 * Trace `count` rays held in DEVICE memory on `stream` (a cudaStream_t, or NULL
 * for the legacy default stream). flags: YRC_TRACE_CLOSEST writes `hits`
 * (and `instances`, per-ray instance index or -1, when non-NULL);
 * YRC_TRACE_ANY writes `occluded`. Asynchronous: returns after the launch.
 */
yrc_status yrc_trace_device(yrc_accel* accel, const yrc_ray* rays, int64_t count, int32_t flags,
                            yrc_hit* hits, int32_t* instances, uint8_t* occluded, void* stream);

/*
 * Same with HOST buffers: copies rays in, traces, copies results out, in
 * pipelined chunks on the library's own streams, and returns when the results
 * are in the host buffers. `stats` (optional) receives summed counters when
 * flags has YRC_TRACE_STATS.
 */
yrc_status yrc_trace_host(yrc_accel* accel, const yrc_ray* rays, int64_t count, int32_t flags,
                          yrc_hit* hits, int32_t* instances, uint8_t* occluded, yrc_trace_stats* stats);

/*
 * Per-ray BvhTraceStats for rays in device memory (diagnostics; same traversal
 * as the closest-hit kernel with counters). Arrays may be NULL.
 */
yrc_status yrc_trace_stats_device(yrc_accel* accel, const yrc_ray* rays, int64_t count, int32_t flags,
                                  uint32_t* node_tests, uint32_t* triangle_tests, uint32_t* sphere_tests,
                                  void* stream);

/* Rays per call accepted by yrc_trace_stats_device_noalloc. */
#define YRC_NOALLOC_STATS_MAX_RAYS 262144

/*
 * yrc_trace_stats_device without any device allocation. No counterpart in the
 * reference: it exists for callers of this library that cannot allocate.
 *
 * yrc_trace_stats_device takes a temporary buffer from the stream-ordered
 * allocator for the hit records that the counting traversal writes and then
 * discards. Some callers cannot let it: an application that hands all device
 * memory to its own pool at start-up (a later allocation fails, or takes
 * memory the pool counts on), or a per-frame loop that must never enter the
 * CUDA allocator. This variant calls no cudaMalloc, cudaFree or other
 * allocating routine; it uses a fixed scratch array that the library keeps on
 * every GPU that loads it, from load until the process exits
 * (256 + 16 * YRC_NOALLOC_STATS_MAX_RAYS bytes, just over 4 MiB).
 *
 * - count above YRC_NOALLOC_STATS_MAX_RAYS returns YRC_ERR_INVALID_ARGUMENT
 *   before any work is queued; split larger batches.
 * - The scratch array's device address is looked up (with the device current)
 *   and cached when an accelerator is created on that device, and the
 *   statistics kernels this accelerator uses are loaded then too. Under lazy
 *   module loading (the CUDA 12 default) both steps take device memory, so
 *   create the accelerator before the caller reserves its pool; later calls
 *   on it allocate nothing. Should the lookup have failed at creation, the
 *   first call retries it (and that retry may allocate): make the first call
 *   before any stream capture begins.
 * - All calls on one device share the scratch array, which keeps whatever the
 *   last call left there. The part that must start at zero (the ray-refill
 *   counter) is reset on `stream` before each launch; the rest is write-only.
 *   Calls whose GPU work overlaps (unordered streams, or several accelerators
 *   or host threads on one device) race on it and return wrong counts: order
 *   them, e.g. on one stream.
 * - Outputs are the per-ray counters of yrc_trace_stats_device; arrays may be
 *   NULL.
 */
yrc_status yrc_trace_stats_device_noalloc(yrc_accel* accel, const yrc_ray* rays, int64_t count, int32_t flags,
                                          uint32_t* node_tests, uint32_t* triangle_tests,
                                          uint32_t* sphere_tests, void* stream);

/*
 * Autotuner: times every compiled launch shape of the flat closest-hit (or,
 * with YRC_TRACE_ANY, any-hit) kernel on `count` device rays (results are
 * discarded) and keeps, for this accelerator, the lowest-numbered shape
 * within 2 % of the fastest (a choice that stays the same from run to run
 * when shapes time alike). `times_ms`
 * (optional, YRC_TRACE_SHAPES floats) receives the measured time per shape.
 * Synchronises `stream`.
 */
#define YRC_TRACE_SHAPES 17
yrc_status yrc_accel_autotune(yrc_accel* accel, const yrc_ray* rays, int64_t count, int32_t flags, void* stream,
                              float* times_ms);
/* Set / get the launch shape (0..YRC_TRACE_SHAPES-1) used for closest-hit
 * (any_hit = 0) or any-hit (any_hit = 1) traces; 0 is the default shape.
 * Shapes 0-6 differ in block size, node visits between ray refills and
 * register budget; shapes 7, 8 and 9 let a lane that reaches a leaf wait
 * until 4, 8 or 16 lanes of its warp are at leaves (or none is at an
 * interior node), so that the leaf tests run for many lanes at once;
 * shapes 10 and 11 are shape 8 with a 40-register budget (12 blocks of 128
 * per SM) and with blocks of 256, shape 12 is shape 9 with a 64-register
 * budget (8 blocks of 128 per SM; the two-level kernel needs more), and
 * shapes 13 and 14 are shape 8 refilling lanes every 16 and 32 steps
 * (every 2 and 4 steps measured slower), shapes 15 and 16 shape 8 with
 * register budgets for 9 and 10 blocks of 128 per SM. No
 * shape changes a hit: every ray keeps the reference's visiting order. */
yrc_status yrc_accel_set_trace_shape(yrc_accel* accel, int32_t any_hit, int32_t shape);
int32_t yrc_accel_get_trace_shape(const yrc_accel* accel, int32_t any_hit);

/* The launch shape of yrc_trace_host's traversal kernels: its chunks'
 * kernels run beside the chunks' host<->device copies, and the shape that
 * is fastest alone is not always the fastest there (on the 2M-triangle
 * set the leaf-batched shape 8 traverses 1.31x faster alone but the host
 * pipeline runs 8 % slower with it than with shape 10). autotune_host
 * times yrc_trace_host on `count` HOST rays (pinned memory, as the caller's
 * own) once per shape and keeps the lowest-numbered shape within 2 % of the
 * fastest; set_host_trace_shape(-1) makes the host path follow
 * yrc_accel_set_trace_shape again (the default). `times_ms` (optional,
 * YRC_TRACE_SHAPES floats) receives the wall time per call and shape.
 * Synchronous. No counterpart in the reference. */
yrc_status yrc_accel_autotune_host(yrc_accel* accel, const yrc_ray* rays, int64_t count, int32_t flags,
                                   float* times_ms);
yrc_status yrc_accel_set_host_trace_shape(yrc_accel* accel, int32_t any_hit, int32_t shape);
int32_t yrc_accel_get_host_trace_shape(const yrc_accel* accel, int32_t any_hit);

/* Four-wide traversal (opt-in). set_wide(1) builds, for a flat BVH of
 * triangles only, a four-wide copy of its hierarchy (the binary tree
 * collapsed two levels at a time, same node boxes and leaves) that later
 * closest- and any-hit traces without per-ray statistics traverse: half the
 * dependent node fetches and the same hits, since a triangle tie goes to the
 * smaller flat index whatever the visiting order (the reference pins BVH4 ==
 * binary hits in tests/accel/bvh_traversal_tests.cpp:112-138). It fails for
 * BVHs with spheres (a sphere tie goes to the first visited) and two-level
 * BVHs. Statistics and probes always use the binary traversal. Off by
 * default: on B200 it measured slower than the binary kernel (0.91x on
 * incoherent rays of the 2M-triangle set). No counterpart in the reference
 * (its BVH4 is a CPU path). */
yrc_status yrc_accel_set_wide(yrc_accel* accel, int32_t enable);
int32_t yrc_accel_get_wide(const yrc_accel* accel);

/* Ray reordering (opt-in) for yrc_trace_device and the autotuner: before a
 * closest- or any-hit trace of at least 65,536 rays, the rays are sorted by
 * a spatial key (a counting sort on the device, in the same stream) and the
 * traversal takes them in that order, so that rays which start close
 * together and head the same way share a warp. Hits are written per ray as
 * before and do not depend on the order. Modes: YRC_RAY_ORDER_OFF;
 * YRC_RAY_ORDER_DIRECTION (key: origin in the root box and direction);
 * YRC_RAY_ORDER_TWO_POINT (key: origin and the point `length` x the root
 * box diagonal along the ray). `key_bits` (8..24, 0 = about eight rays per
 * bin) sets the number of bins. The sort's buffers (8 bytes per ray plus 4
 * per bin) are allocated on the first trace that needs them and kept by the
 * accelerator. Statistics traces, probes and yrc_trace_host keep the
 * caller's order. No counterpart in the reference (its CPU traversal takes
 * rays one at a time, src/accel/bvh_traversal.cpp:253-345). */
#define YRC_RAY_ORDER_OFF 0
#define YRC_RAY_ORDER_DIRECTION 1
#define YRC_RAY_ORDER_TWO_POINT 2
yrc_status yrc_accel_set_ray_order(yrc_accel* accel, int32_t mode, int32_t key_bits, float length);
int32_t yrc_accel_get_ray_order(const yrc_accel* accel);

/* Per-launch device timing of yrc_trace_device: with timing on, each trace
 * records CUDA events in its stream around the reordering and around the
 * traversal kernel; last_timing waits for the last trace and returns both
 * durations in milliseconds (order_ms = 0 when the launch did not sort). */
yrc_status yrc_accel_set_timing(yrc_accel* accel, int32_t enable);
yrc_status yrc_accel_last_timing(yrc_accel* accel, float* order_ms, float* trace_ms);

/* ------------------------------------------------------------------ probe */

#define YRC_PROBE_MAX_HITS 64 /* BvhProbeHits::MaxHits (bvh.hpp:122-127) */

/* Per-ray probe target (IntersectAccelerationProbe arguments); -1 = none. */
typedef struct yrc_probe_target {
    int32_t primitive;
    int32_t instance;
    int32_t sphere;
    int32_t reserved;
} yrc_probe_target;

/*
 * IntersectAccelerationProbe (src/accel/acceleration.cpp:63-108) for rays in
 * device memory: up to 64 target hits per ray, in increasing t, written to
 * hits[ray * 64 + k] (instances likewise when non-NULL); counts[ray] = number
 * of hits; exhausted[ray] = 1 when more than 64 existed.
 */
yrc_status yrc_probe_device(yrc_accel* accel, const yrc_ray* rays, const yrc_probe_target* targets,
                            int64_t count, yrc_hit* hits, int32_t* instances, int32_t* counts,
                            uint8_t* exhausted, void* stream);

/*
 * Synchronise the device and report any error status a kernel recorded for
 * this accelerator since the last check (e.g. a traversal stack overflow,
 * which the depth check at creation rules out for well-formed BVHs).
 */
yrc_status yrc_accel_check(yrc_accel* accel);

/* ================================================================= render */

/* TextureFilter / TextureWrap (include/yaoray/scene/texture_options.hpp:7-17). */
enum {
    YRC_TEX_NEAREST = 0,
    YRC_TEX_BILINEAR = 1,
    YRC_TEX_TRILINEAR = 2,
    YRC_TEX_EWA = 3
};
enum {
    YRC_WRAP_REPEAT = 0,
    YRC_WRAP_CLAMP_TO_EDGE = 1,
    YRC_WRAP_MIRRORED_REPEAT = 2
};

/* RenderTexture (include/yaoray/scene/texture.hpp:37-51): an RGBA32F image
 * in the reference's texel order (row y at texels + 4 * y * width). width or
 * height <= 0, or texels NULL, is a texture without data, which samples as
 * (0, 0, 0, 1). Mip chains are built on the device at upload. */
typedef struct yrc_texture {
    int32_t width;
    int32_t height;
    const float* texels; /* width * height * 4 floats */
    int32_t filter;      /* YRC_TEX_* */
    int32_t wrap_s;      /* YRC_WRAP_* */
    int32_t wrap_t;
    int32_t reserved;
} yrc_texture;

/* SampleTexture4 (src/shading/texture.cpp:297-309) evaluated on the device
 * for n (u, v) pairs and, when `footprints` is not NULL, n TextureFootprints
 * (dudx, dvdx, dudy, dvdy); out receives n RGBA values. Nearest and bilinear
 * lookups are bit-identical to the reference's; trilinear and EWA lookups
 * can differ in the last bits of the level-of-detail blend (log2). The mip
 * chain is built for the call. Synchronous. */
yrc_status yrc_texture_sample_eval(const yrc_texture* texture, const float* uvs, const float* footprints, int64_t n,
                                   float* out);

/* BuildTextureMipChain (src/shading/texture.cpp:242-264) on the device:
 * writes every level, the image first, as RGBA texels into `texels`
 * (`capacity` texels), (width, height) per level into level_dims and the
 * number of levels into *level_count (0 for a texture without data). */
yrc_status yrc_texture_mip_chain_eval(const yrc_texture* texture, float* texels, int64_t capacity, int32_t* level_dims,
                                      int32_t* level_count);

/* MeasuredBrdf (include/yaoray/shading/measured_brdf.hpp:10-24): the RGL
 * tensors LoadMeasuredBrdf reads (src/shading/measured_brdf.cpp:33-190),
 * isotropic only (n_phi_i <= 2), row-major:
 *   ndf, sigma   [ndf_rows][ndf_cols]                   (theta_m x phi_m)
 *   vndf         [n_phi_i][n_theta_i][vndf_rows][vndf_cols]
 *   luminance    [n_phi_i][n_theta_i][res][res]
 *   spectra      [n_phi_i][n_theta_i][n_wavelengths][res][res]
 * The library builds the reference's five warps from them. */
typedef struct yrc_measured_brdf {
    int32_t n_theta_i;
    int32_t n_phi_i;
    int32_t n_wavelengths;
    int32_t ndf_rows;
    int32_t ndf_cols;
    int32_t vndf_rows;
    int32_t vndf_cols;
    int32_t res;
    const float* theta_i;
    const float* phi_i;
    const float* wavelengths;
    const float* ndf;
    const float* sigma;
    const float* vndf;
    const float* luminance;
    const float* spectra;
} yrc_measured_brdf;

/* EvaluateMeasured and PdfMeasured (src/shading/bsdf_measured.cpp:10-61,
 * 177-238) on the device for n rows of 9 floats (wo, wi, normal): f gets 3
 * floats per row, pdf 1. The warp arithmetic follows the reference's
 * (including its fused multiply-adds); the angles go through CUDA's
 * acosf/atan2f, so values agree within rounding. Synchronous. */
yrc_status yrc_measured_eval(const yrc_measured_brdf* brdf, const float* queries, int64_t n, float* f, float* pdf);

/* SampleMeasured (src/shading/bsdf_measured.cpp:67-128) on the device for n
 * rows of 8 floats (wo, normal, u.x, u.y): out gets 8 floats per row (wi,
 * weight, pdf, valid 0/1). Synchronous. */
yrc_status yrc_measured_sample(const yrc_measured_brdf* brdf, const float* queries, int64_t n, float* out);

/* RenderMaterialKind (include/yaoray/scene/material.hpp:7-19). */
enum {
    YRC_MAT_DIFFUSE = 0,
    YRC_MAT_CONDUCTOR = 1,
    YRC_MAT_DIELECTRIC = 2,
    YRC_MAT_THIN_DIELECTRIC = 3,
    YRC_MAT_COATED_DIFFUSE = 4,
    YRC_MAT_COATED_CONDUCTOR = 5,
    YRC_MAT_DIFFUSE_TRANSMISSION = 6,
    YRC_MAT_MIX = 7,
    YRC_MAT_MEASURED = 8,
    YRC_MAT_SUBSURFACE = 9,
    YRC_MAT_SUBSURFACE_EXIT = 10
};

/* RenderMaterial (material.hpp:31-65) with texture slots as indices into
 * yrc_scene_desc.textures. The reference samples three of them
 * (EvaluateMaterialAtSurface, src/shading/material_evaluator.cpp:112-180):
 * reflectance (multiplied in), alpha (a surface with alpha < 0.5 is skipped
 * by every ray) and the tangent-space normal map. */
typedef struct yrc_material {
    int32_t kind;
    float reflectance[3];
    float eta[3];
    float k[3];
    float ior;
    float uroughness;
    float vroughness;
    int32_t remap_roughness;
    int32_t mix_material_a;
    int32_t mix_material_b;
    float mix_amount;
    float coating_ior;
    float coating_roughness;
    float coat_thickness;
    float coat_absorption[3];
    int32_t coat_maxdepth;
    int32_t coat_nsamples;
    float sigma_a[3];
    float sigma_s[3];
    float bssrdf_eta;
    int32_t bssrdf_index;
    float emission[3];
    float alpha;
    float absorption_color[3];
    float absorption_distance;
    int32_t reflectance_texture; /* texture index or -1 */
    int32_t alpha_texture;       /* texture index or -1 (its red channel scales alpha) */
    int32_t normal_map;          /* texture index or -1 */
    int32_t measured_index;
    float normal_scale;          /* scales the normal map's tangent-space x and y (reference default 1) */
} yrc_material;

/* ---- Scattering functions evaluated on the device ------------------------
 * Diagnostics: each evaluates, in a CUDA kernel, the same device code the
 * path tracer shades with, on host inputs and outputs (synchronous), so that
 * it can be checked function by function against the reference's. */

/* EvaluateBsdf then PdfBsdf (src/shading/bsdf.cpp:17-148) for one material
 * (any kind but Measured, which has yrc_measured_eval) on n rows of 9 floats
 * (wo, wi, normal): f gets 3 floats per row, pdf 1. Each row's PCG32 stream
 * is Rng(seeds[i]) (include/yaoray/core/rng.hpp:15-48), drawn by the layered
 * kinds' stochastic walk (src/shading/bsdf_layered.cpp:13-349) in the
 * evaluation and then the pdf, as a path vertex evaluates a light sample. */
yrc_status yrc_bsdf_eval(const yrc_material* material, const float* queries, const uint64_t* seeds, int64_t n,
                         float* f, float* pdf);

/* SampleBsdf (src/shading/bsdf.cpp:150-310) on n rows of 8 floats (wo,
 * normal, u.x, u.y) with Rng(seeds[i]): out gets 9 floats per row (wi,
 * weight, pdf, valid 0/1, specular 0/1). */
yrc_status yrc_bsdf_sample(const yrc_material* material, const float* queries, const uint64_t* seeds, int64_t n,
                           float* out);

/* EmissivePrimitive (include/yaoray/scene/light.hpp:30-34). */
typedef struct yrc_emissive_primitive {
    int32_t primitive_index;
    float radiance[3];
    float area;
} yrc_emissive_primitive;

/* AliasTable (light.hpp:47-51); count 0 = no table. */
typedef struct yrc_alias_table {
    const float* probability;
    const int32_t* alias;
    const float* pmf;
    int32_t count;
} yrc_alias_table;

/* AnalyticLight (light.hpp:38-45). kind: 0 point, 1 spot, 2 distant. */
typedef struct yrc_analytic_light {
    int32_t kind;
    float position[3];
    float direction[3];
    float intensity[3];
    float cone_angle;
    float cone_cos_inner;
} yrc_analytic_light;

/* RenderEnvironment + its RenderTexture (RGBA32F texels, repeat-wrapped,
 * bilinear) + RenderEnvironmentDistribution (light.hpp:8-28). */
typedef struct yrc_environment {
    int32_t active;
    float radiance[3];
    float strength;
    float rotation_radians;
    int32_t width;
    int32_t height;
    const float* texels;          /* width * height * 4 floats, NULL = none */
    const float* texel_weights;   /* width * height, NULL = not sampleable */
    const float* row_weights;     /* height */
    const float* row_cdf;         /* height */
    const float* conditional_cdfs;/* width * height */
    float total_weight;
} yrc_environment;

/* BSSRDFTable (include/yaoray/shading/bssrdf.hpp). */
typedef struct yrc_bssrdf_table {
    int32_t rho_count;
    int32_t radius_count;
    const float* rho_samples;    /* rho_count */
    const float* radius_samples; /* radius_count */
    const float* profile;        /* rho_count * radius_count */
    const float* rho_eff;        /* rho_count */
    const float* profile_cdf;    /* rho_count * radius_count */
} yrc_bssrdf_table;

/*
 * ComputeBeamDiffusionBSSRDF (src/shading/bssrdf.cpp:124-151): fills a
 * rho_count x radius_count photon-beam-diffusion profile table for phase
 * asymmetry g and relative index eta (the reference uses 100 x 64 and g = 0
 * for every subsurface material). Bit-identical to the reference's table.
 */
yrc_status yrc_bssrdf_table_build(float g, float eta, int32_t rho_count, int32_t radius_count, float* rho_samples,
                                  float* radius_samples, float* profile, float* rho_eff, float* profile_cdf);

/* TabulatedBSSRDF(sigma_a, sigma_s, eta, table) (src/shading/bssrdf.cpp:
 * 153-266) on the device for n queries: sample_r[i] = Sample_Sr(channels[i],
 * u[i]) (-1 for a channel without extinction), pdf_sr[i] = Pdf_Sr(channels[i],
 * r[i]), sr[3i..3i+2] = Sr(r[i]). Channels are 0..2. */
yrc_status yrc_bssrdf_eval(const yrc_bssrdf_table* table, const float sigma_a[3], const float sigma_s[3], float eta,
                           const int32_t* channels, const float* u, const float* r, int64_t n, float* sample_r,
                           float* pdf_sr, float* sr);

/* TabulatedBSSRDF::Pdf_Sp (src/shading/bssrdf.cpp:244-266) on n rows of 18 floats
 * (po, ss, ts, ns, pi, ni): the area-measure pdf of exit point pi with normal
 * ni for entry po with shading frame (ss, ts, ns). */
yrc_status yrc_bssrdf_pdf_sp(const yrc_bssrdf_table* table, const float sigma_a[3], const float sigma_s[3], float eta,
                             const float* queries, int64_t n, float* pdf);

/* RenderCamera (include/yaoray/scene/camera.hpp:7-13). */
typedef struct yrc_camera {
    float origin[3];
    float forward[3];
    float right[3];
    float up[3];
    float fov_y_radians;
} yrc_camera;

/* RenderSettings (include/yaoray/scene/render_options.hpp:38-51). sampler:
 * RenderSamplerKind (0 independent, 1 stratified, 2 Owen-Sobol, 3 Z-Sobol). */
typedef struct yrc_render_settings {
    int32_t width;
    int32_t height;
    int32_t spp;
    int32_t max_depth;
    uint64_t seed;
    int32_t sampler;
    float radiance_clamp;
    int32_t adaptive_enabled;
    int32_t adaptive_min_spp;
    float adaptive_relative_error;
    float adaptive_absolute_error;
    float adaptive_confidence;
} yrc_render_settings;

/*
 * A RenderSceneIR plus its prepared acceleration structure. Vertex shading
 * normals (RenderVertex.normal) come from `normals` with `normal_stride`
 * bytes between vertices (NULL when no primitive has normals). Exactly one of
 * `flat` / `two_level` is non-NULL.
 */
typedef struct yrc_scene_desc {
    yrc_geometry geometry;
    const float* normals;
    int64_t normal_stride;
    const yrc_material* materials;
    int32_t material_count;
    const yrc_emissive_primitive* emissive;
    int32_t emissive_count;
    yrc_alias_table emissive_power;
    const yrc_analytic_light* analytic;
    int32_t analytic_count;
    yrc_alias_table analytic_power; /* count 0: built by the library from the lights' power */
    yrc_environment environment;
    const yrc_bssrdf_table* bssrdf_tables;
    int32_t bssrdf_count;
    yrc_camera camera;
    yrc_render_settings settings;
    const yrc_bvh_view* flat;
    const yrc_two_level_view* two_level;
    /* RenderVertex uv, tangent and tangent_handedness (geometry.hpp:12-18),
     * read for primitives whose flags say has_uvs / has_tangents: uv is 2
     * floats at uvs + k * uv_stride bytes, the tangent 3 floats followed by
     * the handedness at tangents + k * tangent_stride (NULL: none). */
    const float* uvs;
    int64_t uv_stride;
    const float* tangents;
    int64_t tangent_stride;
    const yrc_texture* textures;
    int32_t texture_count;
    /* RenderSceneIR::measured_brdfs, indexed by yrc_material.measured_index;
     * a Measured material whose index has no entry renders as the
     * reference's conductor fallback. */
    const yrc_measured_brdf* measured;
    int32_t measured_count;
} yrc_scene_desc;

/* FilmPixel (include/yaoray/film/film.hpp:19-28), byte-identical, 56 bytes. */
typedef struct yrc_film_pixel {
    float sum[3];
    uint32_t samples;
    float luminance_mean;
    float luminance_m2;
    float albedo_sum[3];
    float normal_sum[3];
    float depth_sum;
    uint32_t aov_samples;
} yrc_film_pixel;

/* RenderProgress (include/yaoray/runtime/backend.hpp:16-25). */
typedef struct yrc_render_progress {
    int32_t completed_spp;
    int32_t target_spp;
    uint64_t completed_samples;
    uint64_t target_samples;
    uint64_t active_pixels;
    uint64_t converged_pixels;
    uint64_t rays_traced;
    double elapsed_seconds;
} yrc_render_progress;

/*
 * Progress callback, called on the calling thread after each complete pass
 * with the film so far (host memory, width * height pixels) and the number of
 * non-finite samples dropped. Return non-zero to cancel the render; `error`
 * (capacity `error_capacity`) may then receive the reason.
 */
typedef int32_t (*yrc_progress_fn)(const yrc_render_progress* progress, const yrc_film_pixel* film,
                                    uint64_t bad_samples, void* user, char* error, size_t error_capacity);

/* RenderRequest (backend.hpp:33-38). `stop_flag` (optional) is polled between
 * passes; non-zero cancels like a stop_token. */
typedef struct yrc_render_request {
    const yrc_film_pixel* resume_film; /* host, width * height, or NULL */
    uint64_t resume_bad_samples;
    int32_t resume_completed_spp;
    const volatile int32_t* stop_flag;
    yrc_progress_fn progress;
    void* user;
} yrc_render_request;

/* RenderStats (backend.hpp:40-55). */
typedef struct yrc_render_stats {
    uint64_t samples_rendered;
    uint64_t converged_pixels;
    uint64_t rays_traced;
    uint64_t shadow_rays;
    uint64_t occluded_shadow_rays;
    uint64_t triangle_tests;
    uint64_t sphere_tests;
    uint64_t bvh_node_tests;
    int32_t bvh_nodes;
    int32_t bvh_max_depth;
    uint64_t hits;
    uint64_t misses;
    uint64_t bad_samples;
    int32_t threads;
    double elapsed_seconds;
    double device_seconds;
    uint64_t cache_queries;    /* paths ended at the radiance cache (0 without one) */
    uint64_t cache_records;    /* training records fed to the cache */
    uint64_t kernel_launches;  /* kernels this render launched on the device (graph kernel nodes included) */
} yrc_render_stats;

/*
 * Light-table builders for callers that prepare scenes themselves (the same
 * tables the reference's PrepareLightSampling / BuildEnvironmentDistribution
 * produce): BuildAliasTable (src/lighting/light_sampling.cpp:148-183) into
 * caller arrays of `count`; BuildEnvironmentDistribution
 * (src/lighting/environment.cpp:73-123) for RGBA texels (NULL = black).
 */
yrc_status yrc_alias_table_build(const float* weights, int32_t count, float* probability, int32_t* alias,
                                 float* pmf);
yrc_status yrc_environment_distribution_build(const float* texels, int32_t width, int32_t height,
                                              float* texel_weights, float* row_weights, float* row_cdf,
                                              float* conditional_cdfs, float* total_weight);

typedef struct yrc_render_scene yrc_render_scene;

/* CudaBackend::Prepare (src/runtime/cuda_stub_backend.cpp:20-28): uploads the
 * scene and its acceleration structure. Fails with YRC_ERR_UNSUPPORTED for
 * scene features the device does not shade (analytic lights). */
yrc_status yrc_render_scene_create(const yrc_scene_desc* desc, yrc_render_scene** out);
void yrc_render_scene_destroy(yrc_render_scene* scene);
int64_t yrc_render_scene_device_bytes(const yrc_render_scene* scene);

/* Queue capacity of the wavefront (paths in flight per batch). By default
 * max(pixels, 2^21), bounded to whole passes of the image: at least one
 * pass, at most min(spp, 64). set_capacity(0) restores the default; any
 * other value is bounded the same way. The film does not depend on it: a
 * batch renders whole passes and the film adds samples in pass order.
 * No counterpart in the reference. */
yrc_status yrc_render_scene_set_capacity(yrc_render_scene* scene, int64_t capacity);
int64_t yrc_render_scene_capacity(const yrc_render_scene* scene);

/* Render autotuner: times short probe renders of this scene (sample indices
 * 0..P-1 of every pixel, P = two batches of the largest candidate) for each
 * candidate queue capacity (whole passes of the image between 2^17 and 2^23
 * paths) and each traversal launch shape at the best capacity (one shape
 * for the extend and the shadow traversals; shapes 7-16 batch the leaf tests
 * of a warp, in the shadow-transmittance kernel too); keeps the fastest
 * for later yrc_render calls. The traversal stack depth is not a candidate:
 * it follows the BVH's measured depth (64 or 256 entries). Probes run
 * without an attached radiance cache (they do not train it). Synchronous.
 * No counterpart in the reference. */
#define YRC_TUNE_CAPACITY 1
#define YRC_TUNE_TRACE_SHAPE 2
typedef struct yrc_render_tuning {
    int64_t capacity;          /* chosen queue capacity */
    int32_t trace_shape;       /* chosen traversal launch shape (extend and shadow rays) */
    int32_t candidates;        /* configurations timed */
    double seconds_per_sample; /* device time per sample of the chosen configuration */
} yrc_render_tuning;
yrc_status yrc_render_autotune(yrc_render_scene* scene, int32_t flags, yrc_render_tuning* result);
/* Applies a tuning (capacity and traversal launch shape; the other fields
 * are ignored), e.g. one found by yrc_render_autotune on a scene of the same
 * image size and spp. */
yrc_status yrc_render_scene_set_tuning(yrc_render_scene* scene, const yrc_render_tuning* tuning);

/*
 * CudaBackend::Render (cuda_stub_backend.cpp:30-37) for the Path integrator:
 * the pass loop of RenderCpuPathTrace (src/backends/cpu/cpu_path_tracer.cpp:
 * 39-229) on the device. `film_out` (host, width * height) receives the
 * film; `bad_samples_out` the film's non-finite sample count. On
 * cancellation returns YRC_ERR_CANCELLED with the reference's message
 * ("render cancelled" or the callback's text) and leaves film_out untouched.
 */
yrc_status yrc_render(yrc_render_scene* scene, const yrc_render_request* request, yrc_film_pixel* film_out,
                      uint64_t* bad_samples_out, yrc_render_stats* stats);

/*
 * Renders `count` prepared scenes together: after each scene's setup (as in
 * yrc_render), every step launches ONE CUDA graph that holds the batch graph
 * of every scene still rendering, so uneven jobs share each launch and one
 * host synchronisation; a scene that finishes leaves the combined graph.
 * Per scene the results equal yrc_render's (films byte for byte). requests
 * (optional, per scene) may resume and stop, not report progress; scenes
 * must differ, share one device, and not share a radiance cache.
 * stats[i].device_seconds and *device_seconds (optional) are the device time
 * of the whole call. No counterpart in the reference.
 */
yrc_status yrc_render_many(yrc_render_scene* const* scenes, int32_t count, const yrc_render_request* requests,
                           yrc_film_pixel* const* films_out, uint64_t* bad_samples_out, yrc_render_stats* stats,
                           double* device_seconds);

/*
 * yrc_render_many with pooled traversal: every step is ONE graph launch in
 * which, per bounce, the extend rays of all scenes still rendering are
 * traced by ONE persistent traversal kernel and their shadow rays by ONE
 * shadow kernel (each lane takes a ray from any scene's queue through a
 * device job table and works with that scene's BVH and outputs), while the
 * scenes' generate, shading, next-event and film stages run as parallel
 * branches of the graph. Scenes in one pooled launch share the BVH kind and
 * stack class; a call with both kinds makes one launch per kind. At most
 * 128 scenes per call; otherwise the arguments, results (films byte for
 * byte equal to yrc_render's) and limits are yrc_render_many's. No
 * counterpart in the reference (its CpuWorkerPool renders one job per
 * pass loop, src/backends/cpu/cpu_path_tracer.cpp:109-160).
 */
yrc_status yrc_render_pooled(yrc_render_scene* const* scenes, int32_t count, const yrc_render_request* requests,
                             yrc_film_pixel* const* films_out, uint64_t* bad_samples_out, yrc_render_stats* stats,
                             double* device_seconds);

/*
 * TraceShadowVisibility (src/integrators/path_direct_lighting.cpp:23-113) for
 * n caller rays (host, synchronous) through the scene's own shadow stage, the
 * code the path tracer runs for its next-event rays: each ray's origin,
 * direction and t_max = max_distance, t_min = the first query's t_min (the
 * reference uses 1e-5). `transmittance` gets 4 floats per ray: the RGB
 * transmittance and 1 when visible, all 0 when occluded. No counterpart in
 * the reference's public API (its loop is internal to the integrator).
 */
yrc_status yrc_render_scene_shadow_eval(yrc_render_scene* scene, const yrc_ray* rays, int64_t n,
                                        float* transmittance);

/* A new camera and sampler seed (RenderSettings::seed) for a prepared scene,
 * e.g. the next frame of a camera path: the next yrc_render draws that view.
 * The scene's working memory and captured batch are kept, so that render
 * pays no allocation or capture. An attached radiance cache stays attached.
 * No counterpart in the reference (its prepared scene is immutable). */
yrc_status yrc_render_scene_set_view(yrc_render_scene* scene, const yrc_camera* camera, uint64_t seed);

/* Wait for all work the library queued on `stream` (NULL = legacy default). */
yrc_status yrc_stream_synchronize(void* stream);

/* ------------------------------------------------------------------------
 * Neural radiance cache. No counterpart in the reference (its renderer has
 * no learned component): a multiresolution hash grid over the scene box
 * (16 levels x 2 fp16 features, 2^19 entries per level, resolutions 16 to
 * 2048) plus degree-0..3 spherical harmonics of the view direction and the
 * surface attributes, into a 64-wide MLP (5 hidden ReLU layers, exp RGB
 * output) run on the tensor cores in bf16 with fp32 accumulation, trained
 * with a relative-L2 loss and Adam (lr 1e-2, betas 0.9 / 0.99).
 *
 * A query is 16 floats: position[3], roughness, direction[3] (unit, away
 * from the surface towards the viewer of the cached radiance), normal[3],
 * diffuse albedo[3], specular albedo[3]. Targets and outputs are float4 RGB
 * (w unused). Query, target and output arrays are device memory.
 * ---------------------------------------------------------------------- */
typedef struct yrc_nrc yrc_nrc;

#define YRC_NRC_QUERY_FLOATS 16
#define YRC_NRC_WEIGHT_COUNT (6 * 64 * 64) /* 6 matrices [out][in]; output rows 3..63 zero */
#define YRC_NRC_GRID_COUNT (16 * 524288 * 2)

/* Creates a cache on the current device for positions in the cube
 * [box_lo, box_lo + box_extent]^3; weights and grid from `seed`. */
yrc_status yrc_nrc_create(const float box_lo[3], float box_extent, uint64_t seed, yrc_nrc** out);
void yrc_nrc_destroy(yrc_nrc* cache);

/* Makes `dst` an exact copy of `src` (same device): parameters, optimiser
 * moments, step count, moving average and its decay, and the encoding's box.
 * Synchronous. For evaluating a trained cache several times from the same
 * state. No counterpart in the reference. */
yrc_status yrc_nrc_copy_state(yrc_nrc* dst, yrc_nrc* src);

/* Host copies of the fp32 master parameters (either pointer may be NULL). */
yrc_status yrc_nrc_set_params(yrc_nrc* cache, const float* weights, const float* grid);
yrc_status yrc_nrc_get_params(yrc_nrc* cache, float* weights_out, float* grid_out);

/* The exponential moving average of the parameters that every optimiser
 * step updates (decay min(d, (1 + t) / (10 + t)) at step t, d = 0.99 unless
 * set by yrc_nrc_set_average_decay, restarted at
 * the parameters by yrc_nrc_create / yrc_nrc_set_params), same layout as
 * yrc_nrc_get_params. No counterpart in the reference. */
yrc_status yrc_nrc_get_averaged_params(yrc_nrc* cache, float* weights_out, float* grid_out);

/* Sets the largest decay of that moving average (default 0.99; [0, 1)).
 * Optimiser steps already captured in a prepared scene's batch graph keep
 * the decay they were captured with: set it before attaching the cache. */
yrc_status yrc_nrc_set_average_decay(yrc_nrc* cache, float decay);

/* rgb[i] = cache(queries[i]) for n queries, asynchronous on `stream`. */
yrc_status yrc_nrc_infer(yrc_nrc* cache, const float* queries, int64_t n, float* rgb, void* stream);

/* One optimiser step on n (query, target) pairs, asynchronous on `stream`;
 * `loss_out` (device float, optional) receives the sum of per-sample losses
 * (divide by 3n for the mean). */
yrc_status yrc_nrc_train_step(yrc_nrc* cache, const float* queries, const float* targets, int64_t n,
                              float* loss_out, void* stream);

/* Gradients of the mean loss over n pairs without an optimiser step
 * (synchronous; host outputs, each optional): YRC_NRC_WEIGHT_COUNT and
 * YRC_NRC_GRID_COUNT floats, and the mean loss. */
yrc_status yrc_nrc_gradients(yrc_nrc* cache, const float* queries, const float* targets, int64_t n,
                             float* weight_grads, float* grid_grads, float* loss);

/* Synchronises and reports a tensor-core wait that timed out. */
yrc_status yrc_nrc_check(yrc_nrc* cache);

/* How the path tracer uses an attached radiance cache. */
typedef struct yrc_cache_settings {
    float spread_threshold; /* end a path once its spread exceeds this x its primary footprint (0.01) */
    int32_t train_one_in;   /* 1 in this many paths runs unbiased and trains the cache (16) */
    int32_t train_records;  /* training records per batch (65536) */
    int32_t train;          /* 0 freezes the cache (inference only) */
    int32_t train_steps;    /* optimiser steps per batch on that batch's records (1) */
    int32_t delta_vertices; /* 1: paths may also end at specular (delta) vertices (0) */
    int32_t averaged;       /* 1: query the moving average of the parameters (0: the raw ones) */
} yrc_cache_settings;

/* Attaches `cache` (NULL detaches) to a prepared scene: subsequent
 * yrc_render calls end paths at the cache when the footprint heuristic fires
 * and, unless frozen, train it on the unbiased training paths once per
 * batch. No counterpart in the reference. The cache must outlive the
 * attachment. */
yrc_status yrc_render_scene_set_cache(yrc_render_scene* scene, yrc_nrc* cache, const yrc_cache_settings* settings);

/* ---- Sampling primitives evaluated on the device ------------------------
 * Diagnostics: each evaluates, in a CUDA kernel, the same device code the
 * path tracer draws its samples with, on host inputs and outputs
 * (synchronous). */

/* Sampler::Sample1D / Sample2D (src/sampling/sampler.cpp:173-237) of the sampler
 * `kind` (RenderSamplerKind) constructed for each query's pixel and sample.
 * `queries` holds n rows of 6 int32 (x, y, sample, bounce, dimension, lane);
 * a negative bounce counts as 0. `out` receives n floats (two_d == 0) or
 * 2n floats (x, y per row). */
yrc_status yrc_sampler_eval(int32_t kind, uint64_t seed, int32_t spp, const int32_t* queries, int64_t n,
                            int32_t two_d, float* out);

/* Rng(seed) (include/yaoray/core/rng.hpp:15-48) for each of the n seeds,
 * followed by `draws` calls of NextFloat; out is n x draws floats. */
yrc_status yrc_rng_eval(const uint64_t* seeds, int64_t n, int32_t draws, float* out);

/* SeedForPixelSample(seed, x, y, sample) (src/sampling/sampler.cpp:304-310)
 * for n rows of 3 int64 (x, y, sample). */
yrc_status yrc_pixel_seed_eval(uint64_t seed, const int64_t* queries, int64_t n, uint64_t* out);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* YRCUDA_H */
