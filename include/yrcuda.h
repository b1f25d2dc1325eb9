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

/*
 * Autotuner: times every compiled launch shape of the flat closest-hit (or,
 * with YRC_TRACE_ANY, any-hit) kernel on `count` device rays (results are
 * discarded) and keeps the fastest for this accelerator. `times_ms`
 * (optional, YRC_TRACE_SHAPES floats) receives the measured time per shape.
 * Synchronises `stream`.
 */
#define YRC_TRACE_SHAPES 7
yrc_status yrc_accel_autotune(yrc_accel* accel, const yrc_ray* rays, int64_t count, int32_t flags, void* stream,
                              float* times_ms);
/* Set / get the launch shape (0..YRC_TRACE_SHAPES-1) used for closest-hit
 * (any_hit = 0) or any-hit (any_hit = 1) traces; 0 is the default shape. */
yrc_status yrc_accel_set_trace_shape(yrc_accel* accel, int32_t any_hit, int32_t shape);
int32_t yrc_accel_get_trace_shape(const yrc_accel* accel, int32_t any_hit);

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

/* Wait for all work the library queued on `stream` (NULL = legacy default). */
yrc_status yrc_stream_synchronize(void* stream);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* YRCUDA_H */
