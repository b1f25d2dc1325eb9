/*
 * yr_oracle.h — CPU restatement of the reference (QiuRuhai/YaoRay) hot path in
 * plain C, used ONLY as a test oracle and as the portable CPU baseline. It is
 * checked against the reference itself (oracle/_ref, built from the reference
 * sources by oracle/Makefile) and against golden vectors generated from it
 * (tests/golden). The product (libyrcuda) never links or calls it.
 *
 * Arrays use the reference's in-memory layouts: 32-byte RenderBvhNode,
 * RenderBvhPrimitive as 5 ints, positions as float triples with a byte stride.
 */
#ifndef YR_ORACLE_H
#define YR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct yo_node {
    float lo[3], hi[3];
    int32_t payload_offset, primitive_count;
} yo_node;

typedef struct yo_prim {
    int32_t kind, mesh_primitive, sphere, local_triangle, flat_triangle_index;
} yo_prim;

typedef struct yo_geometry {
    const float* positions; /* first vertex position                 */
    int64_t vertex_count;
    int64_t vertex_stride;  /* bytes between vertices                 */
    const uint32_t* indices;
    int64_t index_count;
    const uint32_t* prim_first_count; /* (first_index, index_count) per mesh primitive */
    int32_t primitive_count;
    const float* spheres; /* cx, cy, cz, radius */
    int32_t sphere_count;
} yo_geometry;

typedef struct yo_bvh {
    const yo_node* nodes;
    int64_t node_count;
    const int32_t* primitive_indices;
    int64_t primitive_index_count;
    const yo_prim* primitives;
    int64_t primitive_count;
} yo_bvh;

typedef struct yo_hit {
    int32_t hit;
    float t;
    int32_t triangle_index;
    int32_t mesh_primitive;
    int32_t instance;
    int32_t sphere;
    float u, v;
} yo_hit;

typedef struct yo_stats {
    uint64_t node_tests, triangle_tests, sphere_tests;
} yo_stats;

/* IntersectBvh (src/accel/bvh_traversal.cpp:253-345). */
yo_hit yo_intersect_bvh(const yo_geometry* g, const yo_bvh* bvh, const float origin[3], const float dir[3],
                        float t_min, float t_max, yo_stats* stats);

/* Two-level: TLAS primitives as (kind, instance, sphere) triples; instances as
 * (blas_index, world_to_object[16]); blases as an array of yo_bvh.
 * IntersectTwoLevelBvh (src/accel/two_level_bvh.cpp:365-481). */
typedef struct yo_two_level {
    const yo_bvh* blases;
    int32_t blas_count;
    const int32_t* instance_blas;      /* per instance */
    const float* instance_w2o;         /* 16 floats per instance, column-major */
    int32_t instance_count;
    const yo_node* tlas_nodes;
    int64_t tlas_node_count;
    const int32_t* tlas_primitive_indices;
    int64_t tlas_primitive_index_count;
    const int32_t* tlas_primitives;    /* kind, instance, sphere per TLAS primitive */
    int64_t tlas_primitive_count;
} yo_two_level;

yo_hit yo_intersect_two_level(const yo_geometry* g, const yo_two_level* tl, const float origin[3],
                              const float dir[3], float t_min, float t_max, yo_stats* stats);

/* Batched drivers over rays of 8 floats (origin, t_min, direction, t_max). */
void yo_trace_flat(const yo_geometry* g, const yo_bvh* bvh, const float* rays, int64_t n, yo_hit* hits,
                   uint32_t* node_tests, uint32_t* tri_tests, uint32_t* sphere_tests, int threads);
void yo_trace_two_level(const yo_geometry* g, const yo_two_level* tl, const float* rays, int64_t n, yo_hit* hits,
                        uint32_t* node_tests, uint32_t* tri_tests, uint32_t* sphere_tests, int threads);

/* IntersectAccelerationProbe (src/accel/acceleration.cpp:63-108) over a flat
 * (tl == NULL) or two-level accelerator. hits: 64 per ray. */
void yo_probe(const yo_geometry* g, const yo_bvh* flat, const yo_two_level* tl, const float* rays, int64_t n,
              const int32_t* targets /* prim, instance, sphere per ray */, int32_t* counts, uint8_t* exhausted,
              yo_hit* hits);

/* Sampler (src/sampling/sampler.cpp): kind 0 Independent, 1 Stratified,
 * 2 OwenSobol, 3 ZSobol. queries: (x, y, sample, bounce, dim, lane). */
void yo_sampler(int kind, uint64_t seed, int spp, const int32_t* queries, int64_t n, int two_d, float* out);
uint64_t yo_seed_for_pixel_sample(uint64_t seed, int x, int y, int sample);
/* Rng (include/yaoray/core/rng.hpp): first `count` NextFloat draws. */
void yo_rng_floats(uint64_t seed, int count, float* out);

/* GeneratePerspectiveCameraRay (src/scene/camera.cpp:20-39). camera: origin,
 * forward, right, up, fov_y. out: origin + direction per row. */
void yo_camera_rays(const float* camera, int width, int height, const int32_t* pixels, const float* samples,
                    int64_t n, float* out);

/* Film::AddSample (src/film/film.cpp:160-183) over 13-float sample rows;
 * pixels_out: 14 x 4 bytes per pixel in FilmPixel order. Returns bad count. */
uint64_t yo_film_accumulate(int width, int height, const float* samples, int64_t n, void* pixels_out);

/* RenderTexture lookups (src/shading/texture.cpp): SampleTexture4 after
 * BuildTextureMipChain. texels: RGBA32F rows; filter 0 nearest, 1 bilinear,
 * 2 trilinear, 3 EWA; wrap 0 repeat, 1 clamp-to-edge, 2 mirrored repeat.
 * uvs: 2 floats per lookup; footprints: 4 per lookup (dudx, dvdx, dudy,
 * dvdy) or NULL; out: 4 per lookup. */
void yo_texture_sample(int width, int height, const float* texels, int filter, int wrap_s, int wrap_t,
                       const float* uvs, const float* footprints, int64_t n, float* out);
/* BuildTextureMipChain: the levels after the image, one after the other, in
 * `out` (sized for width * height + 64 texels suffices); dims: (w, h) per
 * level. Returns the number of levels written. */
int yo_texture_mip_chain(int width, int height, const float* texels, int wrap_s, int wrap_t, float* out,
                         int32_t* dims);

#ifdef __cplusplus
}
#endif

#endif
