// Device-resident render scene and wavefront path state.
//
// HBM layout (structure of arrays, one slot per in-flight path):
//   * geometry for shading: per flat triangle its mesh primitive (int32) and
//     its three vertex indices (int4); vertex positions and normals as float4;
//   * materials as a compact 128-byte record per RenderMaterial;
//   * lights: emissive primitives, their alias table, a per-emissive-primitive
//     cumulative triangle-area table (the reference scans triangles linearly;
//     the same float cumulative sums searched by bisection select the same
//     triangle), and a primitive -> emissive index map;
//   * path state: ray (2 x float4, the trace kernels' yrc_ray layout),
//     throughput, radiance, previous-bounce MIS data, medium state, PCG state,
//     first-hit AOVs, and three pending next-event contributions.
#pragma once

#include <cstdint>

#include "device_layout.cuh"
#include "texture.cuh"

namespace yrc {

struct DevEnvironment {
    int32_t active;
    float radiance[3];
    float strength;
    float rotation;
    int32_t width, height;
    const float* texels;  // RGBA
    const float* texel_weights;
    const float* row_weights;
    const float* row_cdf;
    const float* conditional_cdfs;
    float total_weight;
};

// The view a render draws: RenderCamera (include/yaoray/scene/camera.hpp:
// 7-13) with tan(fov_y / 2) computed on the host, and RenderSettings::seed.
struct alignas(16) DevView {
    float cam_origin[3], cam_forward[3], cam_right[3], cam_up[3];
    float cam_half_height;
    uint64_t seed;
};

struct alignas(16) DevMaterial {
    int32_t kind;
    float reflectance[3];
    float ior;
    float uroughness;
    float vroughness;
    float coating_ior;
    float coat_thickness;
    float coat_absorption[3];
    int32_t coat_maxdepth;
    int32_t coat_nsamples;
    float emission[3];
    float absorption_color[3];
    float absorption_distance;
    float sigma_a[3];
    float sigma_s[3];
    float bssrdf_eta;
    int32_t bssrdf_index;
    int32_t reflectance_texture;  // scene texture indices, -1 = none
    int32_t alpha_texture;
    int32_t normal_map;
    float alpha;
    float normal_scale;
    int32_t measured_index;  // into DevScene::measured, -1 = none
    int32_t pad;
};

struct DevBssrdf {
    int32_t rho_count, radius_count;
    const float* rho;
    const float* radius;
    const float* profile;
    const float* rho_eff;
    const float* profile_cdf;
};

struct DevAnalytic {
    int32_t kind;
    float position[3];
    float direction[3];
    float intensity[3];
    float cone_angle;
    float cone_cos_inner;
};

// LightTreeNode (include/yaoray/scene/light.hpp:53-59).
struct DevLightNode {
    float lo[3], hi[3];
    float power;
    int32_t left, right, light_index;
};

struct DevMeasuredBrdf;  // measured.cuh

struct DevScene {
    AccelParams accel;
    // shading geometry
    const int32_t* tri_prim;      // flat triangle -> mesh primitive
    const int4* tri_vertices;     // flat triangle -> vertex indices (w unused)
    const float4* positions;      // per vertex
    const float4* normals;        // per vertex (w unused), may be null
    const int32_t* prim_material; // per mesh primitive
    const uint32_t* prim_flags;   // per mesh primitive (bit0 has_normals)
    const int32_t* sphere_material;
    const float4* spheres;        // center.xyz, radius
    const int32_t* sphere_flip;
    const float* instance_o2w;    // 16 floats per instance (column-major)
    const uint8_t* tri_clear;     // per flat triangle: 1 if its material passes light (Dielectric / ThinDielectric)
    const uint8_t* sphere_clear;  // per sphere, likewise
    int32_t primitive_count;
    int32_t sphere_count;
    int32_t instance_count;
    // materials
    const DevMaterial* materials;
    int32_t material_count;
    // emissive lights
    int32_t emissive_count;
    const int32_t* emissive_prim;
    const float* emissive_radiance;  // 3 per emissive
    const float* emissive_area;
    const float* alias_prob;
    const int32_t* alias_index;
    const float* alias_pmf;
    int32_t alias_count;            // 0: linear power selection
    float total_emissive_power;
    const int32_t* emissive_tri_offset;  // per emissive: first entry in tri_cdf / tri_local
    const int32_t* emissive_tri_count;
    const float* tri_cdf;               // cumulative triangle areas
    const int32_t* tri_local;           // local triangle index of each entry
    const float* emissive_prim_area;    // sum of triangle areas per emissive primitive
    const int32_t* prim_emissive;       // mesh primitive -> first emissive index or -1
    // analytic lights
    int32_t analytic_count;
    const DevAnalytic* analytic;
    const float* analytic_alias_prob;
    const int32_t* analytic_alias_index;
    const float* analytic_alias_pmf;   // null: uniform selection
    const DevLightNode* analytic_tree;  // power/distance tree (more than 8 lights, none distant)
    int32_t analytic_tree_root;         // -1: no tree
    // environment
    DevEnvironment env;
    // subsurface
    const DevBssrdf* bssrdf;
    int32_t bssrdf_count;
    // camera and sampler seed: device memory, so that a new view of a
    // resident scene is one small copy and the captured batch stays valid
    const DevView* view;
    // settings
    int32_t width, height, spp, max_depth, sampler;
    float radiance_clamp;
    int32_t any_transparent;  // scene has Dielectric / ThinDielectric materials
    int32_t any_subsurface;   // scene has Subsurface materials (probe stage needed)
    // textured shading
    const float2* uvs;           // per vertex, may be null
    const float4* tangents;      // per vertex: tangent xyz, handedness in w; may be null
    const DevTexture* textures;  // texture_count entries
    int32_t texture_count;
    const float* ewa_weights;
    const DevMeasuredBrdf* measured;  // measured BRDFs (RGL warps)
    int32_t measured_count;
    int32_t any_alpha;      // a material can cut surfaces out (alpha < 0.5 or an alpha texture)
    int32_t exact_shadows;  // shadow rays take the per-thread reference loop (cut-outs, textured thin glass)
    int32_t any_layered;    // scene has coated (layered) materials, whose vertices defer their next events
};

// Path state, structure of arrays over `capacity` slots.
struct PathState {
    int32_t* pixel;       // pixel index
    int32_t* sample;      // sample index (Sobol)
    float4* throughput;   // xyz, w = unused
    float4* radiance;     // xyz
    float4* prev;         // origin xyz, bsdf pdf
    uint32_t* flags;      // bit0 prev valid, bit1 prev delta, bit2 medium active, bit3 primary hit, bit4 done
    float4* medium;       // absorption colour xyz, distance
    uint64_t* rng_state;
    uint64_t* rng_inc;
    float4* aov_albedo;   // xyz, w = depth
    float4* aov_normal;
    float4* nee;          // 3 per path: contribution xyz (before throughput), w unused
    float4* nee_tp;       // throughput at the vertex that made the NEE samples
    float* nee_vis;       // 3 per path: shadow transmittance (1 visible, 0 occluded)
    float2* spread;       // radiance cache: primary footprint a0, running spread sum
    // Coated (layered) vertices, whose BSDF draws from the PCG32 stream: 5 per
    // path, the vertex kept across the deferred next-event stages
    // (LayeredNeeKernel, LayeredContinueKernel): [0] position + material
    // index bits, [1] shading normal, [2] direction to the viewer, [3]
    // reflectance (texture scale applied), [4] the pending light direction +
    // its pdf (emissive) or cosine (environment).
    float4* defer;
};

// Radiance-cache stage of the path tracer (device pointers; all counts live
// in `counters`: [0] cache queries, [1] training paths, [2] training records).
struct CacheArgs {
    int32_t enabled;
    float spread_c;        // terminate when spread^2 > spread_c * a0
    int32_t train_one_in;  // 1 in train_one_in paths traces unbiased for training
    int32_t delta_vertices;  // paths may also end at delta vertices
    int32_t train_paths;   // capacity of the training-path slots
    int32_t train_records; // capacity of the training records
    int32_t max_depth;
    float target_max;      // bound on a training target's largest component
    float* queries;        // per terminated path: 16-float query
    int32_t* query_path;
    float4* query_tp;      // throughput at the query vertex
    float4* query_base;    // path radiance up to and including the query vertex's emission
    float4* query_rgb;     // cache output
    int32_t* train_slot;   // per path: training slot or -1
    int32_t* slot_path;    // per training slot: path
    int32_t* slot_len;     // per training slot: recorded vertices
    float* slot_q;         // train_paths * max_depth queries
    float4* slot_lt;       // train_paths * max_depth * 2: radiance before the vertex, throughput
    float* rec_q;          // training records: queries
    float4* rec_t;         //                   targets
    unsigned long long* counters;
};

constexpr uint32_t kPathPrevValid = 1u << 0;
constexpr uint32_t kPathPrevDelta = 1u << 1;
constexpr uint32_t kPathMedium = 1u << 2;
constexpr uint32_t kPathPrimary = 1u << 3;
constexpr uint32_t kPathNee = 1u << 5;  // pending next-event contributions
constexpr uint32_t kPathCacheQueued = 1u << 6;  // the path's image estimate already ended at the cache
// A deferred coated vertex's pending shadow rays: emissive (slot 0),
// analytic (slot 1), environment (slot 2).
constexpr uint32_t kPathDeferEmissive = 1u << 7;
constexpr uint32_t kPathDeferAnalytic = 1u << 8;
constexpr uint32_t kPathDeferEnvironment = 1u << 9;

// Work queues (device counters live in a small array).
struct Queues {
    float4* ray_in;       // 2 per entry
    int32_t* path_in;     // path slot per entry
    float4* hits;         // closest hit per entry (t, id, u, v)
    int32_t* inst;        // instance per entry
    float4* ray_out;      // next bounce rays
    int32_t* path_out;
    float4* shadow_ray;   // 2 per shadow entry
    int32_t* shadow_slot; // path * 3 + light type
    uint8_t* shadow_occluded;
    int32_t* shadow_overflow;  // shadow entries the exact loop traces (see ShadowArgs::overflow)
    int32_t* defer_paths;      // coated vertices awaiting their emissive shadow ray (kCtrDefer)
    int32_t* defer_paths2;     // ... and then their analytic / environment shadow rays (kCtrDefer2)
    int32_t* nee_paths;   // paths with pending NEE
    // Subsurface probes (BSSRDF entry -> probe traversal -> exit), one per
    // path at most: probe_ray 2 per entry (base.xyz + t_min, direction.xyz +
    // length: the yrc_ray layout), target (mesh primitive, instance, sphere,
    // path), probe_entry 2 per entry (entry point.xyz + selection sample,
    // entry normal.xyz + material index bits); the probe stage writes the
    // selected target hit (t, id, u, v) and the number of target hits.
    float4* probe_ray;
    int4* probe_target;
    float4* probe_entry;
    float4* probe_hit;
    int32_t* probe_count;
    float4* tex_normal;   // texture stage: final shading normal per entry, w = 1 when textured
    float4* tex_scale;    // texture stage: reflectance scale per entry
    int32_t* order;       // extend-queue entries sorted by shading class
    uint8_t* shade_class; // shading class per extend-queue entry
    unsigned long long* counters;  // see kCounter*
};

enum CounterIndex {
    kCtrIn = 0,
    kCtrOut = 1,
    kCtrShadow = 2,
    kCtrNee = 3,
    kCtrClass0 = 4,  // entries per shading class (kShadeClasses of them)
    kCtrProbe = 10,  // subsurface probes queued at this depth
    kCtrDefer = 11,  // entries in defer_paths
    kCtrTrace = 12,  // traversal work counter
    kCtrShadowTrace = 13,
    kCtrShadowOverflow = 14,  // entries in shadow_overflow
    kCtrDefer2 = 15,  // entries in defer_paths2
    kCtrStatsBase = 16,  // rays, shadow rays, occluded, hits, misses, bad
    kCtrCursor0 = 24,  // scatter cursors per shading class
    kCtrSamplesDone = 30,  // film samples summed over the pixels after a render
    kCtrCount = 32,
};

// Shading classes: the extend queue is sorted by class before shading and
// each class is shaded by its own kernel instance, whose BSDF dispatch folds
// to the class's one material kind (coherent warps, fewer registers).
enum ShadeClass {
    kClassMiss = 0,
    kClassDiffuse = 1,       // Diffuse and the default material
    kClassConductor = 2,
    kClassDielectric = 3,
    kClassCoatedDiffuse = 4,
    kClassGeneric = 5,       // every other kind, and invalid materials
    kShadeClasses = 6,
};

}  // namespace yrc
