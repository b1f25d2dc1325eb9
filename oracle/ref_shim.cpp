// C shim over the reference implementation's own C++ API, compiled together
// with the reference sources into oracle/_ref/libyaoray_ref.so by
// oracle/Makefile. TEST INFRASTRUCTURE ONLY: it lets the Python tests and the
// CPU-baseline leg of the benchmark call the unmodified reference functions
// (BuildBvh, BuildRenderAcceleration, IntersectBvh, IntersectTwoLevelBvh,
// IntersectAccelerationProbe, Sampler, Rng, GeneratePerspectiveCameraRay, Film,
// LoadPbrtScene/CompilePbrtScene and the CPU backend) on plain arrays.
#include <yaoray/accel/acceleration.hpp>
#include <yaoray/accel/bvh.hpp>
#include <yaoray/accel/two_level_bvh.hpp>
#include <yaoray/backends/cpu/cpu_backend.hpp>
#include <yaoray/core/rng.hpp>
#include <yaoray/film/film.hpp>
#include <yaoray/frontend/pbrt/pbrt_scene.hpp>
#include <yaoray/frontend/pbrt/scene_compiler.hpp>
#include <yaoray/runtime/backend.hpp>
#include <yaoray/sampling/sampler.hpp>
#include <yaoray/scene/camera.hpp>
#include <yaoray/scene/render_scene.hpp>
#include <yaoray/shading/texture.hpp>
#include <yaoray/shading/measured_brdf.hpp>
#include "shading/bsdf_internal.hpp"
#include "yrcuda.h"

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

namespace {

struct RefScene {
    yr::RenderSceneIR ir;
    yr::RenderAcceleration accel;
    bool built = false;
    std::string error;
};

thread_local std::string g_last_error;

int ResolveThreads(int threads) {
    if (threads > 0) return threads;
    const int hw = static_cast<int>(std::thread::hardware_concurrency());
    return hw > 0 ? hw : 1;
}

void NodeToFloats(const yr::RenderBvhNode& node, void* out) {
    std::memcpy(out, &node, sizeof(yr::RenderBvhNode));
}

template <typename F>
void ParallelFor(std::int64_t n, int threads, F&& body) {
    threads = ResolveThreads(threads);
    if (threads <= 1 || n < 1024) {
        for (std::int64_t i = 0; i < n; ++i) body(i, 0);
        return;
    }
    // Static interleave, as the reference's own benchmark harness does.
    std::vector<std::thread> pool;
    pool.reserve(static_cast<std::size_t>(threads));
    for (int w = 0; w < threads; ++w) {
        pool.emplace_back([&, w] {
            for (std::int64_t i = w; i < n; i += threads) body(i, w);
        });
    }
    for (auto& t : pool) t.join();
}

} // namespace

extern "C" {

const char* yrref_last_error() { return g_last_error.c_str(); }

// ---------------------------------------------------------------- geometry ---
// positions: 3 floats per vertex; prims: first_index, index_count per mesh
// primitive; spheres: cx, cy, cz, radius; instances: primitive index + 16-float
// column-major object_to_world.
void* yrref_scene_create(const float* positions, std::int64_t vertex_count,
    const std::uint32_t* indices, std::int64_t index_count,
    const std::uint32_t* prims, int prim_count,
    const float* spheres, int sphere_count,
    const int* instance_prims, const float* instance_o2w, int instance_count) {
    auto* scene = new RefScene();
    scene->ir.vertices.resize(static_cast<std::size_t>(vertex_count));
    for (std::int64_t i = 0; i < vertex_count; ++i) {
        scene->ir.vertices[i].position = yr::Point3f{positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]};
    }
    scene->ir.indices.assign(indices, indices + index_count);
    for (int p = 0; p < prim_count; ++p) {
        yr::RenderPrimitive prim;
        prim.first_index = prims[2 * p];
        prim.index_count = prims[2 * p + 1];
        scene->ir.primitives.push_back(prim);
    }
    for (int s = 0; s < sphere_count; ++s) {
        yr::RenderSphere sphere;
        sphere.center = yr::Point3f{spheres[4 * s], spheres[4 * s + 1], spheres[4 * s + 2]};
        sphere.radius = spheres[4 * s + 3];
        scene->ir.spheres.push_back(sphere);
    }
    for (int i = 0; i < instance_count; ++i) {
        yr::RenderInstance inst;
        inst.primitive = yr::MeshPrimitiveHandle{instance_prims[i]};
        std::copy(instance_o2w + 16 * i, instance_o2w + 16 * i + 16, inst.object_to_world.m.begin());
        scene->ir.instances.push_back(inst);
    }
    return scene;
}

void yrref_scene_destroy(void* handle) { delete static_cast<RefScene*>(handle); }

// split_method: 0 = SAH bucket binning, 1 = longest-axis median.
// Returns the number of build errors (0 on success); the first error is in
// yrref_last_error().
int yrref_scene_build(void* handle, int split_method, int max_leaf, int threads) {
    auto* scene = static_cast<RefScene*>(handle);
    yr::BvhBuildOptions options;
    options.split_method = split_method == 1 ? yr::BvhSplitMethod::LongestAxisMedian
                                             : yr::BvhSplitMethod::SahBucketBinning;
    options.max_leaf_triangles = max_leaf;
    options.thread_count = threads;
    yr::RenderAccelerationBuildResult result = yr::BuildRenderAcceleration(scene->ir.Geometry(), options);
    scene->accel = std::move(result.acceleration);
    scene->built = result.errors.empty();
    g_last_error = result.errors.empty() ? std::string() : result.errors.front();
    return static_cast<int>(result.errors.size());
}

int yrref_scene_is_two_level(void* handle) {
    return static_cast<RefScene*>(handle)->accel.kind == yr::RenderAccelerationKind::TwoLevel ? 1 : 0;
}

// counts[0..3] = nodes, primitive_indices, primitives, max_depth of a RenderBvh.
static void BvhCounts(const yr::RenderBvh& bvh, std::int64_t* counts) {
    counts[0] = static_cast<std::int64_t>(bvh.nodes.size());
    counts[1] = static_cast<std::int64_t>(bvh.primitive_indices.size());
    counts[2] = static_cast<std::int64_t>(bvh.primitives.size());
    counts[3] = bvh.max_depth;
}

// nodes: 32 bytes each (the RenderBvhNode bytes); primitives: 5 ints each
// (kind, mesh_primitive, sphere, local_triangle, flat_triangle_index).
static void BvhCopy(const yr::RenderBvh& bvh, void* nodes, int* primitive_indices, int* primitives) {
    for (std::size_t i = 0; i < bvh.nodes.size(); ++i) {
        NodeToFloats(bvh.nodes[i], static_cast<char*>(nodes) + 32 * i);
    }
    std::copy(bvh.primitive_indices.begin(), bvh.primitive_indices.end(), primitive_indices);
    for (std::size_t i = 0; i < bvh.primitives.size(); ++i) {
        const yr::RenderBvhPrimitive& p = bvh.primitives[i];
        primitives[5 * i + 0] = p.kind == yr::BvhPrimitiveKind::Triangle ? 0 : 1;
        primitives[5 * i + 1] = p.mesh_primitive.Value();
        primitives[5 * i + 2] = p.sphere.Value();
        primitives[5 * i + 3] = p.local_triangle;
        primitives[5 * i + 4] = p.flat_triangle_index;
    }
}

void yrref_flat_counts(void* handle, std::int64_t* counts) {
    BvhCounts(static_cast<RefScene*>(handle)->accel.flat, counts);
}

void yrref_flat_copy(void* handle, void* nodes, int* primitive_indices, int* primitives) {
    BvhCopy(static_cast<RefScene*>(handle)->accel.flat, nodes, primitive_indices, primitives);
}

// counts[0..5] = blases, instances, tlas nodes, tlas primitive_indices,
// tlas primitives, tlas max_depth.
void yrref_two_level_counts(void* handle, std::int64_t* counts) {
    const yr::TwoLevelBvh& tl = static_cast<RefScene*>(handle)->accel.two_level;
    counts[0] = static_cast<std::int64_t>(tl.blases.size());
    counts[1] = static_cast<std::int64_t>(tl.instances.size());
    counts[2] = static_cast<std::int64_t>(tl.tlas.nodes.size());
    counts[3] = static_cast<std::int64_t>(tl.tlas.primitive_indices.size());
    counts[4] = static_cast<std::int64_t>(tl.tlas.primitives.size());
    counts[5] = tl.tlas.max_depth;
}

void yrref_blas_counts(void* handle, int blas, std::int64_t* counts) {
    BvhCounts(static_cast<RefScene*>(handle)->accel.two_level.blases[blas].bvh, counts);
}

// object_bounds: 6 floats (min xyz, max xyz); mesh_primitive: 1 int.
void yrref_blas_copy(void* handle, int blas, void* nodes, int* primitive_indices, int* primitives,
    float* object_bounds, int* mesh_primitive) {
    const yr::RenderBlas& b = static_cast<RefScene*>(handle)->accel.two_level.blases[blas];
    BvhCopy(b.bvh, nodes, primitive_indices, primitives);
    const float bounds[6] = {b.object_bounds.min.x, b.object_bounds.min.y, b.object_bounds.min.z,
        b.object_bounds.max.x, b.object_bounds.max.y, b.object_bounds.max.z};
    std::copy(bounds, bounds + 6, object_bounds);
    *mesh_primitive = b.primitive.Value();
}

// Per instance: primitive, blas_index, object_to_world[16], world_to_object[16], world_bounds[6].
void yrref_instances_copy(void* handle, int* primitive, int* blas_index, float* o2w, float* w2o, float* bounds) {
    const yr::TwoLevelBvh& tl = static_cast<RefScene*>(handle)->accel.two_level;
    for (std::size_t i = 0; i < tl.instances.size(); ++i) {
        const yr::PreparedMeshInstance& inst = tl.instances[i];
        primitive[i] = inst.primitive.Value();
        blas_index[i] = inst.blas_index;
        std::copy(inst.object_to_world.m.begin(), inst.object_to_world.m.end(), o2w + 16 * i);
        std::copy(inst.world_to_object.m.begin(), inst.world_to_object.m.end(), w2o + 16 * i);
        const float b[6] = {inst.world_bounds.min.x, inst.world_bounds.min.y, inst.world_bounds.min.z,
            inst.world_bounds.max.x, inst.world_bounds.max.y, inst.world_bounds.max.z};
        std::copy(b, b + 6, bounds + 6 * i);
    }
}

// TLAS primitives: 3 ints each (kind 0 = instance / 1 = sphere, instance, sphere).
void yrref_tlas_copy(void* handle, void* nodes, int* primitive_indices, int* primitives) {
    const yr::RenderTlas& tlas = static_cast<RefScene*>(handle)->accel.two_level.tlas;
    for (std::size_t i = 0; i < tlas.nodes.size(); ++i) {
        NodeToFloats(tlas.nodes[i], static_cast<char*>(nodes) + 32 * i);
    }
    std::copy(tlas.primitive_indices.begin(), tlas.primitive_indices.end(), primitive_indices);
    for (std::size_t i = 0; i < tlas.primitives.size(); ++i) {
        const yr::RenderTlasPrimitive& p = tlas.primitives[i];
        primitives[3 * i + 0] = p.kind == yr::TlasPrimitiveKind::Instance ? 0 : 1;
        primitives[3 * i + 1] = p.instance.Value();
        primitives[3 * i + 2] = p.sphere.Value();
    }
}

// ------------------------------------------------------------------ tracing ---
// rays: 8 floats each (origin xyz, t_min, direction xyz, t_max).
// Outputs per ray (any pointer may be null): t, triangle_index, sphere,
// mesh_primitive, instance, u, v, hit flag, node_tests, triangle_tests,
// sphere_tests. Runs IntersectAcceleration (flat: IntersectBvh; instanced:
// IntersectTwoLevelBvh) on `threads` std::threads in a static interleave.
void yrref_trace(void* handle, const float* rays, std::int64_t n,
    float* t_out, int* tri_out, int* sphere_out, int* prim_out, int* inst_out,
    float* u_out, float* v_out, std::uint8_t* hit_out,
    std::uint32_t* node_tests, std::uint32_t* tri_tests, std::uint32_t* sphere_tests, int threads) {
    auto* scene = static_cast<RefScene*>(handle);
    const yr::GeometryView geometry = scene->ir.Geometry();
    ParallelFor(n, threads, [&](std::int64_t i, int) {
        const float* r = rays + 8 * i;
        const yr::Ray3f ray{yr::Point3f{r[0], r[1], r[2]}, yr::Vec3f{r[4], r[5], r[6]}};
        yr::BvhTraceStats stats;
        const yr::BvhHit hit = yr::IntersectAcceleration(geometry, scene->accel, ray, stats, r[3], r[7]);
        if (t_out) t_out[i] = hit.t;
        if (tri_out) tri_out[i] = hit.triangle_index;
        if (sphere_out) sphere_out[i] = hit.sphere.Value();
        if (prim_out) prim_out[i] = hit.mesh_primitive.Value();
        if (inst_out) inst_out[i] = hit.instance.Value();
        if (u_out) u_out[i] = hit.bary_u;
        if (v_out) v_out[i] = hit.bary_v;
        if (hit_out) hit_out[i] = hit.hit ? 1 : 0;
        if (node_tests) node_tests[i] = static_cast<std::uint32_t>(stats.node_tests);
        if (tri_tests) tri_tests[i] = static_cast<std::uint32_t>(stats.triangle_tests);
        if (sphere_tests) sphere_tests[i] = static_cast<std::uint32_t>(stats.sphere_tests);
    });
}

// Throughput helper for the CPU baseline: closest hit (or hit flag only when
// any_hit != 0) over n rays, no per-ray stats. Returns the number of hits.
std::int64_t yrref_trace_count(void* handle, const float* rays, std::int64_t n, int any_hit,
    float* t_out, int* tri_out, int threads) {
    auto* scene = static_cast<RefScene*>(handle);
    const yr::GeometryView geometry = scene->ir.Geometry();
    std::atomic<std::int64_t> hits{0};
    threads = ResolveThreads(threads);
    std::vector<std::int64_t> per(static_cast<std::size_t>(threads), 0);
    ParallelFor(n, threads, [&](std::int64_t i, int w) {
        const float* r = rays + 8 * i;
        const yr::Ray3f ray{yr::Point3f{r[0], r[1], r[2]}, yr::Vec3f{r[4], r[5], r[6]}};
        yr::BvhTraceStats stats;
        const yr::BvhHit hit = yr::IntersectAcceleration(geometry, scene->accel, ray, stats, r[3], r[7]);
        if (hit.hit) ++per[static_cast<std::size_t>(w)];
        if (!any_hit) {
            if (t_out) t_out[i] = hit.t;
            if (tri_out) tri_out[i] = hit.triangle_index;
        } else if (tri_out) {
            tri_out[i] = hit.hit ? 1 : 0;
        }
    });
    for (std::int64_t v : per) hits += v;
    return hits.load();
}

// IntersectAccelerationProbe for each ray; targets per ray: primitive,
// instance, sphere (-1 = none). Outputs: count, exhausted flag, and up to 64
// hits per ray (t, triangle_index, instance, u, v).
void yrref_probe(void* handle, const float* rays, std::int64_t n,
    const int* target_prim, const int* target_inst, const int* target_sphere,
    int* count_out, std::uint8_t* exhausted_out, float* t_out, int* tri_out, int* inst_out,
    float* u_out, float* v_out, int threads) {
    auto* scene = static_cast<RefScene*>(handle);
    const yr::GeometryView geometry = scene->ir.Geometry();
    ParallelFor(n, threads, [&](std::int64_t i, int) {
        const float* r = rays + 8 * i;
        const yr::Ray3f ray{yr::Point3f{r[0], r[1], r[2]}, yr::Vec3f{r[4], r[5], r[6]}};
        const yr::BvhProbeHits hits = yr::IntersectAccelerationProbe(geometry, scene->accel, ray,
            yr::MeshPrimitiveHandle{target_prim[i]}, yr::InstanceHandle{target_inst[i]},
            yr::SphereHandle{target_sphere[i]}, r[3], r[7]);
        count_out[i] = hits.count;
        exhausted_out[i] = hits.exhausted ? 1 : 0;
        for (int k = 0; k < hits.count; ++k) {
            const std::int64_t o = i * yr::BvhProbeHits::MaxHits + k;
            t_out[o] = hits.hits[k].t;
            tri_out[o] = hits.hits[k].triangle_index;
            inst_out[o] = hits.hits[k].instance.Value();
            u_out[o] = hits.hits[k].bary_u;
            v_out[o] = hits.hits[k].bary_v;
        }
    });
}

// ------------------------------------------------------------------ sampler ---
// queries: n rows of (x, y, sample, bounce, dim, lane) ints; kind is the
// RenderSamplerKind value; two_d selects Sample2D (out gets 2 floats per row).
void yrref_sampler(int kind, std::uint64_t seed, int spp, const int* queries, std::int64_t n,
    int two_d, float* out) {
    for (std::int64_t i = 0; i < n; ++i) {
        const int* q = queries + 6 * i;
        yr::Sampler sampler(static_cast<yr::RenderSamplerKind>(kind), seed, q[0], q[1], q[2], spp, 1);
        sampler.BeginBounce(q[3]);
        const auto dim = static_cast<yr::SampleDimension>(q[4]);
        if (two_d) {
            const yr::Vec2f v = sampler.Sample2D(dim, q[5]);
            out[2 * i] = v.x;
            out[2 * i + 1] = v.y;
        } else {
            out[i] = sampler.Sample1D(dim, q[5]);
        }
    }
}

std::uint64_t yrref_seed_for_pixel_sample(std::uint64_t seed, int x, int y, int sample) {
    return yr::SeedForPixelSample(seed, x, y, sample);
}

// ------------------------------------------------------------------ texture ---
// An RGBA32F image prepared as the reference prepares scene textures
// (BuildTextureSamplingCaches) and looked up with SampleTexture4; footprints
// are 4 floats per lookup or NULL (no footprint).
static yr::RenderTexture MakeTexture(int width, int height, const float* texels, int filter, int wrap_s,
    int wrap_t) {
    yr::RenderTexture t;
    t.width = width;
    t.height = height;
    if (texels && width > 0 && height > 0) {
        t.texels.resize(static_cast<std::size_t>(width) * static_cast<std::size_t>(height));
        for (std::size_t i = 0; i < t.texels.size(); ++i) {
            t.texels[i] = yr::Color4f{texels[4 * i], texels[4 * i + 1], texels[4 * i + 2], texels[4 * i + 3]};
        }
    }
    t.filter = static_cast<yr::TextureFilter>(filter);
    t.wrap_s = static_cast<yr::TextureWrap>(wrap_s);
    t.wrap_t = static_cast<yr::TextureWrap>(wrap_t);
    return t;
}

void yrref_texture_sample(int width, int height, const float* texels, int filter, int wrap_s, int wrap_t,
    const float* uvs, const float* footprints, std::int64_t n, float* out) {
    std::vector<yr::RenderTexture> textures;
    textures.push_back(MakeTexture(width, height, texels, filter, wrap_s, wrap_t));
    yr::BuildTextureSamplingCaches(textures);
    for (std::int64_t i = 0; i < n; ++i) {
        const yr::Vec2f uv{uvs[2 * i], uvs[2 * i + 1]};
        yr::TextureFootprint f;
        if (footprints) f = yr::TextureFootprint{footprints[4 * i], footprints[4 * i + 1], footprints[4 * i + 2],
            footprints[4 * i + 3]};
        const yr::Color4f c = yr::SampleTexture4(textures[0], uv, f);
        out[4 * i] = c.x;
        out[4 * i + 1] = c.y;
        out[4 * i + 2] = c.z;
        out[4 * i + 3] = c.w;
    }
}

// BuildTextureMipChain: the levels after the image into `out`, (w, h) per
// level into dims; returns the level count.
int yrref_texture_mip_chain(int width, int height, const float* texels, int wrap_s, int wrap_t, float* out,
    int* dims) {
    yr::RenderTexture t = MakeTexture(width, height, texels, 1, wrap_s, wrap_t);
    yr::BuildTextureMipChain(t);
    std::size_t at = 0;
    for (std::size_t l = 0; l < t.mip_levels.size(); ++l) {
        dims[2 * l] = t.mip_levels[l].width;
        dims[2 * l + 1] = t.mip_levels[l].height;
        for (const yr::Color4f& c : t.mip_levels[l].texels) {
            out[at++] = c.x;
            out[at++] = c.y;
            out[at++] = c.z;
            out[at++] = c.w;
        }
    }
    return static_cast<int>(t.mip_levels.size());
}

// ------------------------------------------------------------ measured BRDF ---
// A MeasuredBrdf from the C-ABI arrays, with its five warps built exactly as
// LoadMeasuredBrdf builds them from a tensor file.
static std::shared_ptr<yr::MeasuredBrdf> MakeMeasured(const yrc_measured_brdf& b) {
    auto m = std::make_shared<yr::MeasuredBrdf>();
    const std::size_t nv = static_cast<std::size_t>(b.n_phi_i) * b.n_theta_i;
    m->theta_i.assign(b.theta_i, b.theta_i + b.n_theta_i);
    m->phi_i.assign(b.phi_i, b.phi_i + b.n_phi_i);
    m->wavelengths.assign(b.wavelengths, b.wavelengths + b.n_wavelengths);
    const std::size_t nd = static_cast<std::size_t>(b.ndf_rows) * b.ndf_cols;
    m->ndf.assign(b.ndf, b.ndf + nd);
    m->sigma.assign(b.sigma, b.sigma + nd);
    m->vndf.assign(b.vndf, b.vndf + nv * b.vndf_rows * b.vndf_cols);
    m->luminance.assign(b.luminance, b.luminance + nv * b.res * b.res);
    m->spectra.assign(b.spectra, b.spectra + nv * b.n_wavelengths * b.res * b.res);
    m->isotropic = b.n_phi_i <= 2;
    m->res = b.res;
    m->ndf_warp = yr::PiecewiseLinear2D<0>(m->ndf.data(), b.ndf_cols, b.ndf_rows, {}, {}, false, false);
    m->sigma_warp = yr::PiecewiseLinear2D<0>(m->sigma.data(), b.ndf_cols, b.ndf_rows, {}, {}, false, false);
    m->vndf_warp = yr::PiecewiseLinear2D<2>(m->vndf.data(), b.vndf_cols, b.vndf_rows, {b.n_phi_i, b.n_theta_i},
                                            {m->phi_i.data(), m->theta_i.data()}, true, true);
    m->luminance_warp = yr::PiecewiseLinear2D<2>(m->luminance.data(), b.res, b.res, {b.n_phi_i, b.n_theta_i},
                                                 {m->phi_i.data(), m->theta_i.data()}, true, true);
    m->spectra_warp = yr::PiecewiseLinear2D<3>(m->spectra.data(), b.res, b.res,
                                               {b.n_phi_i, b.n_theta_i, b.n_wavelengths},
                                               {m->phi_i.data(), m->theta_i.data(), m->wavelengths.data()},
                                               false, false);
    return m;
}

// EvaluateMeasured / PdfMeasured for rows of (wo, wi, normal).
void yrref_measured_eval(const yrc_measured_brdf* b, const float* q, std::int64_t n, float* f, float* pdf) {
    const auto m = MakeMeasured(*b);
    for (std::int64_t i = 0; i < n; ++i) {
        const float* r = q + 9 * i;
        const yr::Vec3f wo{r[0], r[1], r[2]}, wi{r[3], r[4], r[5]}, nn{r[6], r[7], r[8]};
        const yr::Color3f c = yr::EvaluateMeasured(*m, wo, wi, nn);
        f[3 * i] = c.x;
        f[3 * i + 1] = c.y;
        f[3 * i + 2] = c.z;
        pdf[i] = yr::PdfMeasured(*m, wo, wi, nn);
    }
}

// SampleMeasured for rows of (wo, normal, u): out rows (wi, weight, pdf, valid).
void yrref_measured_sample(const yrc_measured_brdf* b, const float* q, std::int64_t n, float* out) {
    const auto m = MakeMeasured(*b);
    for (std::int64_t i = 0; i < n; ++i) {
        const float* r = q + 8 * i;
        const yr::BsdfSample s = yr::SampleMeasured(*m, yr::Vec3f{r[0], r[1], r[2]}, yr::Vec3f{r[3], r[4], r[5]},
                                                    yr::Vec2f{r[6], r[7]});
        float* o = out + 8 * i;
        o[0] = s.wi.x;
        o[1] = s.wi.y;
        o[2] = s.wi.z;
        o[3] = s.weight.x;
        o[4] = s.weight.y;
        o[5] = s.weight.z;
        o[6] = s.pdf;
        o[7] = s.valid ? 1.0f : 0.0f;
    }
}

// First `count` NextFloat() draws of Rng(seed).
void yrref_rng_floats(std::uint64_t seed, int count, float* out) {
    yr::Rng rng(seed);
    for (int i = 0; i < count; ++i) out[i] = rng.NextFloat();
}

// camera: origin[3], forward[3], right[3], up[3], fov_y_radians. Rows of
// (pixel_x, pixel_y) ints with (sample_x, sample_y) floats; out: 6 floats
// (origin, direction) per row.
void yrref_camera_rays(const float* camera, int width, int height, const int* pixels,
    const float* samples, std::int64_t n, float* out) {
    yr::RenderCamera cam;
    cam.origin = yr::Point3f{camera[0], camera[1], camera[2]};
    cam.forward = yr::Vec3f{camera[3], camera[4], camera[5]};
    cam.right = yr::Vec3f{camera[6], camera[7], camera[8]};
    cam.up = yr::Vec3f{camera[9], camera[10], camera[11]};
    cam.fov_y_radians = camera[12];
    for (std::int64_t i = 0; i < n; ++i) {
        const yr::Ray3f ray = yr::GeneratePerspectiveCameraRay(cam, width, height,
            pixels[2 * i], pixels[2 * i + 1], yr::Vec2f{samples[2 * i], samples[2 * i + 1]});
        out[6 * i + 0] = ray.origin.x;
        out[6 * i + 1] = ray.origin.y;
        out[6 * i + 2] = ray.origin.z;
        out[6 * i + 3] = ray.direction.x;
        out[6 * i + 4] = ray.direction.y;
        out[6 * i + 5] = ray.direction.z;
    }
}

// Film::AddSample over a sample stream. samples: rows of 11 floats
// (x, y, beauty rgb, albedo rgb, normal xyz) + depth + primary flag are given
// as 13 floats per row: x, y, beauty[3], albedo[3], normal[3], depth, primary.
// pixels_out: 14 floats per pixel in FilmPixel field order (sum[3], samples
// as float-cast uint bits, mean, m2, albedo_sum[3], normal_sum[3], depth_sum,
// aov_samples bits). Returns the bad-sample count.
std::uint64_t yrref_film_accumulate(int width, int height, const float* samples, std::int64_t n,
    void* pixels_out) {
    yr::Film film(width, height);
    for (std::int64_t i = 0; i < n; ++i) {
        const float* s = samples + 13 * i;
        yr::FilmSample fs;
        fs.beauty = yr::Color3f{s[2], s[3], s[4]};
        fs.albedo = yr::Color3f{s[5], s[6], s[7]};
        fs.normal = yr::Vec3f{s[8], s[9], s[10]};
        fs.depth = s[11];
        fs.primary_hit = s[12] != 0.0f;
        film.AddSample(static_cast<int>(s[0]), static_cast<int>(s[1]), fs);
    }
    static_assert(sizeof(yr::FilmPixel) == 56);
    std::memcpy(pixels_out, film.Pixels().data(), film.Pixels().size() * sizeof(yr::FilmPixel));
    return film.BadSampleCount();
}

} // extern "C"

// ============================================================== rendering ==
// RenderJobs for the CPU backend: loaded from a PBRT file through the
// reference frontend (LoadPbrtScene + CompilePbrtScene) or assembled from the
// C-ABI scene description, exported back as arrays, and rendered with
// CpuBackend::Prepare / Render.

#include "yrcuda.h"

#include <yaoray/lighting/environment.hpp>
#include <yaoray/lighting/light_sampling.hpp>
#include <yaoray/shading/bssrdf.hpp>
#include "integrators/path_integrator_internal.hpp"

namespace {

struct RefJob {
    yr::RenderSceneIR ir;
    yr::RenderSettings settings;
    std::vector<float> alias_prob;
    std::vector<int> alias_index;
    std::vector<float> alias_pmf;
};

void CopyRgb(const yr::Color3f& c, float* out) {
    out[0] = c.x;
    out[1] = c.y;
    out[2] = c.z;
}

yr::Color3f Rgb(const float* c) { return yr::Color3f{c[0], c[1], c[2]}; }

yr::RenderMaterial MaterialFrom(const yrc_material& m) {
    yr::RenderMaterial r;
    r.kind = static_cast<yr::RenderMaterialKind>(m.kind);
    r.reflectance.value = Rgb(m.reflectance);
    r.eta.value = Rgb(m.eta);
    r.k.value = Rgb(m.k);
    r.ior = m.ior;
    r.uroughness.value = m.uroughness;
    r.vroughness.value = m.vroughness;
    r.remap_roughness = m.remap_roughness != 0;
    r.coating_ior = m.coating_ior;
    r.coating_roughness.value = m.coating_roughness;
    r.coat_thickness = m.coat_thickness;
    r.coat_absorption = Rgb(m.coat_absorption);
    r.coat_maxdepth = m.coat_maxdepth;
    r.coat_nsamples = m.coat_nsamples;
    r.sigma_a = Rgb(m.sigma_a);
    r.sigma_s = Rgb(m.sigma_s);
    r.bssrdf_eta = m.bssrdf_eta;
    r.bssrdf_index = m.bssrdf_index;
    r.emission = Rgb(m.emission);
    r.alpha.value = m.alpha;
    r.absorption_color = Rgb(m.absorption_color);
    r.absorption_distance = m.absorption_distance;
    r.reflectance.texture = m.reflectance_texture;
    r.alpha.texture = m.alpha_texture;
    r.normal_map = m.normal_map;
    r.normal_scale = m.normal_scale;
    r.measured_index = m.measured_index;
    return r;
}

void PrepareAlias(RefJob& job) {
    yr::RenderSceneIR copy = job.ir;
    yr::PrepareLightSampling(copy);
    job.alias_prob = copy.light_sampling.emissive_power.probability;
    job.alias_index = copy.light_sampling.emissive_power.alias;
    job.alias_pmf = copy.light_sampling.emissive_power.pmf;
}

}  // namespace

extern "C" {

// Returns a job handle, or null with the first error diagnostic in yrref_last_error().
void* yrref_pbrt_load(const char* path) {
    yr::PbrtSceneLoadResult loaded = yr::LoadPbrtScene(path);
    if (!loaded.scene) {
        g_last_error = loaded.diagnostics.empty() ? "PBRT load failed" : loaded.diagnostics.front().message;
        return nullptr;
    }
    yr::SceneCompileResult compiled = yr::CompilePbrtScene(*loaded.scene);
    if (!compiled.scene) {
        g_last_error = compiled.diagnostics.empty() ? "PBRT compile failed" : compiled.diagnostics.front().message;
        return nullptr;
    }
    auto* job = new RefJob();
    job->ir = std::move(*compiled.scene);
    job->settings = compiled.settings;
    PrepareAlias(*job);
    return job;
}

void yrref_job_destroy(void* job) { delete static_cast<RefJob*>(job); }

// counts: vertices, indices, primitives, spheres, instances, materials,
// emissive, analytic, env width, env height, alias count.
void yrref_job_counts(void* handle, std::int64_t* c) {
    const RefJob& j = *static_cast<RefJob*>(handle);
    c[0] = static_cast<std::int64_t>(j.ir.vertices.size());
    c[1] = static_cast<std::int64_t>(j.ir.indices.size());
    c[2] = static_cast<std::int64_t>(j.ir.primitives.size());
    c[3] = static_cast<std::int64_t>(j.ir.spheres.size());
    c[4] = static_cast<std::int64_t>(j.ir.instances.size());
    c[5] = static_cast<std::int64_t>(j.ir.materials.size());
    c[6] = static_cast<std::int64_t>(j.ir.emissive_primitives.size());
    c[7] = static_cast<std::int64_t>(j.ir.analytic_lights.size());
    const yr::RenderEnvironment& env = j.ir.environment;
    const bool tex = env.texture_index >= 0 && static_cast<std::size_t>(env.texture_index) < j.ir.textures.size();
    c[8] = tex ? j.ir.textures[env.texture_index].width : 0;
    c[9] = tex ? j.ir.textures[env.texture_index].height : 0;
    c[10] = static_cast<std::int64_t>(j.alias_pmf.size());
}

// vertices: 12 floats each (position, normal, uv, tangent, handedness).
void yrref_job_geometry(void* handle, float* vertices, std::uint32_t* indices, yrc_primitive* prims,
                        yrc_sphere* spheres, yrc_instance* instances) {
    const RefJob& j = *static_cast<RefJob*>(handle);
    for (std::size_t i = 0; i < j.ir.vertices.size(); ++i) {
        const yr::RenderVertex& v = j.ir.vertices[i];
        const float row[12] = {v.position.x, v.position.y, v.position.z, v.normal.x, v.normal.y, v.normal.z,
                               v.uv.x, v.uv.y, v.tangent.x, v.tangent.y, v.tangent.z, v.tangent_handedness};
        std::copy(row, row + 12, vertices + 12 * i);
    }
    std::copy(j.ir.indices.begin(), j.ir.indices.end(), indices);
    for (std::size_t i = 0; i < j.ir.primitives.size(); ++i) {
        const yr::RenderPrimitive& p = j.ir.primitives[i];
        prims[i] = yrc_primitive{p.first_index, p.index_count, p.material_index,
                                 (p.has_normals ? 1u : 0u) | (p.has_uvs ? 2u : 0u) | (p.has_tangents ? 4u : 0u)};
    }
    for (std::size_t i = 0; i < j.ir.spheres.size(); ++i) {
        const yr::RenderSphere& s = j.ir.spheres[i];
        spheres[i] = yrc_sphere{{s.center.x, s.center.y, s.center.z}, s.radius, s.material_index, s.area_light_index,
                                s.flip_normals ? 1 : 0, 0};
    }
    for (std::size_t i = 0; i < j.ir.instances.size(); ++i) {
        instances[i].primitive = j.ir.instances[i].primitive.Value();
        std::copy(j.ir.instances[i].object_to_world.m.begin(), j.ir.instances[i].object_to_world.m.end(),
                  instances[i].object_to_world);
    }
}

void yrref_job_materials(void* handle, yrc_material* out) {
    const RefJob& j = *static_cast<RefJob*>(handle);
    for (std::size_t i = 0; i < j.ir.materials.size(); ++i) {
        const yr::RenderMaterial& m = j.ir.materials[i];
        yrc_material& o = out[i];
        std::memset(&o, 0, sizeof(o));
        o.kind = static_cast<int32_t>(m.kind);
        CopyRgb(m.reflectance.value, o.reflectance);
        CopyRgb(m.eta.value, o.eta);
        CopyRgb(m.k.value, o.k);
        o.ior = m.ior;
        o.uroughness = m.uroughness.value;
        o.vroughness = m.vroughness.value;
        o.remap_roughness = m.remap_roughness ? 1 : 0;
        o.mix_material_a = m.mix_material_a;
        o.mix_material_b = m.mix_material_b;
        o.mix_amount = m.mix_amount.value;
        o.coating_ior = m.coating_ior;
        o.coating_roughness = m.coating_roughness.value;
        o.coat_thickness = m.coat_thickness;
        CopyRgb(m.coat_absorption, o.coat_absorption);
        o.coat_maxdepth = m.coat_maxdepth;
        o.coat_nsamples = m.coat_nsamples;
        CopyRgb(m.sigma_a, o.sigma_a);
        CopyRgb(m.sigma_s, o.sigma_s);
        o.bssrdf_eta = m.bssrdf_eta;
        o.bssrdf_index = m.bssrdf_index;
        CopyRgb(m.emission, o.emission);
        o.alpha = m.alpha.value;
        CopyRgb(m.absorption_color, o.absorption_color);
        o.absorption_distance = m.absorption_distance;
        o.reflectance_texture = m.reflectance.texture;
        o.alpha_texture = m.alpha.texture;
        o.normal_map = m.normal_map;
        o.measured_index = m.measured_index;
        o.normal_scale = m.normal_scale;
    }
}

// Emissive primitives, the emissive power alias table, camera and settings.
void yrref_job_lights(void* handle, yrc_emissive_primitive* emissive, float* alias_prob, int32_t* alias_index,
                      float* alias_pmf, yrc_camera* camera, yrc_render_settings* settings) {
    const RefJob& j = *static_cast<RefJob*>(handle);
    for (std::size_t i = 0; i < j.ir.emissive_primitives.size(); ++i) {
        const yr::EmissivePrimitive& e = j.ir.emissive_primitives[i];
        emissive[i].primitive_index = e.primitive_index;
        CopyRgb(e.radiance, emissive[i].radiance);
        emissive[i].area = e.area;
    }
    std::copy(j.alias_prob.begin(), j.alias_prob.end(), alias_prob);
    std::copy(j.alias_index.begin(), j.alias_index.end(), alias_index);
    std::copy(j.alias_pmf.begin(), j.alias_pmf.end(), alias_pmf);
    const yr::RenderCamera& c = j.ir.camera;
    *camera = yrc_camera{{c.origin.x, c.origin.y, c.origin.z}, {c.forward.x, c.forward.y, c.forward.z},
                         {c.right.x, c.right.y, c.right.z}, {c.up.x, c.up.y, c.up.z}, c.fov_y_radians};
    const yr::RenderSettings& s = j.settings;
    std::memset(settings, 0, sizeof(*settings));
    settings->width = s.width;
    settings->height = s.height;
    settings->spp = s.spp;
    settings->max_depth = s.max_depth;
    settings->seed = s.seed;
    settings->sampler = static_cast<int32_t>(s.sampler);
    settings->radiance_clamp = s.radiance_clamp;
    settings->adaptive_enabled = s.adaptive_sampling.enabled ? 1 : 0;
    settings->adaptive_min_spp = s.adaptive_sampling.min_spp;
    settings->adaptive_relative_error = s.adaptive_sampling.relative_error;
    settings->adaptive_absolute_error = s.adaptive_sampling.absolute_error;
    settings->adaptive_confidence = s.adaptive_sampling.confidence;
}

// Builds a job from the C-ABI scene description. The environment texture becomes a
// bilinear, repeat-wrapped RGBA texture with its distribution rebuilt by
// BuildEnvironmentDistribution.
void* yrref_job_from_desc(const yrc_scene_desc* d) {
    auto* job = new RefJob();
    yr::RenderSceneIR& ir = job->ir;
    const yrc_geometry& g = d->geometry;
    ir.vertices.resize(static_cast<std::size_t>(g.vertex_count));
    for (std::int64_t v = 0; v < g.vertex_count; ++v) {
        const float* p = reinterpret_cast<const float*>(reinterpret_cast<const char*>(g.positions) + v * g.vertex_stride);
        ir.vertices[v].position = yr::Point3f{p[0], p[1], p[2]};
        if (d->normals) {
            const float* n = reinterpret_cast<const float*>(reinterpret_cast<const char*>(d->normals) + v * d->normal_stride);
            ir.vertices[v].normal = yr::Vec3f{n[0], n[1], n[2]};
        }
        if (d->uvs) {
            const float* t = reinterpret_cast<const float*>(reinterpret_cast<const char*>(d->uvs) + v * d->uv_stride);
            ir.vertices[v].uv = yr::Vec2f{t[0], t[1]};
        }
        if (d->tangents) {
            const float* t =
                reinterpret_cast<const float*>(reinterpret_cast<const char*>(d->tangents) + v * d->tangent_stride);
            ir.vertices[v].tangent = yr::Vec3f{t[0], t[1], t[2]};
            ir.vertices[v].tangent_handedness = t[3];
        }
    }
    ir.indices.assign(g.indices, g.indices + g.index_count);
    for (int32_t p = 0; p < g.primitive_count; ++p) {
        const yrc_primitive& s = g.primitives[p];
        ir.primitives.push_back(yr::RenderPrimitive{s.first_index, s.index_count, s.material_index,
                                                    (s.flags & 1u) != 0, (s.flags & 2u) != 0, (s.flags & 4u) != 0});
    }
    for (int32_t i = 0; i < g.sphere_count; ++i) {
        const yrc_sphere& s = g.spheres[i];
        ir.spheres.push_back(yr::RenderSphere{yr::Point3f{s.center[0], s.center[1], s.center[2]}, s.radius,
                                              s.material_index, s.area_light_index, s.flip_normals != 0});
    }
    for (int32_t i = 0; i < g.instance_count; ++i) {
        yr::RenderInstance inst;
        inst.primitive = yr::MeshPrimitiveHandle{g.instances[i].primitive};
        std::copy(g.instances[i].object_to_world, g.instances[i].object_to_world + 16, inst.object_to_world.m.begin());
        ir.instances.push_back(inst);
    }
    for (int32_t i = 0; i < d->material_count; ++i) ir.materials.push_back(MaterialFrom(d->materials[i]));
    for (int32_t i = 0; d->measured && i < d->measured_count; ++i) ir.measured_brdfs.push_back(MakeMeasured(d->measured[i]));
    // Scene textures keep their indices; the environment texture follows them.
    for (int32_t i = 0; d->textures && i < d->texture_count; ++i) {
        const yrc_texture& t = d->textures[i];
        yr::RenderTexture tex = MakeTexture(t.width, t.height, t.texels, t.filter, t.wrap_s, t.wrap_t);
        ir.textures.push_back(std::move(tex));
    }
    for (int32_t i = 0; i < d->emissive_count; ++i) {
        const yrc_emissive_primitive& e = d->emissive[i];
        ir.emissive_primitives.push_back(yr::EmissivePrimitive{e.primitive_index, Rgb(e.radiance), e.area});
    }
    for (int32_t i = 0; d->analytic && i < d->analytic_count; ++i) {
        const yrc_analytic_light& a = d->analytic[i];
        yr::AnalyticLight l;
        l.kind = static_cast<yr::AnalyticLightKind>(a.kind);
        l.position = yr::Point3f{a.position[0], a.position[1], a.position[2]};
        l.direction = yr::Vec3f{a.direction[0], a.direction[1], a.direction[2]};
        l.intensity = Rgb(a.intensity);
        l.cone_angle = a.cone_angle;
        l.cone_cos_inner = a.cone_cos_inner;
        ir.analytic_lights.push_back(l);
    }
    const yrc_environment& env = d->environment;
    for (int32_t i = 0; d->bssrdf_tables && i < d->bssrdf_count; ++i) {
        const yrc_bssrdf_table& t = d->bssrdf_tables[i];
        auto table = std::make_shared<yr::BSSRDFTable>(t.rho_count, t.radius_count);
        const std::size_t cells = static_cast<std::size_t>(t.rho_count) * t.radius_count;
        std::copy(t.rho_samples, t.rho_samples + t.rho_count, table->rho_samples.begin());
        std::copy(t.radius_samples, t.radius_samples + t.radius_count, table->radius_samples.begin());
        std::copy(t.profile, t.profile + cells, table->profile.begin());
        std::copy(t.rho_eff, t.rho_eff + t.rho_count, table->rho_eff.begin());
        std::copy(t.profile_cdf, t.profile_cdf + cells, table->profile_cdf.begin());
        ir.bssrdf_tables.push_back(std::move(table));
    }
    ir.environment.active = env.active != 0;
    ir.environment.radiance = Rgb(env.radiance);
    ir.environment.strength = env.strength;
    ir.environment.rotation_radians = env.rotation_radians;
    if (env.active && env.texels && env.width > 0 && env.height > 0) {
        yr::RenderTexture tex;
        tex.width = env.width;
        tex.height = env.height;
        tex.texels.resize(static_cast<std::size_t>(env.width) * env.height);
        for (std::size_t i = 0; i < tex.texels.size(); ++i) {
            tex.texels[i] = yr::Color4f{env.texels[4 * i], env.texels[4 * i + 1], env.texels[4 * i + 2], env.texels[4 * i + 3]};
        }
        ir.environment_distributions.push_back(yr::BuildEnvironmentDistribution(tex));
        ir.environment.texture_index = static_cast<int>(ir.textures.size());
        ir.environment.distribution_index = 0;
        ir.textures.push_back(std::move(tex));
    }
    const yrc_camera& c = d->camera;
    ir.camera.origin = yr::Point3f{c.origin[0], c.origin[1], c.origin[2]};
    ir.camera.forward = yr::Vec3f{c.forward[0], c.forward[1], c.forward[2]};
    ir.camera.right = yr::Vec3f{c.right[0], c.right[1], c.right[2]};
    ir.camera.up = yr::Vec3f{c.up[0], c.up[1], c.up[2]};
    ir.camera.fov_y_radians = c.fov_y_radians;
    const yrc_render_settings& s = d->settings;
    job->settings.integrator = yr::RenderIntegratorKind::Path;
    job->settings.sampler = static_cast<yr::RenderSamplerKind>(s.sampler);
    job->settings.width = s.width;
    job->settings.height = s.height;
    job->settings.spp = s.spp;
    job->settings.max_depth = s.max_depth;
    job->settings.seed = s.seed;
    job->settings.radiance_clamp = s.radiance_clamp;
    job->settings.adaptive_sampling.enabled = s.adaptive_enabled != 0;
    job->settings.adaptive_sampling.min_spp = s.adaptive_min_spp;
    job->settings.adaptive_sampling.relative_error = s.adaptive_relative_error;
    job->settings.adaptive_sampling.absolute_error = s.adaptive_absolute_error;
    job->settings.adaptive_sampling.confidence = s.adaptive_confidence;
    PrepareAlias(*job);
    return job;
}

namespace {

int RenderJobImpl(const RefJob& j, int threads, int spp_override, const void* resume_film, int resume_spp,
                  void* film_out, std::uint64_t* stats, int stat_count, double* seconds) {
    yr::RenderJob job{j.ir, j.settings};
    job.settings.requested_backend = yr::RenderBackendKind::Cpu;
    job.settings.threads = threads;
    if (spp_override > 0) job.settings.spp = spp_override;
    const int width = job.settings.width, height = job.settings.height;
    yr::CpuBackend backend;
    yr::BackendPrepareResult prepared = backend.Prepare(std::move(job));
    if (!prepared.ok) {
        g_last_error = prepared.error;
        return 1;
    }
    yr::RenderRequest request;
    std::unique_ptr<yr::Film> resume;
    if (resume_film) {
        resume = std::make_unique<yr::Film>(width, height);
        const auto* px = static_cast<const yr::FilmPixel*>(resume_film);
        for (int y = 0; y < height; ++y) {
            for (int x = 0; x < width; ++x) resume->SetPixelForCheckpoint(x, y, px[y * width + x]);
        }
        request.resume_film = resume.get();
        request.resume_completed_spp = resume_spp;
    }
    yr::RenderResult result = backend.Render(*prepared.scene, request);
    if (!result.ok || !result.film) {
        g_last_error = result.error;
        return 2;
    }
    std::memcpy(film_out, result.film->Pixels().data(), result.film->Pixels().size() * sizeof(yr::FilmPixel));
    if (stats) {
        const std::uint64_t all[8] = {result.stats.samples_rendered, result.stats.rays_traced,
                                      result.stats.shadow_rays,      result.stats.occluded_shadow_rays,
                                      result.stats.hits,             result.stats.misses,
                                      result.film->BadSampleCount(), result.stats.converged_pixels};
        for (int k = 0; k < stat_count; ++k) stats[k] = all[k];
    }
    if (seconds) *seconds = result.stats.elapsed_seconds;
    return 0;
}

}  // namespace

// Renders the job with the reference CPU backend. film_out: width*height
// FilmPixel (56 bytes each). stats: samples, rays_traced, shadow_rays,
// occluded, hits, misses, bad samples (7 uint64). Returns 0 on success.
int yrref_job_render(void* handle, int threads, int spp_override, void* film_out, std::uint64_t* stats,
                     double* seconds) {
    return RenderJobImpl(*static_cast<RefJob*>(handle), threads, spp_override, nullptr, 0, film_out, stats, 7,
                         seconds);
}

// The same render resumed from `resume_film` (width*height FilmPixel, no bad
// samples) after `resume_spp` completed passes, as RenderRequest's
// resume_film / resume_completed_spp do; stats gets an eighth entry, the
// converged pixels of the last pass (RenderStats::converged_pixels).
int yrref_job_render_resume(void* handle, int threads, int spp_override, const void* resume_film, int resume_spp,
                            void* film_out, std::uint64_t* stats, double* seconds) {
    return RenderJobImpl(*static_cast<RefJob*>(handle), threads, spp_override, resume_film, resume_spp, film_out,
                         stats, 8, seconds);
}

// TraceShadowVisibility (src/integrators/path_direct_lighting.cpp:23-113) on
// the job's scene, prepared as the CPU backend prepares it, for n rays of 8
// floats (origin, unused, direction, max_distance): out rows of 4 floats
// (transmittance RGB, visible 0/1). Returns 0, or 1 on a build error.
int yrref_job_shadow_visibility(void* handle, const float* rays, std::int64_t n, float* out) {
    const RefJob& j = *static_cast<RefJob*>(handle);
    yr::RenderSceneIR ir = j.ir;
    yr::BuildTextureSamplingCaches(ir.textures);
    yr::PrepareLightSampling(ir);
    yr::RenderAccelerationBuildResult build = yr::BuildRenderAcceleration(ir.Geometry());
    if (!build.errors.empty()) {
        g_last_error = build.errors.front();
        return 1;
    }
    for (std::int64_t i = 0; i < n; ++i) {
        const float* r = rays + 8 * i;
        yr::PathTraceStats stats;
        const yr::ShadowVisibility v = yr::TraceShadowVisibility(
            ir, build.acceleration, yr::Ray3f{yr::Point3f{r[0], r[1], r[2]}, yr::Vec3f{r[4], r[5], r[6]}}, r[7], stats);
        CopyRgb(v.transmittance, out + 4 * i);
        out[4 * i + 3] = v.visible ? 1.0f : 0.0f;
    }
    return 0;
}

// EvaluateBsdf then PdfBsdf with Rng(seeds[i]) for rows of (wo, wi, normal).
void yrref_bsdf_eval(const yrc_material* material, const float* q, const std::uint64_t* seeds, std::int64_t n,
                     float* f, float* pdf) {
    const yr::RenderMaterial m = MaterialFrom(*material);
    for (std::int64_t i = 0; i < n; ++i) {
        const float* r = q + 9 * i;
        const yr::Vec3f wo{r[0], r[1], r[2]}, wi{r[3], r[4], r[5]}, nn{r[6], r[7], r[8]};
        yr::Rng rng{seeds[i]};
        CopyRgb(yr::EvaluateBsdf(m, wo, wi, nn, rng), f + 3 * i);
        pdf[i] = yr::PdfBsdf(m, wo, wi, nn, rng);
    }
}

// SampleBsdf with Rng(seeds[i]) for rows of (wo, normal, u): out rows (wi,
// weight, pdf, valid, specular).
void yrref_bsdf_sample(const yrc_material* material, const float* q, const std::uint64_t* seeds, std::int64_t n,
                       float* out) {
    const yr::RenderMaterial m = MaterialFrom(*material);
    for (std::int64_t i = 0; i < n; ++i) {
        const float* r = q + 8 * i;
        yr::Rng rng{seeds[i]};
        const yr::BsdfSample s =
            yr::SampleBsdf(m, yr::Vec3f{r[0], r[1], r[2]}, yr::Vec3f{r[3], r[4], r[5]}, yr::Vec2f{r[6], r[7]}, rng);
        float* o = out + 9 * i;
        o[0] = s.wi.x;
        o[1] = s.wi.y;
        o[2] = s.wi.z;
        CopyRgb(s.weight, o + 3);
        o[6] = s.pdf;
        o[7] = s.valid ? 1.0f : 0.0f;
        o[8] = s.specular ? 1.0f : 0.0f;
    }
}

// ComputeBeamDiffusionBSSRDF of the reference, for checking the product's
// table builder.
void yrref_bssrdf_table(float g, float eta, int rho_count, int radius_count, float* rho, float* radius,
                        float* profile, float* rho_eff, float* cdf) {
    yr::BSSRDFTable t(rho_count, radius_count);
    yr::ComputeBeamDiffusionBSSRDF(g, eta, t);
    std::copy(t.rho_samples.begin(), t.rho_samples.end(), rho);
    std::copy(t.radius_samples.begin(), t.radius_samples.end(), radius);
    std::copy(t.profile.begin(), t.profile.end(), profile);
    std::copy(t.rho_eff.begin(), t.rho_eff.end(), rho_eff);
    std::copy(t.profile_cdf.begin(), t.profile_cdf.end(), cdf);
}

// The reference's TabulatedBSSRDF evaluated at n points (for checking the
// device restatement): sample_r[i] = Sample_Sr(ch[i], u[i]),
// pdf[i] = Pdf_Sr(ch[i], r[i]), sr[3 i..] = Sr(r[i]).
void yrref_bssrdf_eval(const float* sigma_a, const float* sigma_s, float eta, float g, int n, const int* ch,
                       const float* u, const float* r, float* sample_r, float* pdf, float* sr) {
    yr::BSSRDFTable t(100, 64);
    yr::ComputeBeamDiffusionBSSRDF(g, eta, t);
    const yr::TabulatedBSSRDF b(yr::Color3f{sigma_a[0], sigma_a[1], sigma_a[2]},
                                yr::Color3f{sigma_s[0], sigma_s[1], sigma_s[2]}, eta, t);
    for (int i = 0; i < n; ++i) {
        sample_r[i] = b.Sample_Sr(ch[i], u[i]);
        pdf[i] = b.Pdf_Sr(ch[i], r[i]);
        const yr::Color3f c = b.Sr(r[i]);
        sr[3 * i] = c.x;
        sr[3 * i + 1] = c.y;
        sr[3 * i + 2] = c.z;
    }
}

// TabulatedBSSRDF::Pdf_Sp for rows of (po, ss, ts, ns, pi, ni).
void yrref_bssrdf_pdf_sp(const float* sigma_a, const float* sigma_s, float eta, float g, int n, const float* q,
                         float* pdf) {
    yr::BSSRDFTable t(100, 64);
    yr::ComputeBeamDiffusionBSSRDF(g, eta, t);
    const yr::TabulatedBSSRDF b(yr::Color3f{sigma_a[0], sigma_a[1], sigma_a[2]},
                                yr::Color3f{sigma_s[0], sigma_s[1], sigma_s[2]}, eta, t);
    for (int i = 0; i < n; ++i) {
        const float* p = q + 18 * i;
        pdf[i] = b.Pdf_Sp(yr::Point3f{p[0], p[1], p[2]}, yr::Vec3f{p[3], p[4], p[5]}, yr::Vec3f{p[6], p[7], p[8]},
                          yr::Vec3f{p[9], p[10], p[11]}, yr::Point3f{p[12], p[13], p[14]},
                          yr::Vec3f{p[15], p[16], p[17]});
    }
}

}  // extern "C"
