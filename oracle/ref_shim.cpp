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
