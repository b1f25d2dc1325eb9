// yr::CudaBackend over libyrcuda — the file a YaoRay maintainer drops in
// place of src/runtime/cuda_stub_backend.cpp (and cuda_stub_prepared_scene.cpp)
// to make `yaoray render scene.pbrt --backend cuda` run on a B200.
//
// It keeps the reference's contracts: Prepare() takes the RenderJob by value,
// builds the light-sampling tables and the SAH acceleration structure with the
// reference's own host builders (PrepareLightSampling, BuildRenderAcceleration),
// and uploads the scene through yrc_render_scene_create; Render() runs the
// pass loop on the device with the RenderRequest's resume film, stop token and
// per-pass progress callback, and returns a yr::Film and RenderStats.
// Only the C ABI (include/yrcuda.h) crosses into the CUDA library.
#include <yaoray/shading/measured_brdf.hpp>
#include <yaoray/accel/acceleration.hpp>
#include <yaoray/lighting/light_sampling.hpp>
#include <yaoray/runtime/cuda_stub_backend.hpp>

#include "yrcuda.h"

#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <stop_token>
#include <string>
#include <vector>

namespace yr {
namespace {

// Prepared scene: owns the RenderJob, the reference's acceleration structure
// (kept alive for the device upload's lifetime), and the device scene handle.
class DeviceScene final : public PreparedScene {
public:
    DeviceScene(RenderJob job, RenderAcceleration accel, yrc_render_scene* handle)
        : job_(std::move(job)), accel_(std::move(accel)), handle_(handle) {}
    ~DeviceScene() override { yrc_render_scene_destroy(handle_); }

    RenderBackendKind Kind() const override { return RenderBackendKind::Cuda; }
    const RenderSceneIR& SourceScene() const override { return job_.scene; }
    const RenderSettings& Settings() const override { return job_.settings; }
    yrc_render_scene* Handle() const { return handle_; }
    const RenderAcceleration& Acceleration() const { return accel_; }

private:
    RenderJob job_;
    RenderAcceleration accel_;
    yrc_render_scene* handle_;
};

void Rgb(const Color3f& c, float* out) {
    out[0] = c.x;
    out[1] = c.y;
    out[2] = c.z;
}

yrc_bvh_view View(const RenderBvh& bvh, std::vector<yrc_bvh_primitive>& prims) {
    prims.resize(bvh.primitives.size());
    for (std::size_t i = 0; i < bvh.primitives.size(); ++i) {
        const RenderBvhPrimitive& p = bvh.primitives[i];
        prims[i] = yrc_bvh_primitive{p.kind == BvhPrimitiveKind::Triangle ? 0 : 1, p.mesh_primitive.Value(),
                                     p.sphere.Value(), p.local_triangle, p.flat_triangle_index};
    }
    static_assert(sizeof(RenderBvhNode) == sizeof(yrc_bvh_node), "node layouts must match");
    yrc_bvh_view v{};
    v.nodes = reinterpret_cast<const yrc_bvh_node*>(bvh.nodes.data());
    v.node_count = static_cast<int64_t>(bvh.nodes.size());
    v.primitive_indices = bvh.primitive_indices.data();
    v.primitive_index_count = static_cast<int64_t>(bvh.primitive_indices.size());
    v.primitives = prims.data();
    v.primitive_count = static_cast<int64_t>(prims.size());
    v.max_depth = bvh.max_depth;
    return v;
}

Film ToFilm(const std::vector<yrc_film_pixel>& pixels, std::uint64_t bad, int width, int height) {
    static_assert(sizeof(FilmPixel) == sizeof(yrc_film_pixel), "film pixel layouts must match");
    Film film(width, height);
    for (int y = 0; y < height; ++y) {
        for (int x = 0; x < width; ++x) {
            FilmPixel p;
            std::memcpy(&p, &pixels[static_cast<std::size_t>(y) * width + x], sizeof(p));
            film.SetPixelForCheckpoint(x, y, p);
        }
    }
    // Film exposes no setter for the dropped-sample counter; non-finite
    // samples increment it without touching any pixel.
    const float nan = std::numeric_limits<float>::quiet_NaN();
    for (std::uint64_t i = 0; i < bad; ++i) film.AddSample(0, 0, Color3f{nan, nan, nan});
    return film;
}

struct ProgressBridge {
    const RenderRequest* request;
    int width, height;
    std::vector<yrc_film_pixel> scratch;
};

int32_t ProgressThunk(const yrc_render_progress* p, const yrc_film_pixel* film, uint64_t bad, void* user,
                      char* error, size_t capacity) {
    auto* bridge = static_cast<ProgressBridge*>(user);
    const std::size_t n = static_cast<std::size_t>(bridge->width) * bridge->height;
    bridge->scratch.assign(film, film + n);
    const Film f = ToFilm(bridge->scratch, bad, bridge->width, bridge->height);
    const RenderProgress progress{p->completed_spp, p->target_spp, p->completed_samples, p->target_samples,
                                  p->active_pixels, p->converged_pixels, p->rays_traced, p->elapsed_seconds};
    const RenderProgressDecision decision = bridge->request->progress_callback(progress, f);
    if (!decision.cancel) return 0;
    if (!decision.error.empty() && capacity > 0) {
        const std::size_t len = std::min(capacity - 1, decision.error.size());
        std::memcpy(error, decision.error.data(), len);
        error[len] = '\0';
    }
    return 1;
}

}  // namespace

RenderBackendKind CudaBackend::Kind() const { return RenderBackendKind::Cuda; }

RenderBackendCapabilities CudaBackend::Capabilities() const {
    return RenderBackendCapabilities{RenderBackendKind::Cuda, yrc_device_available() != 0, false, true, true, false};
}

BackendPrepareResult CudaBackend::Prepare(RenderJob job) {
    BackendPrepareResult result;
    if (job.settings.requested_backend != RenderBackendKind::Cuda) {
        result.error = "CUDA backend cannot prepare a scene requested for " +
                       std::string{RenderBackendName(job.settings.requested_backend)};
        return result;
    }
    if (job.settings.integrator != RenderIntegratorKind::Path) {
        result.error = "CUDA backend renders the path integrator only";
        return result;
    }
    const auto start = std::chrono::steady_clock::now();
    RenderSceneIR& ir = job.scene;
    PrepareLightSampling(ir);
    const auto accel_start = std::chrono::steady_clock::now();
    BvhBuildOptions options;
    options.thread_count = job.settings.threads;
    RenderAccelerationBuildResult built = BuildRenderAcceleration(ir.Geometry(), options);
    if (!built.errors.empty()) {
        result.error = built.errors.front();
        return result;
    }
    result.acceleration_build_seconds =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - accel_start).count();

    // Marshal the IR into the C-ABI scene description.
    yrc_scene_desc d{};
    yrc_geometry& g = d.geometry;
    static_assert(sizeof(RenderVertex) == 48, "RenderVertex stride");
    g.positions = ir.vertices.empty() ? nullptr : &ir.vertices[0].position.x;
    g.vertex_count = static_cast<int64_t>(ir.vertices.size());
    g.vertex_stride = sizeof(RenderVertex);
    d.normals = ir.vertices.empty() ? nullptr : &ir.vertices[0].normal.x;
    d.normal_stride = sizeof(RenderVertex);
    g.indices = ir.indices.data();
    g.index_count = static_cast<int64_t>(ir.indices.size());
    std::vector<yrc_primitive> prims;
    for (const RenderPrimitive& p : ir.primitives) {
        prims.push_back(yrc_primitive{p.first_index, p.index_count, p.material_index,
                                      (p.has_normals ? 1u : 0u) | (p.has_uvs ? 2u : 0u) | (p.has_tangents ? 4u : 0u)});
    }
    g.primitives = prims.data();
    g.primitive_count = static_cast<int32_t>(prims.size());
    std::vector<yrc_sphere> spheres;
    for (const RenderSphere& s : ir.spheres) {
        spheres.push_back(yrc_sphere{{s.center.x, s.center.y, s.center.z}, s.radius, s.material_index,
                                     s.area_light_index, s.flip_normals ? 1 : 0, 0});
    }
    g.spheres = spheres.data();
    g.sphere_count = static_cast<int32_t>(spheres.size());
    std::vector<yrc_material> materials(ir.materials.size());
    for (std::size_t i = 0; i < ir.materials.size(); ++i) {
        const RenderMaterial& m = ir.materials[i];
        yrc_material& o = materials[i];
        o.kind = static_cast<int32_t>(m.kind);
        Rgb(m.reflectance.value, o.reflectance);
        Rgb(m.eta.value, o.eta);
        Rgb(m.k.value, o.k);
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
        Rgb(m.coat_absorption, o.coat_absorption);
        o.coat_maxdepth = m.coat_maxdepth;
        o.coat_nsamples = m.coat_nsamples;
        Rgb(m.sigma_a, o.sigma_a);
        Rgb(m.sigma_s, o.sigma_s);
        o.bssrdf_eta = m.bssrdf_eta;
        o.bssrdf_index = m.bssrdf_index;
        Rgb(m.emission, o.emission);
        o.alpha = m.alpha.value;
        Rgb(m.absorption_color, o.absorption_color);
        o.absorption_distance = m.absorption_distance;
        o.reflectance_texture = m.reflectance.texture;
        o.alpha_texture = m.alpha.texture;
        o.normal_map = m.normal_map;
        o.measured_index = m.measured_index;
        o.normal_scale = m.normal_scale;
    }
    // Vertex uvs and tangents, and every texture of the IR by index (the
    // device builds the mip chains).
    d.uvs = ir.vertices.empty() ? nullptr : &ir.vertices[0].uv.x;
    d.uv_stride = sizeof(RenderVertex);
    d.tangents = ir.vertices.empty() ? nullptr : &ir.vertices[0].tangent.x;
    d.tangent_stride = sizeof(RenderVertex);
    std::vector<yrc_texture> textures;
    for (const RenderTexture& t : ir.textures) {
        const std::vector<Color4f>& texels = t.sampling_cache ? t.sampling_cache->texels : t.texels;
        textures.push_back(yrc_texture{t.width, t.height, texels.empty() ? nullptr : &texels[0].x,
                                       static_cast<int32_t>(t.filter), static_cast<int32_t>(t.wrap_s),
                                       static_cast<int32_t>(t.wrap_t), 0});
    }
    d.textures = textures.data();
    d.texture_count = static_cast<int32_t>(textures.size());
    // Measured BRDFs: the raw RGL tensors (the library builds the warps).
    std::vector<yrc_measured_brdf> measured;
    for (const std::shared_ptr<MeasuredBrdf>& mb : ir.measured_brdfs) {
        const MeasuredBrdf& m = *mb;
        measured.push_back(yrc_measured_brdf{
            static_cast<int32_t>(m.theta_i.size()), static_cast<int32_t>(m.phi_i.size()),
            static_cast<int32_t>(m.wavelengths.size()), static_cast<int32_t>(m.ndf_shape[0]),
            static_cast<int32_t>(m.ndf_shape[1]), static_cast<int32_t>(m.vndf_shape[2]),
            static_cast<int32_t>(m.vndf_shape[3]), m.res, m.theta_i.data(), m.phi_i.data(), m.wavelengths.data(),
            m.ndf.data(), m.sigma.data(), m.vndf.data(), m.luminance.data(), m.spectra.data()});
    }
    d.measured = measured.data();
    d.measured_count = static_cast<int32_t>(measured.size());
    d.materials = materials.data();
    d.material_count = static_cast<int32_t>(materials.size());
    std::vector<yrc_emissive_primitive> emissive;
    for (const EmissivePrimitive& e : ir.emissive_primitives) {
        emissive.push_back(yrc_emissive_primitive{e.primitive_index, {e.radiance.x, e.radiance.y, e.radiance.z}, e.area});
    }
    d.emissive = emissive.data();
    d.emissive_count = static_cast<int32_t>(emissive.size());
    const AliasTable& at = ir.light_sampling.emissive_power;
    d.emissive_power = yrc_alias_table{at.probability.data(), at.alias.data(), at.pmf.data(),
                                       static_cast<int32_t>(at.pmf.size())};
    std::vector<yrc_analytic_light> analytic;
    for (const AnalyticLight& l : ir.analytic_lights) {
        yrc_analytic_light a{};
        a.kind = static_cast<int32_t>(l.kind);
        Rgb(l.position, a.position);
        Rgb(l.direction, a.direction);
        Rgb(l.intensity, a.intensity);
        a.cone_angle = l.cone_angle;
        a.cone_cos_inner = l.cone_cos_inner;
        analytic.push_back(a);
    }
    d.analytic = analytic.data();
    d.analytic_count = static_cast<int32_t>(analytic.size());
    // Environment: texels and the prepared distribution.
    const RenderEnvironment& env = ir.environment;
    d.environment.active = env.active ? 1 : 0;
    Rgb(env.radiance, d.environment.radiance);
    d.environment.strength = env.strength;
    d.environment.rotation_radians = env.rotation_radians;
    std::vector<float> texels;
    if (env.active && env.texture_index >= 0 && static_cast<std::size_t>(env.texture_index) < ir.textures.size()) {
        const RenderTexture& t = ir.textures[static_cast<std::size_t>(env.texture_index)];
        texels.resize(t.texels.size() * 4);
        for (std::size_t i = 0; i < t.texels.size(); ++i) {
            texels[4 * i] = t.texels[i].x;
            texels[4 * i + 1] = t.texels[i].y;
            texels[4 * i + 2] = t.texels[i].z;
            texels[4 * i + 3] = t.texels[i].w;
        }
        d.environment.width = t.width;
        d.environment.height = t.height;
        d.environment.texels = texels.data();
        if (env.distribution_index >= 0 &&
            static_cast<std::size_t>(env.distribution_index) < ir.environment_distributions.size()) {
            const RenderEnvironmentDistribution& dist = ir.environment_distributions[env.distribution_index];
            d.environment.texel_weights = dist.texel_weights.data();
            d.environment.row_weights = dist.row_weights.data();
            d.environment.row_cdf = dist.row_cdf.data();
            d.environment.conditional_cdfs = dist.conditional_cdfs.data();
            d.environment.total_weight = dist.total_weight;
        }
    }
    const RenderCamera& c = ir.camera;
    d.camera = yrc_camera{{c.origin.x, c.origin.y, c.origin.z}, {c.forward.x, c.forward.y, c.forward.z},
                          {c.right.x, c.right.y, c.right.z}, {c.up.x, c.up.y, c.up.z}, c.fov_y_radians};
    const RenderSettings& s = job.settings;
    d.settings = yrc_render_settings{s.width, s.height, s.spp, s.max_depth, s.seed, static_cast<int32_t>(s.sampler),
                                     s.radiance_clamp, s.adaptive_sampling.enabled ? 1 : 0,
                                     s.adaptive_sampling.min_spp, s.adaptive_sampling.relative_error,
                                     s.adaptive_sampling.absolute_error, s.adaptive_sampling.confidence};
    // Acceleration structure: the reference builder's own arrays.
    const RenderAcceleration& accel = built.acceleration;
    std::vector<yrc_bvh_primitive> flat_prims;
    yrc_bvh_view flat_view{};
    std::vector<std::vector<yrc_bvh_primitive>> blas_prims;
    std::vector<yrc_blas_view> blases;
    std::vector<yrc_prepared_instance> instances;
    std::vector<yrc_tlas_primitive> tlas_prims;
    yrc_two_level_view tl{};
    if (accel.kind == RenderAccelerationKind::FlatReference) {
        flat_view = View(accel.flat, flat_prims);
        d.flat = &flat_view;
    } else {
        const TwoLevelBvh& t = accel.two_level;
        blas_prims.resize(t.blases.size());
        for (std::size_t b = 0; b < t.blases.size(); ++b) {
            yrc_blas_view v{};
            v.mesh_primitive = t.blases[b].primitive.Value();
            Rgb(t.blases[b].object_bounds.min, v.object_bounds_min);
            Rgb(t.blases[b].object_bounds.max, v.object_bounds_max);
            v.bvh = View(t.blases[b].bvh, blas_prims[b]);
            blases.push_back(v);
        }
        for (const PreparedMeshInstance& in : t.instances) {
            yrc_prepared_instance o{};
            o.primitive = in.primitive.Value();
            o.blas_index = in.blas_index;
            std::memcpy(o.object_to_world, in.object_to_world.m.data(), sizeof(o.object_to_world));
            std::memcpy(o.world_to_object, in.world_to_object.m.data(), sizeof(o.world_to_object));
            Rgb(in.world_bounds.min, o.world_bounds_min);
            Rgb(in.world_bounds.max, o.world_bounds_max);
            instances.push_back(o);
        }
        for (const RenderTlasPrimitive& p : t.tlas.primitives) {
            yrc_tlas_primitive o{};
            o.kind = p.kind == TlasPrimitiveKind::Instance ? 0 : 1;
            o.instance = p.instance.Value();
            o.sphere = p.sphere.Value();
            Rgb(p.world_bounds.min, o.world_bounds_min);
            Rgb(p.world_bounds.max, o.world_bounds_max);
            tlas_prims.push_back(o);
        }
        tl.blases = blases.data();
        tl.blas_count = static_cast<int32_t>(blases.size());
        tl.instances = instances.data();
        tl.instance_count = static_cast<int32_t>(instances.size());
        tl.tlas_nodes = reinterpret_cast<const yrc_bvh_node*>(t.tlas.nodes.data());
        tl.tlas_node_count = static_cast<int64_t>(t.tlas.nodes.size());
        tl.tlas_primitive_indices = t.tlas.primitive_indices.data();
        tl.tlas_primitive_index_count = static_cast<int64_t>(t.tlas.primitive_indices.size());
        tl.tlas_primitives = tlas_prims.data();
        tl.tlas_primitive_count = static_cast<int64_t>(tlas_prims.size());
        tl.tlas_max_depth = t.tlas.max_depth;
        d.two_level = &tl;
    }
    yrc_render_scene* handle = nullptr;
    if (yrc_render_scene_create(&d, &handle) != YRC_OK) {
        result.error = yrc_last_error();
        return result;
    }
    result.ok = true;
    result.scene = std::make_unique<DeviceScene>(std::move(job), std::move(built.acceleration), handle);
    result.elapsed_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    return result;
}

RenderResult CudaBackend::Render(const PreparedScene& scene, const RenderRequest& request) {
    RenderResult result;
    const auto* device = dynamic_cast<const DeviceScene*>(&scene);
    if (scene.Kind() != RenderBackendKind::Cuda || device == nullptr) {
        result.error = "CUDA backend received a non-CUDA prepared scene.";
        return result;
    }
    const RenderSettings& s = scene.Settings();
    std::vector<yrc_film_pixel> resume;
    yrc_render_request r{};
    if (request.resume_film != nullptr) {
        if (request.resume_film->Width() != s.width || request.resume_film->Height() != s.height) {
            result.error = "resume film dimensions do not match render scene";
            return result;
        }
        const auto& px = request.resume_film->Pixels();
        resume.resize(px.size());
        std::memcpy(resume.data(), px.data(), px.size() * sizeof(yrc_film_pixel));
        r.resume_film = resume.data();
        r.resume_bad_samples = request.resume_film->BadSampleCount();
    }
    r.resume_completed_spp = request.resume_completed_spp;
    // The stop token is observed between passes through the stop flag.
    std::atomic<int32_t> stop_flag{request.stop_token.stop_requested() ? 1 : 0};
    std::stop_callback on_stop(request.stop_token, [&] { stop_flag.store(1); });
    r.stop_flag = reinterpret_cast<const volatile int32_t*>(&stop_flag);
    ProgressBridge bridge{&request, s.width, s.height, {}};
    if (request.progress_callback) {
        r.progress = &ProgressThunk;
        r.user = &bridge;
    }
    std::vector<yrc_film_pixel> film(static_cast<std::size_t>(s.width) * s.height);
    uint64_t bad = 0;
    yrc_render_stats st{};
    const yrc_status status = yrc_render(device->Handle(), &r, film.data(), &bad, &st);
    if (status != YRC_OK) {
        result.error = yrc_last_error();
        return result;
    }
    result.ok = true;
    result.film.emplace(ToFilm(film, bad, s.width, s.height));
    result.stats.samples_rendered = st.samples_rendered;
    result.stats.converged_pixels = st.converged_pixels;
    result.stats.rays_traced = st.rays_traced;
    result.stats.shadow_rays = st.shadow_rays;
    result.stats.occluded_shadow_rays = st.occluded_shadow_rays;
    result.stats.triangle_tests = st.triangle_tests;
    result.stats.sphere_tests = st.sphere_tests;
    result.stats.bvh_node_tests = st.bvh_node_tests;
    result.stats.bvh_nodes = device->Acceleration().NodeCount();
    result.stats.bvh_max_depth = device->Acceleration().MaxDepth();
    result.stats.hits = st.hits;
    result.stats.misses = st.misses;
    result.stats.threads = 1;
    result.stats.elapsed_seconds = st.elapsed_seconds;
    return result;
}

}  // namespace yr
