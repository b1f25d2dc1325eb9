// Render scene upload and the device pass loop behind yrc_render_scene_create
// / yrc_render — the CUDA backend's Prepare and Render.
//
// Pass semantics follow RenderCpuPathTrace (src/backends/cpu/cpu_path_tracer.cpp:
// 39-229): every active pixel takes one sample attempt per pass, its sample
// index is the film's current sample count, a non-finite sample is dropped
// and counted, and (with adaptive sampling) converged pixels stop. To fill
// the GPU, one batch renders several consecutive passes at once: pixel p's
// j-th path uses sample index count(p) + j, and the film kernel accepts them
// in order, stopping at the first non-finite sample (whose index the next
// batch re-uses, as the reference's next pass would) or at convergence.
// With a progress callback the batch is one pass, so the callback sees the
// film after every pass exactly as the reference's does.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <vector>

#include "nrc.hpp"
#include "render_kernels.hpp"
#include "render_types.hpp"
#include "measured.hpp"
#include "texture.hpp"
#include "trace_kernels.hpp"
#include "yrc_internal.hpp"

namespace yrc {
namespace {

yrc_status CudaError(cudaError_t err, const char* what) {
    return Fail(err == cudaErrorMemoryAllocation ? YRC_ERR_OUT_OF_MEMORY : YRC_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(err));
}

// Device allocation bookkeeping for one render scene.
struct DeviceArena {
    std::vector<void*> blocks;
    int64_t bytes = 0;
    cudaError_t err = cudaSuccess;

    template <typename T>
    T* Alloc(size_t count) {
        if (err != cudaSuccess) return nullptr;
        void* p = nullptr;
        const size_t n = std::max<size_t>(count, 1) * sizeof(T);
        err = cudaMalloc(&p, n);
        if (err != cudaSuccess) return nullptr;
        blocks.push_back(p);
        bytes += static_cast<int64_t>(n);
        return static_cast<T*>(p);
    }
    template <typename T>
    T* Upload(const T* src, size_t count) {
        T* d = Alloc<T>(count);
        if (d && count && src) err = cudaMemcpy(d, src, count * sizeof(T), cudaMemcpyHostToDevice);
        return d;
    }
    template <typename T>
    T* Upload(const std::vector<T>& v) {
        return Upload(v.data(), v.size());
    }
    void Release() {
        for (void* p : blocks) cudaFree(p);
        blocks.clear();
        bytes = 0;
    }
};

float HostTriangleArea(const float* a, const float* b, const float* c) {
    const float e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    const float e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    const float cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    const float area = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]) * 0.5f;
    return std::isfinite(area) && area > 0.0f ? area : 0.0f;
}

float HostLuminance(const float* c) { return std::max(0.0f, 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2]); }

constexpr int kMaxBatch = 64;

DevView MakeView(const yrc_camera& c, uint64_t seed) {
    DevView v{};
    std::memcpy(v.cam_origin, c.origin, sizeof(v.cam_origin));
    std::memcpy(v.cam_forward, c.forward, sizeof(v.cam_forward));
    std::memcpy(v.cam_right, c.right, sizeof(v.cam_right));
    std::memcpy(v.cam_up, c.up, sizeof(v.cam_up));
    v.cam_half_height = std::tan(c.fov_y_radians * 0.5f);
    v.seed = seed;
    return v;
}

}  // namespace
}  // namespace yrc

struct yrc_render_scene {
    int device = 0;
    int sm_count = 148;
    yrc_accel* accel = nullptr;
    yrc::DevScene dev{};
    yrc::DeviceArena arena;
    yrc_render_settings settings{};
    int bvh_nodes = 0;
    int bvh_max_depth = 0;
    // Render resources, allocated on first render.
    yrc::DeviceArena work;
    int64_t capacity = 0;
    yrc::PathState ps{};
    yrc::Queues q{};
    float4* transmittance = nullptr;
    yrc_film_pixel* film = nullptr;
    int32_t* attempts = nullptr;
    int32_t* active = nullptr;
    unsigned long long* scalars = nullptr;  // active count, next count, bad, converged
    int32_t* batch = nullptr;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    cudaGraph_t graph_template = nullptr;  // the captured batch, kept for multi-scene launches
    int64_t graph_kernels = 0;             // kernel nodes of the captured batch
    int32_t graph_max_batch = -1;
    int64_t capacity_choice = 0;  // queue capacity chosen by the autotuner or the caller (0: from the image)
    // Radiance cache (optional).
    yrc_nrc* cache = nullptr;
    yrc_cache_settings cache_settings{};
    yrc::DeviceArena cache_work;
    int64_t cache_capacity = 0;
    yrc::TextureSet textures;  // scene textures and their mip chains
    yrc::MeasuredSet measured;  // measured BRDF warps
    yrc::CacheArgs cargs{};
    yrc::DevView* view = nullptr;  // camera and seed (device), see yrc_render_scene_set_view
    std::mutex mutex;
};

namespace yrc {
namespace {
// How a scene traces its shadow rays: the exact per-thread loop (cut-outs,
// textured thin glass), the single-pass transmittance kernel with its
// exact-loop overflow (surfaces that pass light), or the any-hit kernel.
enum class ShadowKind { kExact, kTransmittance, kAnyHit };

ShadowKind ShadowKindOf(const yrc_render_scene* s) {
    if (s->dev.exact_shadows) return ShadowKind::kExact;
    return s->dev.any_transparent ? ShadowKind::kTransmittance : ShadowKind::kAnyHit;
}

ShadowArgs TransmittanceArgs(yrc_render_scene* s, const Queues& q, int64_t C, int* error) {
    const DevScene& sc = s->dev;
    ShadowArgs sa{};
    sa.accel = sc.accel;
    sa.rays = q.shadow_ray;
    sa.count_ptr = q.counters + kCtrShadow;
    sa.capacity = 2 * C;
    sa.out_index = q.shadow_slot;
    sa.transmittance = s->transmittance;
    sa.tri_prim = sc.tri_prim;
    sa.prim_material = sc.prim_material;
    sa.sphere_material = sc.sphere_material;
    sa.materials = sc.materials;
    sa.tri_clear = sc.tri_clear;
    sa.sphere_clear = sc.sphere_clear;
    sa.counter = q.counters + kCtrShadowTrace;
    sa.occluded_count = q.counters + kCtrStatsBase + 2;
    sa.overflow = q.shadow_overflow;
    sa.overflow_count = q.counters + kCtrShadowOverflow;
    sa.error = error;
    sa.leaf_batch = LeafBatchOfShape(TraceShapeOf(s->accel, 1));
    return sa;
}

TraceArgs AnyHitShadowArgs(const Queues& q, const AccelParams& accel, int64_t C, int* error) {
    TraceArgs sh{};
    sh.accel = accel;
    sh.rays = q.shadow_ray;
    sh.count = 2 * C;
    sh.count_ptr = q.counters + kCtrShadow;
    sh.occluded = q.shadow_occluded;
    sh.out_index = q.shadow_slot;
    sh.counter = q.counters + kCtrShadowTrace;
    sh.occluded_count = q.counters + kCtrStatsBase + 2;
    sh.error = error;
    return sh;
}

// Rays that passed more than 16 clear surfaces in the transmittance kernel:
// the exact loop.
void ShadowOverflow(yrc_render_scene* s, const Queues& q, int64_t C, int* error, cudaStream_t st) {
    LaunchShadowExact(s->dev, q, s->transmittance, q.counters + kCtrStatsBase + 2, 2 * C, s->sm_count, error, st,
                      q.shadow_overflow);
}

// The shadow stage of a bounce over the queued shadow rays.
cudaError_t ShadowStage(yrc_render_scene* s, const Queues& q, int64_t C, int* error, cudaStream_t st) {
    cudaError_t err = cudaSuccess;
    switch (ShadowKindOf(s)) {
        case ShadowKind::kExact:
            LaunchShadowExact(s->dev, q, s->transmittance, q.counters + kCtrStatsBase + 2, 2 * C, s->sm_count, error,
                              st);
            err = cudaGetLastError();
            break;
        case ShadowKind::kTransmittance:
            err = LaunchShadowTransmittance(TransmittanceArgs(s, q, C, error), st, s->sm_count);
            if (err == cudaSuccess) {
                ShadowOverflow(s, q, C, error, st);
                err = cudaGetLastError();
            }
            break;
        case ShadowKind::kAnyHit:
            err = LaunchTrace(AnyHitShadowArgs(q, s->dev.accel, C, error), true, false, TraceShapeOf(s->accel, 1), st,
                              s->sm_count);
            break;
    }
    return err;
}

// Releases the scene's captured batch (executable and template).
void DropGraph(yrc_render_scene* s) {
    if (s->graph) cudaGraphExecDestroy(s->graph);
    if (s->graph_template) cudaGraphDestroy(s->graph_template);
    s->graph = nullptr;
    s->graph_template = nullptr;
}
}  // namespace
}  // namespace yrc

extern "C" {

void yrc_render_scene_destroy(yrc_render_scene* scene) {
    if (!scene) return;
    cudaSetDevice(scene->device);
    yrc::DropGraph(scene);
    if (scene->stream) cudaStreamDestroy(scene->stream);
    scene->cache_work.Release();
    scene->work.Release();
    scene->arena.Release();
    scene->textures.Release();
    scene->measured.Release();
    yrc_accel_destroy(scene->accel);
    delete scene;
}

yrc_status yrc_render_scene_set_cache(yrc_render_scene* scene, yrc_nrc* cache, const yrc_cache_settings* settings) {
    using namespace yrc;
    if (!scene) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_render_scene_set_cache: null scene");
    yrc_cache_settings cs{0.01f, 16, 65536, 1, 1};
    if (settings) cs = *settings;
    if (cache && (!(cs.spread_threshold > 0.0f) || cs.train_one_in < 1 || cs.train_records < 0 ||
                  cs.train_steps < 0 || cs.train_steps > 64)) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_render_scene_set_cache: bad settings");
    }
    std::lock_guard<std::mutex> lock(scene->mutex);
    cudaSetDevice(scene->device);
    if (scene->stream) cudaStreamSynchronize(scene->stream);
    yrc::DropGraph(scene);
    scene->cache_work.Release();
    scene->cargs = CacheArgs{};
    scene->cache_capacity = 0;
    scene->cache = cache;
    scene->cache_settings = cs;
    return Ok();
}

int64_t yrc_render_scene_device_bytes(const yrc_render_scene* scene) {
    return scene ? scene->arena.bytes + scene->work.bytes + scene->textures.bytes + scene->measured.bytes +
                       yrc_accel_device_bytes(scene->accel)
                 : 0;
}

yrc_status yrc_render_scene_create(const yrc_scene_desc* desc, yrc_render_scene** out) {
    using namespace yrc;
    if (!desc || !out) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_render_scene_create: null argument");
    *out = nullptr;
    const yrc_geometry& g = desc->geometry;
    const yrc_render_settings& st = desc->settings;
    if (st.width <= 0 || st.height <= 0) return Fail(YRC_ERR_INVALID_ARGUMENT, "Film dimensions must be positive");
    if ((desc->flat == nullptr) == (desc->two_level == nullptr)) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "exactly one of flat / two_level acceleration must be given");
    }
    if (desc->material_count < 0 || (desc->material_count > 0 && !desc->materials) || desc->emissive_count < 0 ||
        (desc->emissive_count > 0 && !desc->emissive)) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "invalid material or light arrays");
    }
    if (desc->analytic_count < 0 || (desc->analytic_count > 0 && !desc->analytic)) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "invalid analytic light array");
    }
    if (desc->texture_count < 0 || (desc->texture_count > 0 && !desc->textures)) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "invalid texture array");
    }
    for (int32_t i = 0; i < desc->material_count; ++i) {
        const yrc_material& m = desc->materials[i];
        if (m.kind == YRC_MAT_SUBSURFACE) {
            if (m.bssrdf_index < 0 || m.bssrdf_index >= desc->bssrdf_count || !desc->bssrdf_tables) {
                return Fail(YRC_ERR_UNSUPPORTED,
                            "material " + std::to_string(i) + ": subsurface material without a BSSRDF table");
            }
            const yrc_bssrdf_table& t = desc->bssrdf_tables[m.bssrdf_index];
            if (t.rho_count < 4 || t.radius_count < 4 || !t.rho_samples || !t.radius_samples || !t.profile ||
                !t.rho_eff || !t.profile_cdf) {
                return Fail(YRC_ERR_INVALID_ARGUMENT, "material " + std::to_string(i) + ": malformed BSSRDF table");
            }
        }
    }
    auto* s = new (std::nothrow) yrc_render_scene();
    if (!s) return Fail(YRC_ERR_OUT_OF_MEMORY, "host allocation failed");
    cudaGetDevice(&s->device);
    cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, s->device);
    s->settings = st;

    yrc_status status = desc->flat ? yrc_accel_create_flat(&g, desc->flat, &s->accel)
                                   : yrc_accel_create_two_level(&g, desc->two_level, &s->accel);
    if (status != YRC_OK) {
        const std::string msg = yrc_last_error();
        yrc_render_scene_destroy(s);
        return Fail(status, msg);
    }
    if (desc->flat) {
        s->bvh_nodes = static_cast<int>(desc->flat->node_count);
        s->bvh_max_depth = desc->flat->max_depth;
    } else {
        int64_t nodes = desc->two_level->tlas_node_count;
        int blas_depth = 0;
        for (int32_t b = 0; b < desc->two_level->blas_count; ++b) {
            nodes += desc->two_level->blases[b].bvh.node_count;
            blas_depth = std::max(blas_depth, desc->two_level->blases[b].bvh.max_depth);
        }
        s->bvh_nodes = static_cast<int>(nodes);
        s->bvh_max_depth = desc->two_level->tlas_max_depth + blas_depth;
    }

    DeviceArena& A = s->arena;
    DevScene& d = s->dev;
    d.accel = AccelParamsOf(s->accel);

    // Shading geometry: flat triangle -> (primitive, vertex indices).
    std::vector<int32_t> tri_prim;
    std::vector<int4> tri_vertices;
    std::vector<int32_t> prim_first_flat(static_cast<size_t>(g.primitive_count), 0);
    for (int32_t p = 0; p < g.primitive_count; ++p) {
        prim_first_flat[static_cast<size_t>(p)] = static_cast<int32_t>(tri_prim.size());
        const uint32_t tris = g.primitives[p].index_count / 3;
        for (uint32_t t = 0; t < tris; ++t) {
            const uint64_t o = static_cast<uint64_t>(g.primitives[p].first_index) + 3ull * t;
            int4 v = make_int4(0, 0, 0, 0);
            if (o + 2 < static_cast<uint64_t>(g.index_count)) {
                v = make_int4(static_cast<int>(g.indices[o]), static_cast<int>(g.indices[o + 1]),
                              static_cast<int>(g.indices[o + 2]), 0);
            }
            tri_prim.push_back(p);
            tri_vertices.push_back(v);
        }
    }
    std::vector<float4> pos(static_cast<size_t>(g.vertex_count));
    for (int64_t v = 0; v < g.vertex_count; ++v) {
        const float* q = VertexPosition(g, static_cast<uint64_t>(v));
        pos[static_cast<size_t>(v)] = make_float4(q[0], q[1], q[2], 0.0f);
    }
    std::vector<float4> nrm;
    if (desc->normals) {
        nrm.resize(static_cast<size_t>(g.vertex_count));
        for (int64_t v = 0; v < g.vertex_count; ++v) {
            const float* q = reinterpret_cast<const float*>(reinterpret_cast<const char*>(desc->normals) +
                                                            v * desc->normal_stride);
            nrm[static_cast<size_t>(v)] = make_float4(q[0], q[1], q[2], 0.0f);
        }
    }
    std::vector<int32_t> prim_material(static_cast<size_t>(g.primitive_count));
    std::vector<uint32_t> prim_flags(static_cast<size_t>(g.primitive_count));
    for (int32_t p = 0; p < g.primitive_count; ++p) {
        const int32_t mi = g.primitives[p].material_index;
        prim_material[static_cast<size_t>(p)] = (mi >= 0 && mi < desc->material_count) ? mi : -1;
        prim_flags[static_cast<size_t>(p)] = g.primitives[p].flags;
    }
    std::vector<float4> spheres(static_cast<size_t>(g.sphere_count));
    std::vector<int32_t> sphere_material(static_cast<size_t>(g.sphere_count)), sphere_flip(static_cast<size_t>(g.sphere_count));
    for (int32_t i = 0; i < g.sphere_count; ++i) {
        const yrc_sphere& sp = g.spheres[i];
        spheres[static_cast<size_t>(i)] = make_float4(sp.center[0], sp.center[1], sp.center[2], sp.radius);
        sphere_material[static_cast<size_t>(i)] =
            (sp.material_index >= 0 && sp.material_index < desc->material_count) ? sp.material_index : -1;
        sphere_flip[static_cast<size_t>(i)] = sp.flip_normals ? 1 : 0;
    }
    std::vector<float> o2w;
    if (desc->two_level) {
        for (int32_t i = 0; i < desc->two_level->instance_count; ++i) {
            const float* m = desc->two_level->instances[i].object_to_world;
            o2w.insert(o2w.end(), m, m + 16);
        }
    }
    d.tri_prim = A.Upload(tri_prim);
    d.tri_vertices = A.Upload(tri_vertices);
    d.positions = A.Upload(pos);
    d.normals = nrm.empty() ? nullptr : A.Upload(nrm);
    d.prim_material = A.Upload(prim_material);
    d.prim_flags = A.Upload(prim_flags);
    d.spheres = A.Upload(spheres);
    d.sphere_material = A.Upload(sphere_material);
    d.sphere_flip = A.Upload(sphere_flip);
    d.instance_o2w = A.Upload(o2w);
    // RenderVertex uv and tangent (+ handedness), when given.
    if (desc->uvs) {
        std::vector<float2> uv(static_cast<size_t>(g.vertex_count));
        for (int64_t v = 0; v < g.vertex_count; ++v) {
            const float* q = reinterpret_cast<const float*>(reinterpret_cast<const char*>(desc->uvs) + v * desc->uv_stride);
            uv[static_cast<size_t>(v)] = make_float2(q[0], q[1]);
        }
        d.uvs = A.Upload(uv);
    }
    if (desc->tangents) {
        std::vector<float4> tg(static_cast<size_t>(g.vertex_count));
        for (int64_t v = 0; v < g.vertex_count; ++v) {
            const float* q =
                reinterpret_cast<const float*>(reinterpret_cast<const char*>(desc->tangents) + v * desc->tangent_stride);
            tg[static_cast<size_t>(v)] = make_float4(q[0], q[1], q[2], q[3]);
        }
        d.tangents = A.Upload(tg);
    }
    d.primitive_count = g.primitive_count;
    d.sphere_count = g.sphere_count;
    d.instance_count = desc->two_level ? desc->two_level->instance_count : 0;

    // Materials.
    std::vector<DevMaterial> mats(static_cast<size_t>(desc->material_count));
    bool transparent = false;
    for (int32_t i = 0; i < desc->material_count; ++i) {
        const yrc_material& m = desc->materials[i];
        DevMaterial& dm = mats[static_cast<size_t>(i)];
        std::memset(&dm, 0, sizeof(dm));
        dm.kind = m.kind;
        std::memcpy(dm.reflectance, m.reflectance, sizeof(dm.reflectance));
        dm.ior = m.ior;
        dm.uroughness = m.uroughness;
        dm.vroughness = m.vroughness;
        dm.coating_ior = m.coating_ior;
        dm.coat_thickness = m.coat_thickness;
        std::memcpy(dm.coat_absorption, m.coat_absorption, sizeof(dm.coat_absorption));
        dm.coat_maxdepth = m.coat_maxdepth;
        dm.coat_nsamples = m.coat_nsamples;
        std::memcpy(dm.emission, m.emission, sizeof(dm.emission));
        std::memcpy(dm.absorption_color, m.absorption_color, sizeof(dm.absorption_color));
        dm.absorption_distance = m.absorption_distance;
        std::memcpy(dm.sigma_a, m.sigma_a, sizeof(dm.sigma_a));
        std::memcpy(dm.sigma_s, m.sigma_s, sizeof(dm.sigma_s));
        dm.bssrdf_eta = m.bssrdf_eta;
        dm.bssrdf_index = m.bssrdf_index;
        dm.reflectance_texture = m.reflectance_texture;
        dm.alpha_texture = m.alpha_texture;
        dm.normal_map = m.normal_map;
        dm.alpha = m.alpha;
        dm.normal_scale = m.normal_scale;
        dm.measured_index = (m.kind == YRC_MAT_MEASURED && m.measured_index >= 0 && m.measured_index < desc->measured_count)
                                ? m.measured_index
                                : -1;
        if (m.kind == YRC_MAT_DIELECTRIC || m.kind == YRC_MAT_THIN_DIELECTRIC) transparent = true;
        if (m.kind == YRC_MAT_COATED_DIFFUSE || m.kind == YRC_MAT_COATED_CONDUCTOR) d.any_layered = 1;
        const bool tex_alpha = m.alpha_texture >= 0 && m.alpha_texture < desc->texture_count;
        const bool tex_refl = m.reflectance_texture >= 0 && m.reflectance_texture < desc->texture_count;
        if (m.alpha < 0.5f || tex_alpha) d.any_alpha = 1;
        if (m.alpha < 0.5f || tex_alpha || (m.kind == YRC_MAT_THIN_DIELECTRIC && tex_refl)) d.exact_shadows = 1;
    }
    d.materials = A.Upload(mats);
    d.material_count = desc->material_count;
    d.any_transparent = transparent ? 1 : 0;
    if (transparent) {
        // Surfaces a shadow ray may pass (TraceShadowVisibility continues only
        // through Dielectric and ThinDielectric hits).
        auto clear = [&](int32_t mi) {
            return static_cast<uint8_t>(mi >= 0 && (mats[static_cast<size_t>(mi)].kind == YRC_MAT_DIELECTRIC ||
                                                    mats[static_cast<size_t>(mi)].kind == YRC_MAT_THIN_DIELECTRIC));
        };
        std::vector<uint8_t> tri_clear(tri_prim.size()), sphere_clear(sphere_material.size());
        for (size_t t = 0; t < tri_prim.size(); ++t) {
            const int32_t p = tri_prim[t];
            tri_clear[t] = p >= 0 ? clear(prim_material[static_cast<size_t>(p)]) : 0;
        }
        for (size_t i = 0; i < sphere_material.size(); ++i) sphere_clear[i] = clear(sphere_material[i]);
        d.tri_clear = A.Upload(tri_clear);
        d.sphere_clear = A.Upload(sphere_clear);
    }

    // Emissive lights, alias table, per-light triangle area CDF.
    const int32_t ne = desc->emissive_count;
    std::vector<int32_t> e_prim(static_cast<size_t>(ne)), tri_off(static_cast<size_t>(ne)), tri_cnt(static_cast<size_t>(ne));
    std::vector<float> e_rad(static_cast<size_t>(ne) * 3), e_area(static_cast<size_t>(ne)), e_parea(static_cast<size_t>(ne));
    std::vector<float> cdf;
    std::vector<int32_t> cdf_tri;
    std::vector<int32_t> prim_emissive(static_cast<size_t>(g.primitive_count), -1);
    float total_power = 0.0f;
    for (int32_t e = 0; e < ne; ++e) {
        const yrc_emissive_primitive& ep = desc->emissive[e];
        e_prim[static_cast<size_t>(e)] = ep.primitive_index;
        std::memcpy(&e_rad[3 * static_cast<size_t>(e)], ep.radiance, 3 * sizeof(float));
        e_area[static_cast<size_t>(e)] = ep.area;
        const float area = std::isfinite(ep.area) && ep.area > 0.0f ? ep.area : 0.0f;
        total_power += area * HostLuminance(ep.radiance);
        tri_off[static_cast<size_t>(e)] = static_cast<int32_t>(cdf.size());
        float cum = 0.0f;
        if (ep.primitive_index >= 0 && ep.primitive_index < g.primitive_count) {
            if (prim_emissive[static_cast<size_t>(ep.primitive_index)] < 0) {
                prim_emissive[static_cast<size_t>(ep.primitive_index)] = e;
            }
            const yrc_primitive& pr = g.primitives[ep.primitive_index];
            const uint32_t tris = pr.index_count / 3;
            for (uint32_t t = 0; t < tris; ++t) {
                const uint64_t o = static_cast<uint64_t>(pr.first_index) + 3ull * t;
                const float a = HostTriangleArea(VertexPosition(g, g.indices[o]), VertexPosition(g, g.indices[o + 1]),
                                                 VertexPosition(g, g.indices[o + 2]));
                if (a <= 0.0f) continue;
                cum += a;
                cdf.push_back(cum);
                cdf_tri.push_back(prim_first_flat[static_cast<size_t>(ep.primitive_index)] + static_cast<int32_t>(t));
            }
        }
        tri_cnt[static_cast<size_t>(e)] = static_cast<int32_t>(cdf.size()) - tri_off[static_cast<size_t>(e)];
        e_parea[static_cast<size_t>(e)] = cum;
    }
    d.emissive_count = ne;
    d.emissive_prim = A.Upload(e_prim);
    d.emissive_radiance = A.Upload(e_rad);
    d.emissive_area = A.Upload(e_area);
    d.emissive_tri_offset = A.Upload(tri_off);
    d.emissive_tri_count = A.Upload(tri_cnt);
    d.tri_cdf = A.Upload(cdf);
    d.tri_local = A.Upload(cdf_tri);
    d.emissive_prim_area = A.Upload(e_parea);
    d.prim_emissive = A.Upload(prim_emissive);
    d.total_emissive_power = total_power;
    const yrc_alias_table& at = desc->emissive_power;
    d.alias_count = (at.count == ne && at.probability && at.alias && at.pmf) ? ne : 0;
    d.alias_prob = d.alias_count ? A.Upload(at.probability, static_cast<size_t>(ne)) : nullptr;
    d.alias_index = d.alias_count ? A.Upload(at.alias, static_cast<size_t>(ne)) : nullptr;
    d.alias_pmf = d.alias_count ? A.Upload(at.pmf, static_cast<size_t>(ne)) : nullptr;

    // Environment.
    const yrc_environment& env = desc->environment;
    DevEnvironment& de = d.env;
    std::memset(&de, 0, sizeof(de));
    de.active = env.active;
    std::memcpy(de.radiance, env.radiance, sizeof(de.radiance));
    de.strength = env.strength;
    de.rotation = env.rotation_radians;
    if (env.active && env.texels && env.width > 0 && env.height > 0) {
        const size_t texels = static_cast<size_t>(env.width) * static_cast<size_t>(env.height);
        de.width = env.width;
        de.height = env.height;
        de.texels = A.Upload(env.texels, texels * 4);
        if (env.texel_weights && env.row_weights && env.row_cdf && env.conditional_cdfs) {
            de.texel_weights = A.Upload(env.texel_weights, texels);
            de.row_weights = A.Upload(env.row_weights, static_cast<size_t>(env.height));
            de.row_cdf = A.Upload(env.row_cdf, static_cast<size_t>(env.height));
            de.conditional_cdfs = A.Upload(env.conditional_cdfs, texels);
            de.total_weight = env.total_weight;
        }
    }

    // BSSRDF tables (ComputeBeamDiffusionBSSRDF output, consumed as given).
    if (desc->bssrdf_count > 0 && desc->bssrdf_tables) {
        std::vector<DevBssrdf> tables(static_cast<size_t>(desc->bssrdf_count));
        for (int32_t i = 0; i < desc->bssrdf_count; ++i) {
            const yrc_bssrdf_table& t = desc->bssrdf_tables[i];
            DevBssrdf& b = tables[static_cast<size_t>(i)];
            const size_t cells = static_cast<size_t>(t.rho_count) * static_cast<size_t>(t.radius_count);
            b.rho_count = t.rho_count;
            b.radius_count = t.radius_count;
            b.rho = A.Upload(t.rho_samples, static_cast<size_t>(t.rho_count));
            b.radius = A.Upload(t.radius_samples, static_cast<size_t>(t.radius_count));
            b.profile = A.Upload(t.profile, cells);
            b.rho_eff = A.Upload(t.rho_eff, static_cast<size_t>(t.rho_count));
            b.profile_cdf = A.Upload(t.profile_cdf, cells);
        }
        d.bssrdf = A.Upload(tables);
        d.bssrdf_count = desc->bssrdf_count;
    }
    for (int32_t i = 0; i < desc->material_count; ++i) {
        if (desc->materials[i].kind == YRC_MAT_SUBSURFACE) d.any_subsurface = 1;
    }

    // Analytic lights (PrepareLightSampling, src/lighting/light_sampling.cpp:
    // 205-275): the power alias table (the caller's, else built here from the
    // same weights) and, when every light is local and there are more than
    // 8, the power / distance tree.
    d.analytic_count = desc->analytic_count;
    d.analytic_tree_root = -1;
    if (desc->analytic_count > 0) {
        const int32_t n = desc->analytic_count;
        std::vector<DevAnalytic> lights(static_cast<size_t>(n));
        std::vector<float> weights(static_cast<size_t>(n));
        std::vector<int> local;
        for (int32_t i = 0; i < n; ++i) {
            const yrc_analytic_light& l = desc->analytic[i];
            DevAnalytic& a = lights[static_cast<size_t>(i)];
            a.kind = l.kind;
            std::memcpy(a.position, l.position, sizeof(a.position));
            std::memcpy(a.direction, l.direction, sizeof(a.direction));
            std::memcpy(a.intensity, l.intensity, sizeof(a.intensity));
            a.cone_angle = l.cone_angle;
            a.cone_cos_inner = l.cone_cos_inner;
            float power = std::max(0.0f, 0.2126f * l.intensity[0] + 0.7152f * l.intensity[1] + 0.0722f * l.intensity[2]);
            if (l.kind == 1) {
                power *= std::max(0.0f, 2.0f * 3.14159265358979323846f * (1.0f - l.cone_angle));
            } else if (l.kind == 0) {
                power *= 4.0f * 3.14159265358979323846f;
            }
            weights[static_cast<size_t>(i)] = power;
            if (l.kind != 2 && power > 0.0f) local.push_back(i);
        }
        d.analytic = A.Upload(lights);
        std::vector<float> prob(static_cast<size_t>(n)), pmf(static_cast<size_t>(n));
        std::vector<int32_t> alias(static_cast<size_t>(n));
        const yrc_alias_table& at = desc->analytic_power;
        if (at.count == n && at.probability && at.alias && at.pmf) {
            prob.assign(at.probability, at.probability + n);
            alias.assign(at.alias, at.alias + n);
            pmf.assign(at.pmf, at.pmf + n);
        } else {
            yrc_alias_table_build(weights.data(), n, prob.data(), alias.data(), pmf.data());
        }
        d.analytic_alias_prob = A.Upload(prob);
        d.analytic_alias_index = A.Upload(alias);
        d.analytic_alias_pmf = A.Upload(pmf);
        if (static_cast<int32_t>(local.size()) == n && n > 8) {
            std::vector<DevLightNode> nodes;
            nodes.reserve(local.size() * 2);
            std::function<int(size_t, size_t)> build = [&](size_t begin, size_t end) -> int {
                float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
                float power = 0.0f;
                for (size_t i = begin; i < end; ++i) {
                    const float* pos = desc->analytic[local[i]].position;
                    for (int k = 0; k < 3; ++k) {
                        lo[k] = std::min(lo[k], pos[k]);
                        hi[k] = std::max(hi[k], pos[k]);
                    }
                    power += weights[static_cast<size_t>(local[i])];
                }
                const int node = static_cast<int>(nodes.size());
                nodes.push_back(DevLightNode{{lo[0], lo[1], lo[2]}, {hi[0], hi[1], hi[2]}, power, -1, -1, -1});
                if (end - begin == 1) {
                    nodes[static_cast<size_t>(node)].light_index = local[begin];
                    return node;
                }
                const float ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
                const int axis = ex >= ey && ex >= ez ? 0 : (ey >= ez ? 1 : 2);
                const size_t middle = begin + (end - begin) / 2;
                std::nth_element(local.begin() + static_cast<std::ptrdiff_t>(begin),
                                 local.begin() + static_cast<std::ptrdiff_t>(middle),
                                 local.begin() + static_cast<std::ptrdiff_t>(end), [&](int a, int b) {
                                     return desc->analytic[a].position[axis] < desc->analytic[b].position[axis];
                                 });
                const int left = build(begin, middle);
                const int right = build(middle, end);
                nodes[static_cast<size_t>(node)].left = left;
                nodes[static_cast<size_t>(node)].right = right;
                return node;
            };
            d.analytic_tree_root = build(0, local.size());
            d.analytic_tree = A.Upload(nodes);
        }
    }

    // Camera and settings.
    const DevView view = MakeView(desc->camera, st.seed);
    s->view = A.Upload(&view, 1);
    d.view = s->view;
    d.width = st.width;
    d.height = st.height;
    d.spp = std::max(1, st.spp);
    d.max_depth = std::max(1, st.max_depth);
    d.sampler = st.sampler;
    d.radiance_clamp = st.radiance_clamp;

    if (A.err != cudaSuccess) {
        const cudaError_t err = A.err;
        yrc_render_scene_destroy(s);
        return CudaError(err, "render scene upload");
    }
    // Textures: BuildTextureSamplingCaches on the device.
    if (desc->texture_count > 0) {
        const yrc_status ts = UploadTextures(desc->textures, desc->texture_count, nullptr, s->textures);
        if (ts != YRC_OK) {
            const std::string msg = yrc_last_error();
            yrc_render_scene_destroy(s);
            return Fail(ts, msg);
        }
        d.textures = s->textures.textures;
        d.texture_count = s->textures.count;
        d.ewa_weights = s->textures.ewa_weights;
    }
    if (desc->measured_count > 0) {
        const yrc_status ms = UploadMeasured(desc->measured, desc->measured_count, s->measured);
        if (ms != YRC_OK) {
            const std::string msg = yrc_last_error();
            yrc_render_scene_destroy(s);
            return Fail(ms, msg);
        }
        d.measured = s->measured.brdfs;
        d.measured_count = s->measured.count;
    }
    *out = s;
    return Ok();
}

}  // extern "C"

namespace yrc {
namespace {

// Concurrent paths of a render: the autotuned (or caller's) choice, else
// enough for several passes of a small image at once and one full pass of a
// large one; always at least one pass of every pixel (a batch renders whole
// passes) and at most kMaxBatch passes.
int64_t RenderCapacity(const yrc_render_scene* s) {
    const int64_t pixels = static_cast<int64_t>(s->settings.width) * s->settings.height;
    const int64_t most = pixels * std::min(std::max(1, s->settings.spp), kMaxBatch);
    const int64_t c = s->capacity_choice > 0 ? s->capacity_choice : std::max<int64_t>(pixels, int64_t{1} << 21);
    return std::min(std::max(c, pixels), most);
}

// Allocates the path state and queues for `capacity` paths.
yrc_status EnsureWork(yrc_render_scene* s, int64_t capacity) {
    const int64_t pixels = static_cast<int64_t>(s->settings.width) * s->settings.height;
    if (s->capacity == capacity && s->film) return Ok();
    DropGraph(s);
    s->work.Release();
    DeviceArena& W = s->work;
    PathState& ps = s->ps;
    ps.pixel = W.Alloc<int32_t>(capacity);
    ps.sample = W.Alloc<int32_t>(capacity);
    ps.throughput = W.Alloc<float4>(capacity);
    ps.radiance = W.Alloc<float4>(capacity);
    ps.prev = W.Alloc<float4>(capacity);
    ps.flags = W.Alloc<uint32_t>(capacity);
    ps.medium = W.Alloc<float4>(capacity);
    ps.rng_state = W.Alloc<uint64_t>(capacity);
    ps.rng_inc = W.Alloc<uint64_t>(capacity);
    ps.aov_albedo = W.Alloc<float4>(capacity);
    ps.aov_normal = W.Alloc<float4>(capacity);
    ps.nee = W.Alloc<float4>(3 * capacity);
    ps.nee_tp = W.Alloc<float4>(capacity);
    ps.spread = W.Alloc<float2>(capacity);
    ps.nee_vis = nullptr;
    ps.defer = s->dev.any_layered ? W.Alloc<float4>(5 * capacity) : nullptr;
    Queues& q = s->q;
    q.ray_in = W.Alloc<float4>(2 * capacity);
    q.path_in = W.Alloc<int32_t>(capacity);
    q.hits = W.Alloc<float4>(capacity);
    q.inst = W.Alloc<int32_t>(capacity);
    q.ray_out = W.Alloc<float4>(2 * capacity);
    q.path_out = W.Alloc<int32_t>(capacity);
    q.shadow_ray = W.Alloc<float4>(2 * 2 * capacity);
    q.shadow_slot = W.Alloc<int32_t>(2 * capacity);
    q.shadow_occluded = W.Alloc<uint8_t>(3 * capacity);
    q.shadow_overflow =
        (s->dev.any_transparent && !s->dev.exact_shadows) ? W.Alloc<int32_t>(2 * capacity) : nullptr;
    q.nee_paths = W.Alloc<int32_t>(capacity);
    q.defer_paths = s->dev.any_layered ? W.Alloc<int32_t>(capacity) : nullptr;
    q.defer_paths2 = s->dev.any_layered ? W.Alloc<int32_t>(capacity) : nullptr;
    q.order = W.Alloc<int32_t>(capacity);
    q.shade_class = W.Alloc<uint8_t>(capacity);
    q.tex_normal = s->dev.texture_count > 0 ? W.Alloc<float4>(capacity) : nullptr;
    q.tex_scale = s->dev.texture_count > 0 ? W.Alloc<float4>(capacity) : nullptr;
    q.counters = W.Alloc<unsigned long long>(kCtrCount);
    s->transmittance = (s->dev.any_transparent || s->dev.exact_shadows) ? W.Alloc<float4>(3 * capacity) : nullptr;
    if (s->dev.any_subsurface) {
        q.probe_ray = W.Alloc<float4>(2 * capacity);
        q.probe_target = W.Alloc<int4>(capacity);
        q.probe_entry = W.Alloc<float4>(2 * capacity);
        q.probe_hit = W.Alloc<float4>(capacity);
        q.probe_count = W.Alloc<int32_t>(capacity);
    }
    s->film = W.Alloc<yrc_film_pixel>(static_cast<size_t>(pixels));
    s->attempts = W.Alloc<int32_t>(static_cast<size_t>(pixels));
    s->active = W.Alloc<int32_t>(static_cast<size_t>(pixels));
    s->scalars = W.Alloc<unsigned long long>(4);
    s->batch = W.Alloc<int32_t>(1);
    if (W.err == cudaSuccess && !s->stream) W.err = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (W.err != cudaSuccess) {
        const cudaError_t err = W.err;
        s->work.Release();
        s->film = nullptr;
        s->capacity = 0;
        return CudaError(err, "render working memory");
    }
    if (s->transmittance) cudaMemsetAsync(s->transmittance, 0, sizeof(float4) * 3 * capacity, s->stream);
    cudaMemsetAsync(q.shadow_occluded, 1, 3 * capacity, s->stream);
    s->capacity = capacity;
    return Ok();
}

// Allocates the radiance-cache queues for `capacity` paths (or releases
// them when no cache is attached).
yrc_status EnsureCache(yrc_render_scene* s) {
    if (!s->cache) {
        s->cargs = CacheArgs{};
        return Ok();
    }
    if (s->cache_capacity == s->capacity && s->cargs.enabled) return Ok();
    DropGraph(s);
    s->cache_work.Release();
    DeviceArena& W = s->cache_work;
    const yrc_cache_settings& cs = s->cache_settings;
    const int64_t cap = s->capacity;
    CacheArgs c{};
    c.enabled = 1;
    c.spread_c = cs.spread_threshold;
    c.train_one_in = std::max(1, cs.train_one_in);
    c.delta_vertices = cs.delta_vertices != 0;
    c.train_records = cs.train ? std::max(128, cs.train_records) : 0;
    c.train_paths = cs.train ? static_cast<int32_t>(std::min<int64_t>(cap, c.train_records)) : 0;
    c.max_depth = s->dev.max_depth;
    // The film's radiance clamp when set, else the brightest emitter the
    // instanced scenes carry (a 1e4 sun).
    c.target_max = s->dev.radiance_clamp > 0.0f ? s->dev.radiance_clamp : 1.0e4f;
    c.queries = W.Alloc<float>(16 * cap);
    c.query_path = W.Alloc<int32_t>(cap);
    c.query_tp = W.Alloc<float4>(cap);
    c.query_base = W.Alloc<float4>(cap);
    c.query_rgb = W.Alloc<float4>(cap);
    c.train_slot = W.Alloc<int32_t>(cap);
    const int64_t tp = std::max<int32_t>(c.train_paths, 1);
    c.slot_path = W.Alloc<int32_t>(tp);
    c.slot_len = W.Alloc<int32_t>(tp);
    c.slot_q = W.Alloc<float>(16 * tp * std::max(1, c.max_depth));
    c.slot_lt = W.Alloc<float4>(2 * tp * std::max(1, c.max_depth));
    c.rec_q = W.Alloc<float>(16 * static_cast<int64_t>(std::max(c.train_records, 1)));
    c.rec_t = W.Alloc<float4>(std::max(c.train_records, 1));
    c.counters = W.Alloc<unsigned long long>(4);
    if (W.err != cudaSuccess) {
        const cudaError_t err = W.err;
        s->cache_work.Release();
        s->cargs = CacheArgs{};
        s->cache_capacity = 0;
        return CudaError(err, "radiance cache working memory");
    }
    s->cargs = c;
    s->cache_capacity = cap;
    return Ok();
}

// One batch of a scene in stages (generate; per bounce: counters, extend
// trace, shading, shadow trace, next-event resolve; film), so that a pooled
// batch of several scenes can interleave them with shared traversal
// launches. Queues `q` are the scene's queues at this bounce (the extend
// queues alternate between bounces).

yrc_status BatchPrologue(yrc_render_scene* s, cudaStream_t st) {
    const CacheArgs& cache = s->cargs;
    if (cache.enabled) {
        const cudaError_t err = cudaMemsetAsync(cache.counters, 0, 4 * sizeof(unsigned long long), st);
        if (err != cudaSuccess) return CudaError(err, "cache counters");
    }
    BatchArgs b{s->active, s->scalars + 0, s->scalars + 1, s->batch, s->film};
    LaunchGenerate(s->dev, s->ps, s->q, b, cache, s->capacity, s->sm_count, st);
    return Ok();
}

// The extend trace's arguments (closest hit over the current queue).
TraceArgs ExtendTraceArgs(yrc_render_scene* s, const Queues& q) {
    TraceArgs ta{};
    ta.accel = s->dev.accel;
    ta.rays = q.ray_in;
    ta.count = s->capacity;
    ta.count_ptr = q.counters + kCtrIn;
    ta.hits = reinterpret_cast<yrc_hit*>(q.hits);
    ta.instances = q.inst;
    ta.counter = q.counters + kCtrTrace;
    ta.error = AccelErrorWord(s->accel);
    return ta;
}

// Shading after the extend trace, in three parts: alpha skips and the sort
// of the extend queue by shading class; the class shade kernels (pooled
// over several scenes in a pooled batch); subsurface probes and exits.
void BounceShadeSort(yrc_render_scene* s, const Queues& q, int depth, cudaStream_t st) {
    const DevScene& sc = s->dev;
    const int64_t C = s->capacity;
    if (sc.any_alpha) LaunchAlphaExtend(sc, s->ps, q, depth, C, s->sm_count, AccelErrorWord(s->accel), st);
    LaunchShadeSort(sc, s->ps, q, depth, C, s->sm_count, st);
}

yrc_status BounceSubsurface(yrc_render_scene* s, const Queues& q, int depth, cudaStream_t st) {
    const DevScene& sc = s->dev;
    const int64_t C = s->capacity;
    if (sc.any_subsurface) {
        RenderProbeArgs pa{};
        pa.accel = sc.accel;
        pa.rays = q.probe_ray;
        pa.targets = q.probe_target;
        pa.selection = q.probe_entry;
        pa.count_ptr = q.counters + kCtrProbe;
        pa.capacity = C;
        pa.hit = q.probe_hit;
        pa.hits = q.probe_count;
        pa.error = AccelErrorWord(s->accel);
        const cudaError_t perr = LaunchRenderProbe(pa, st, s->sm_count);
        if (perr != cudaSuccess) return CudaError(perr, "subsurface probe");
        LaunchSubsurfaceExit(sc, s->ps, q, depth, C, s->sm_count, st);
    }
    return Ok();
}

yrc_status BounceShade(yrc_render_scene* s, const Queues& q, int depth, cudaStream_t st) {
    BounceShadeSort(s, q, depth, st);
    LaunchShadeClasses(s->dev, s->ps, q, s->cargs, depth, s->capacity, s->sm_count, st);
    return BounceSubsurface(s, q, depth, st);
}

// After the shadow trace: next-event resolve, coated vertices (with their
// own second shadow stage), and the next bounce's queue.
yrc_status BounceResolve(yrc_render_scene* s, const Queues& q, int depth, cudaStream_t st) {
    const DevScene& sc = s->dev;
    const int64_t C = s->capacity;
    LaunchNeeResolve(s->ps, q, s->transmittance, C, s->sm_count, st);
    if (sc.any_layered) {
        // Coated vertices: their next events in the reference's PCG32
        // order, with a second shadow stage in between.
        LaunchLayeredNee(sc, s->ps, q, s->transmittance, depth, C, s->sm_count, st);
        const cudaError_t err = ShadowStage(s, q, C, AccelErrorWord(s->accel), st);
        if (err != cudaSuccess) return CudaError(err, "coated-vertex shadow trace");
        LaunchLayeredContinue(sc, s->ps, q, s->transmittance, depth, C, s->sm_count, st);
    }
    LaunchAdvanceQueue(q, st);
    return Ok();
}

// After the last bounce: the radiance cache's inference and training, the
// film, and the next batch's active list.
yrc_status BatchEpilogue(yrc_render_scene* s, int32_t max_batch, cudaStream_t st) {
    const DevScene& sc = s->dev;
    const int64_t C = s->capacity;
    const int64_t pixels = static_cast<int64_t>(sc.width) * sc.height;
    BatchArgs b{s->active, s->scalars + 0, s->scalars + 1, s->batch, s->film};
    FilmArgs f{s->attempts, s->scalars + 2, s->scalars + 3, s->settings.adaptive_enabled, s->settings.adaptive_min_spp,
               s->settings.adaptive_relative_error, s->settings.adaptive_absolute_error,
               s->settings.adaptive_confidence};
    const CacheArgs& cache = s->cargs;
    if (cache.enabled) {
        // Training targets from the unbiased training paths' full radiance;
        // then every path that ended at the cache (training paths at their
        // first terminal vertex too) gets its image estimate; then the
        // training steps.
        yrc_status cs = nrc::Infer(s->cache, cache.queries, C, cache.counters + 0,
                                   reinterpret_cast<float*>(cache.query_rgb), st, s->cache_settings.averaged != 0);
        if (cs != YRC_OK) return cs;
        if (cache.train_records > 0) LaunchCacheTargets(s->ps, cache, s->sm_count, st);
        LaunchCacheResolve(s->ps, cache, C, s->sm_count, st);
        if (cache.train_records > 0) {
            for (int k = 0; k < std::max(1, s->cache_settings.train_steps); ++k) {
                cs = nrc::TrainStep(s->cache, cache.rec_q, reinterpret_cast<const float*>(cache.rec_t),
                                    cache.train_records, cache.counters + 2, st);
                if (cs != YRC_OK) return cs;
            }
        }
    }
    LaunchFilm(sc, s->ps, b, f, pixels, s->sm_count, st);
    LaunchActivePixels(sc, b, f, pixels, s->sm_count, st);
    LaunchFinishActive(s->scalars + 0, s->scalars + 1, s->batch, max_batch, C, st);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return CudaError(err, "batch launch");
    return Ok();
}

// Records one batch (generate, max_depth bounces, film, next active list).
yrc_status EnqueueBatch(yrc_render_scene* s, int32_t max_batch) {
    cudaStream_t st = s->stream;
    yrc_status status = BatchPrologue(s, st);
    Queues q = s->q;
    for (int depth = 0; depth < s->dev.max_depth && status == YRC_OK; ++depth) {
        LaunchResetCounters(q, st);
        const TraceArgs ta = ExtendTraceArgs(s, q);
        cudaError_t err = LaunchTrace(ta, false, false, TraceShapeOf(s->accel, 0), st, s->sm_count);
        if (err != cudaSuccess) return CudaError(err, "extend trace");
        status = BounceShade(s, q, depth, st);
        if (status != YRC_OK) return status;
        err = ShadowStage(s, q, s->capacity, ta.error, st);
        if (err != cudaSuccess) return CudaError(err, "shadow trace");
        status = BounceResolve(s, q, depth, st);
        std::swap(q.ray_in, q.ray_out);
        std::swap(q.path_in, q.path_out);
    }
    if (status != YRC_OK) return status;
    return BatchEpilogue(s, max_batch, st);
}

// Captures one batch as a CUDA graph (all sizes are read on the device),
// unless the scene holds one for this batch bound.
yrc_status EnsureGraph(yrc_render_scene* s, int32_t max_batch) {
    if (s->graph && s->graph_max_batch == max_batch) return Ok();
    DropGraph(s);
    cudaGraph_t graph = nullptr;
    cudaError_t err = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
    if (err != cudaSuccess) return CudaError(err, "graph capture");
    const yrc_status status = EnqueueBatch(s, max_batch);
    err = cudaStreamEndCapture(s->stream, &graph);
    if (status != YRC_OK) {
        if (graph) cudaGraphDestroy(graph);
        return status;
    }
    if (err != cudaSuccess) return CudaError(err, "graph capture");
    err = cudaGraphInstantiate(&s->graph, graph, 0);
    if (err != cudaSuccess) {
        cudaGraphDestroy(graph);
        return CudaError(err, "graph instantiate");
    }
    s->graph_template = graph;
    s->graph_max_batch = max_batch;
    size_t nodes = 0;
    s->graph_kernels = 0;
    if (cudaGraphGetNodes(graph, nullptr, &nodes) == cudaSuccess && nodes > 0) {
        std::vector<cudaGraphNode_t> list(nodes);
        if (cudaGraphGetNodes(graph, list.data(), &nodes) == cudaSuccess) {
            for (size_t i = 0; i < nodes; ++i) {
                cudaGraphNodeType type;
                if (cudaGraphNodeGetType(list[i], &type) == cudaSuccess && type == cudaGraphNodeTypeKernel) {
                    ++s->graph_kernels;
                }
            }
        }
    }
    return Ok();
}

// Renders sample indices 0..passes-1 of every pixel into the device film
// with the scene's current capacity and launch shapes (no resume, no
// progress, no readback); returns the device time of the batches.
yrc_status ProbeRender(yrc_render_scene* s, int32_t passes, double* seconds) {
    const int64_t pixels = static_cast<int64_t>(s->settings.width) * s->settings.height;
    const int spp = std::max(1, s->settings.spp);
    yrc_status status = EnsureWork(s, RenderCapacity(s));
    if (status == YRC_OK) status = EnsureCache(s);
    if (status != YRC_OK) return status;
    cudaStream_t stream = s->stream;
    const std::vector<int32_t> attempts(static_cast<size_t>(pixels), passes);
    cudaMemsetAsync(s->film, 0, sizeof(yrc_film_pixel) * pixels, stream);
    cudaMemcpyAsync(s->attempts, attempts.data(), sizeof(int32_t) * pixels, cudaMemcpyHostToDevice, stream);
    cudaMemsetAsync(s->scalars, 0, 4 * sizeof(unsigned long long), stream);
    cudaMemsetAsync(s->q.counters, 0, sizeof(unsigned long long) * kCtrCount, stream);
    const int32_t max_batch = std::min(spp, kMaxBatch);
    {
        BatchArgs b{s->active, s->scalars + 0, s->scalars + 1, s->batch, s->film};
        FilmArgs f{s->attempts, s->scalars + 2, s->scalars + 3, 0, 0, 0.0f, 0.0f, 0.0f};
        LaunchActivePixels(s->dev, b, f, pixels, s->sm_count, stream);
        LaunchFinishActive(s->scalars + 0, s->scalars + 1, s->batch, max_batch, s->capacity, stream);
    }
    status = EnsureGraph(s, max_batch);
    if (status != YRC_OK) return status;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, stream);
    unsigned long long active = 0;
    cudaMemcpyAsync(&active, s->scalars, sizeof(active), cudaMemcpyDeviceToHost, stream);
    cudaError_t err = cudaStreamSynchronize(stream);
    for (int guard = 0; err == cudaSuccess && active > 0 && guard <= passes; ++guard) {
        err = cudaGraphLaunch(s->graph, stream);
        if (err == cudaSuccess) err = cudaMemcpyAsync(&active, s->scalars, sizeof(active), cudaMemcpyDeviceToHost, stream);
        if (err == cudaSuccess) err = cudaStreamSynchronize(stream);
    }
    cudaEventRecord(e1, stream);
    if (err == cudaSuccess) err = cudaEventSynchronize(e1);
    float ms = 0.0f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err != cudaSuccess) return CudaError(err, "autotune probe");
    status = CheckDeviceError(s->accel);
    if (status != YRC_OK) return status;
    *seconds = ms / 1e3;
    return Ok();
}

}  // namespace
}  // namespace yrc

namespace yrc {
namespace {

// One render call on one prepared scene, split into the steps that a
// multi-scene call interleaves: Begin (checks, uploads, active list, batch
// graph), per batch Queue / Collect, Finish (film and statistics).
struct RenderRun {
    yrc_render_scene* s = nullptr;
    yrc_render_request r{};
    yrc_film_pixel* film_out = nullptr;
    uint64_t* bad_out = nullptr;
    yrc_render_stats* stats = nullptr;
    std::chrono::steady_clock::time_point start;
    std::vector<yrc_film_pixel> host_film;
    int64_t pixels = 0;
    int spp = 1;
    int completed_passes = 0;
    unsigned long long sc_host[4] = {0, 0, 0, 0};  // active, next, bad, converged
    unsigned long long cache_host[4] = {0, 0, 0, 0};
    int32_t batch_host = 0;
    int32_t this_batch = 0;
    uint64_t converged = 0;
    uint64_t cache_queries = 0, cache_records = 0;
    uint64_t kernels = 3;  // the set-up (attempt counts, active-pixel list), then the batch graphs
    bool active() const { return sc_host[0] > 0; }
};

yrc_status BeginRender(RenderRun& run) {
    yrc_render_scene* s = run.s;
    cudaSetDevice(s->device);
    run.start = std::chrono::steady_clock::now();
    const yrc_render_settings& st = s->settings;
    run.pixels = static_cast<int64_t>(st.width) * st.height;
    run.spp = std::max(1, st.spp);
    const yrc_render_request& r = run.r;
    if (r.resume_completed_spp < 0 || r.resume_completed_spp > run.spp) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "invalid resume completed spp");
    }
    if (r.resume_film) {
        for (int64_t i = 0; i < run.pixels; ++i) {
            const uint32_t count = r.resume_film[i].samples;
            const bool bad = st.adaptive_enabled ? count > static_cast<uint32_t>(r.resume_completed_spp)
                                                 : count != static_cast<uint32_t>(r.resume_completed_spp);
            if (bad) return Fail(YRC_ERR_INVALID_ARGUMENT, "resume film sample counts do not match resume completed spp");
        }
    }
    if (r.stop_flag && *r.stop_flag) return Fail(YRC_ERR_CANCELLED, "render cancelled");

    yrc_status status = EnsureWork(s, RenderCapacity(s));
    if (status == YRC_OK) status = EnsureCache(s);
    if (status != YRC_OK) return status;
    cudaStream_t stream = s->stream;
    if (r.progress) run.host_film.resize(static_cast<size_t>(run.pixels));  // the callback's copy of the film
    if (r.resume_film) {
        cudaMemcpyAsync(s->film, r.resume_film, sizeof(yrc_film_pixel) * run.pixels, cudaMemcpyHostToDevice, stream);
    } else {
        cudaMemsetAsync(s->film, 0, sizeof(yrc_film_pixel) * run.pixels, stream);
    }
    LaunchFillInt32(s->attempts, run.pixels, run.spp - r.resume_completed_spp, s->sm_count, stream);
    const unsigned long long init_scalars[4] = {0, 0, r.resume_bad_samples, 0};
    cudaMemcpyAsync(s->scalars, init_scalars, sizeof(init_scalars), cudaMemcpyHostToDevice, stream);
    cudaMemsetAsync(s->q.counters, 0, sizeof(unsigned long long) * kCtrCount, stream);
    const int32_t max_batch = r.progress ? 1 : std::min(run.spp, kMaxBatch);
    {
        const DevScene& sc = s->dev;
        BatchArgs b{s->active, s->scalars + 0, s->scalars + 1, s->batch, s->film};
        FilmArgs f{s->attempts, s->scalars + 2, s->scalars + 3, st.adaptive_enabled, st.adaptive_min_spp,
                   st.adaptive_relative_error, st.adaptive_absolute_error, st.adaptive_confidence};
        LaunchActivePixels(sc, b, f, run.pixels, s->sm_count, stream);
        LaunchFinishActive(s->scalars + 0, s->scalars + 1, s->batch, max_batch, s->capacity, stream);
    }
    status = EnsureGraph(s, max_batch);
    if (status != YRC_OK) return status;
    run.completed_passes = r.resume_completed_spp;
    cudaMemcpyAsync(run.sc_host, s->scalars, sizeof(run.sc_host), cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(&run.batch_host, s->batch, sizeof(int32_t), cudaMemcpyDeviceToHost, stream);
    const cudaError_t err = cudaStreamSynchronize(stream);
    if (err != cudaSuccess) return CudaError(err, "render setup");
    run.converged = run.sc_host[3];
    return Ok();
}

// Work before a batch launch and the readback after it, on `stream`.
void QueueBatchPrologue(RenderRun& run, cudaStream_t stream) {
    run.this_batch = run.batch_host;
    cudaMemsetAsync(run.s->scalars + 3, 0, sizeof(unsigned long long), stream);  // recounted by the batch
}
void QueueBatchReadback(RenderRun& run, cudaStream_t stream) {
    yrc_render_scene* s = run.s;
    cudaMemcpyAsync(run.sc_host, s->scalars, sizeof(run.sc_host), cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(&run.batch_host, s->batch, sizeof(int32_t), cudaMemcpyDeviceToHost, stream);
    if (s->cargs.enabled) {
        cudaMemcpyAsync(run.cache_host, s->cargs.counters, sizeof(run.cache_host), cudaMemcpyDeviceToHost, stream);
    }
}
// After the readback completed.
void CollectBatch(RenderRun& run) {
    yrc_render_scene* s = run.s;
    if (s->cargs.enabled) {
        run.cache_queries += run.cache_host[0];
        run.cache_records += std::min<unsigned long long>(
            run.cache_host[2], static_cast<unsigned long long>(std::max(s->cargs.train_records, 0)));
    }
    run.completed_passes += run.this_batch;
    run.converged = run.sc_host[3];
    run.kernels += static_cast<uint64_t>(s->graph_kernels);
}

yrc_status FinishRender(RenderRun& run, double device_seconds) {
    yrc_render_scene* s = run.s;
    cudaStream_t stream = s->stream;
    const int64_t pixels = run.pixels;
    // samples_rendered: summed on the device rather than over the host film.
    cudaError_t err = cudaMemsetAsync(s->q.counters + kCtrSamplesDone, 0, sizeof(unsigned long long), stream);
    if (err == cudaSuccess) {
        LaunchSumSamples(s->film, pixels, s->q.counters + kCtrSamplesDone, s->sm_count, stream);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) {
        err = cudaMemcpyAsync(run.film_out, s->film, sizeof(yrc_film_pixel) * pixels, cudaMemcpyDeviceToHost, stream);
    }
    unsigned long long counters[kCtrCount];
    if (err == cudaSuccess) {
        err = cudaMemcpyAsync(counters, s->q.counters, sizeof(counters), cudaMemcpyDeviceToHost, stream);
    }
    unsigned long long fin[4];
    if (err == cudaSuccess) err = cudaMemcpyAsync(fin, s->scalars, sizeof(fin), cudaMemcpyDeviceToHost, stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(stream);
    if (err != cudaSuccess) return CudaError(err, "render readback");
    const yrc_status status = CheckDeviceError(s->accel);
    if (status != YRC_OK) return status;
    if (run.bad_out) *run.bad_out = fin[2];
    if (run.stats) {
        yrc_render_stats* stats = run.stats;
        std::memset(stats, 0, sizeof(*stats));
        stats->samples_rendered = counters[kCtrSamplesDone];
        stats->converged_pixels = run.converged;
        stats->rays_traced = counters[kCtrStatsBase + 0];
        stats->shadow_rays = counters[kCtrStatsBase + 1];
        stats->occluded_shadow_rays = counters[kCtrStatsBase + 2];
        stats->hits = counters[kCtrStatsBase + 3];
        stats->misses = counters[kCtrStatsBase + 4];
        stats->cache_queries = run.cache_queries;
        stats->cache_records = run.cache_records;
        stats->kernel_launches = run.kernels;
        stats->bad_samples = fin[2];
        stats->bvh_nodes = s->bvh_nodes;
        stats->bvh_max_depth = s->bvh_max_depth;
        stats->threads = 1;
        stats->device_seconds = device_seconds;
        stats->elapsed_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - run.start).count();
    }
    return Ok();
}

}  // namespace
}  // namespace yrc

extern "C" yrc_status yrc_render(yrc_render_scene* s, const yrc_render_request* req, yrc_film_pixel* film_out,
                                 uint64_t* bad_samples_out, yrc_render_stats* stats) {
    using namespace yrc;
    if (!s || !film_out) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_render: null argument");
    std::lock_guard<std::mutex> lock(s->mutex);
    RenderRun run;
    run.s = s;
    if (req) run.r = *req;
    run.film_out = film_out;
    run.bad_out = bad_samples_out;
    run.stats = stats;
    yrc_status status = BeginRender(run);
    if (status != YRC_OK) return status;
    const yrc_render_request& r = run.r;
    cudaStream_t stream = s->stream;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, stream);
    while (run.active()) {
        if (r.stop_flag && *r.stop_flag) return Fail(YRC_ERR_CANCELLED, "render cancelled");
        QueueBatchPrologue(run, stream);
        cudaError_t err = cudaGraphLaunch(s->graph, stream);
        if (err != cudaSuccess) return CudaError(err, "batch launch");
        QueueBatchReadback(run, stream);
        err = cudaStreamSynchronize(stream);
        if (err != cudaSuccess) return CudaError(err, "batch");
        CollectBatch(run);
        if (r.progress) {
            const int64_t pixels = run.pixels;
            cudaMemcpy(run.host_film.data(), s->film, sizeof(yrc_film_pixel) * pixels, cudaMemcpyDeviceToHost);
            uint64_t done = 0;
            for (int64_t i = 0; i < pixels; ++i) done += run.host_film[static_cast<size_t>(i)].samples;
            unsigned long long counters[kCtrCount];
            cudaMemcpy(counters, s->q.counters, sizeof(counters), cudaMemcpyDeviceToHost);
            yrc_render_progress prog{};
            prog.completed_spp = std::min(run.completed_passes, run.spp);
            prog.target_spp = run.spp;
            prog.completed_samples = done;
            prog.target_samples = static_cast<uint64_t>(run.spp) * static_cast<uint64_t>(pixels);
            prog.active_pixels = run.sc_host[0];
            prog.converged_pixels = run.sc_host[3];
            prog.rays_traced = counters[kCtrStatsBase + 0];
            prog.elapsed_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - run.start).count();
            char msg[512] = {0};
            if (r.progress(&prog, run.host_film.data(), run.sc_host[2], r.user, msg, sizeof(msg))) {
                return Fail(YRC_ERR_CANCELLED, msg[0] ? msg : "render cancelled by progress callback");
            }
        }
    }
    cudaEventRecord(e1, stream);
    cudaEventSynchronize(e1);
    float device_ms = 0.0f;
    cudaEventElapsedTime(&device_ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return FinishRender(run, device_ms / 1e3);
}

namespace yrc {
namespace {

// Pooled batch of several scenes: per bounce, the extend rays of every
// scene go through ONE persistent traversal launch and the shadow rays
// through ONE transmittance (or any-hit) launch, the lanes taking rays from
// all scenes' queues (TracePool / ShadowPool); each scene's generate,
// shading, next-event and film stages run as parallel branches of the same
// graph. Holds the instantiated graph and the device job tables it reads.
struct PooledBatch {
    cudaGraphExec_t exec = nullptr;
    DeviceArena mem;
    std::vector<cudaEvent_t> events;
    void Release() {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        mem.Release();
        mem.err = cudaSuccess;
        for (cudaEvent_t e : events) cudaEventDestroy(e);
        events.clear();
    }
    ~PooledBatch() { Release(); }
};

// The scene's queues at bounce `depth` (the extend queues alternate).
Queues QueuesAt(const yrc_render_scene* s, int depth) {
    Queues q = s->q;
    if (depth & 1) {
        std::swap(q.ray_in, q.ray_out);
        std::swap(q.path_in, q.path_out);
    }
    return q;
}

// Pool group of a scene: scenes in one pooled launch share the BVH kind
// and the traversal stack class.
int PoolGroup(const yrc_render_scene* s) {
    return (s->dev.accel.two_level ? 2 : 0) + (s->dev.accel.stack_limit > 64 ? 1 : 0);
}

// Makes `side` wait for the work recorded on `main` so far (fork), or
// `main` wait for each of `side` (join); inside a capture these become the
// graph's dependencies.
cudaError_t Fork(cudaStream_t main, const std::vector<cudaStream_t>& side, PooledBatch& pb) {
    cudaEvent_t e = nullptr;
    cudaError_t err = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    if (err != cudaSuccess) return err;
    pb.events.push_back(e);
    err = cudaEventRecord(e, main);
    for (size_t i = 0; i < side.size() && err == cudaSuccess; ++i) err = cudaStreamWaitEvent(side[i], e, 0);
    return err;
}
cudaError_t Join(cudaStream_t main, const std::vector<cudaStream_t>& side, PooledBatch& pb) {
    cudaError_t err = cudaSuccess;
    for (size_t i = 0; i < side.size() && err == cudaSuccess; ++i) {
        cudaEvent_t e = nullptr;
        err = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        if (err != cudaSuccess) break;
        pb.events.push_back(e);
        err = cudaEventRecord(e, side[i]);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(main, e, 0);
    }
    return err;
}

struct PoolLaunch {
    int kind;  // 0 extend (closest hit), 1 shadow transmittance, 2 shadow any hit
    int group;
    size_t first;  // into the trace or shadow job table
    int32_t count;
    int64_t capacity;
};

// Records the pooled batch of `ss` (every scene set up by BeginRender) on
// `main` under stream capture and instantiates it.
yrc_status CapturePooledBatch(const std::vector<yrc_render_scene*>& ss, cudaStream_t main, PooledBatch& pb) {
    pb.Release();
    int max_depth = 0;
    for (const yrc_render_scene* s : ss) max_depth = std::max(max_depth, s->dev.max_depth);
    std::vector<TraceArgs> trace_jobs;
    std::vector<ShadowArgs> shadow_jobs;
    std::vector<std::vector<PoolLaunch>> launches(static_cast<size_t>(max_depth));
    for (int d = 0; d < max_depth; ++d) {
        for (int kind = 0; kind < 3; ++kind) {
            for (int g = 0; g < 4; ++g) {
                PoolLaunch L{kind, g, kind == 1 ? shadow_jobs.size() : trace_jobs.size(), 0, 0};
                for (yrc_render_scene* s : ss) {
                    if (d >= s->dev.max_depth || PoolGroup(s) != g) continue;
                    const Queues q = QueuesAt(s, d);
                    int* error = AccelErrorWord(s->accel);
                    if (kind == 0) {
                        trace_jobs.push_back(ExtendTraceArgs(s, q));
                        L.capacity += s->capacity;
                    } else if (kind == 1 && ShadowKindOf(s) == ShadowKind::kTransmittance) {
                        shadow_jobs.push_back(TransmittanceArgs(s, q, s->capacity, error));
                        L.capacity += 2 * s->capacity;
                    } else if (kind == 2 && ShadowKindOf(s) == ShadowKind::kAnyHit) {
                        trace_jobs.push_back(AnyHitShadowArgs(q, s->dev.accel, s->capacity, error));
                        L.capacity += 2 * s->capacity;
                    } else {
                        continue;
                    }
                    ++L.count;
                }
                if (L.count > 0) launches[static_cast<size_t>(d)].push_back(L);
            }
        }
    }
    // Per bounce, the shade jobs of the scenes that reach it.
    std::vector<ShadeJob> shade_jobs;
    std::vector<size_t> shade_first(static_cast<size_t>(max_depth) + 1, 0);
    std::vector<int64_t> shade_capacity(static_cast<size_t>(max_depth), 0);
    for (int d = 0; d < max_depth; ++d) {
        shade_first[static_cast<size_t>(d)] = shade_jobs.size();
        for (yrc_render_scene* s : ss) {
            if (d >= s->dev.max_depth) continue;
            ShadeJob j{};
            j.sc = s->dev;
            j.ps = s->ps;
            j.q = QueuesAt(s, d);
            j.cache = s->cargs;
            j.depth = d;
            shade_jobs.push_back(j);
            shade_capacity[static_cast<size_t>(d)] += s->capacity;
        }
    }
    shade_first[static_cast<size_t>(max_depth)] = shade_jobs.size();
    size_t n_launches = 0;
    for (const auto& v : launches) n_launches += v.size();
    const ShadeJob* d_shade = pb.mem.Upload(shade_jobs);
    const TraceArgs* d_trace = pb.mem.Upload(trace_jobs);
    const ShadowArgs* d_shadow = pb.mem.Upload(shadow_jobs);
    unsigned long long* counters = pb.mem.Alloc<unsigned long long>(n_launches);
    if (pb.mem.err != cudaSuccess) return CudaError(pb.mem.err, "pooled batch tables");
    const int sm_count = ss.front()->sm_count;

    std::vector<cudaStream_t> side;
    for (yrc_render_scene* s : ss) side.push_back(s->stream);
    cudaError_t err = cudaStreamBeginCapture(main, cudaStreamCaptureModeThreadLocal);
    if (err != cudaSuccess) return CudaError(err, "pooled batch capture");
    yrc_status status = Ok();
    auto run = [&](cudaError_t e, const char* what) {
        if (status == YRC_OK && e != cudaSuccess) status = CudaError(e, what);
        return status == YRC_OK;
    };
    auto per_scene = [&](auto&& body) {
        if (!run(Fork(main, side, pb), "pooled batch fork")) return;
        for (size_t i = 0; i < ss.size() && status == YRC_OK; ++i) status = body(ss[i]);
        run(Join(main, side, pb), "pooled batch join");
    };
    per_scene([&](yrc_render_scene* s) { return BatchPrologue(s, s->stream); });
    size_t k = 0;
    auto pooled = [&](int d, bool shadow) {
        for (const PoolLaunch& L : launches[static_cast<size_t>(d)]) {
            if ((L.kind != 0) != shadow || status != YRC_OK) continue;
            unsigned long long* counter = counters + k++;
            if (!run(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), main), "pooled counter")) return;
            const bool two = (L.group & 2) != 0, deep = (L.group & 1) != 0;
            cudaError_t e;
            if (L.kind == 1) {
                e = LaunchPooledShadowTransmittance(ShadowPool{d_shadow + L.first, L.count, L.capacity, counter}, two,
                                                    deep, main, sm_count);
            } else {
                e = LaunchPooledTrace(TracePool{d_trace + L.first, L.count, L.capacity, counter}, L.kind == 2, two,
                                      deep, main, sm_count);
            }
            run(e, L.kind == 0 ? "pooled extend trace" : "pooled shadow trace");
        }
    };
    for (int d = 0; d < max_depth && status == YRC_OK; ++d) {
        per_scene([&](yrc_render_scene* s) {
            if (d < s->dev.max_depth) LaunchResetCounters(QueuesAt(s, d), s->stream);
            return Ok();
        });
        pooled(d, false);
        per_scene([&](yrc_render_scene* s) {
            if (d < s->dev.max_depth) BounceShadeSort(s, QueuesAt(s, d), d, s->stream);
            return Ok();
        });
        const size_t first = shade_first[static_cast<size_t>(d)];
        LaunchPooledShade(d_shade + first, static_cast<int>(shade_first[static_cast<size_t>(d) + 1] - first),
                          shade_capacity[static_cast<size_t>(d)], sm_count, main);
        run(cudaGetLastError(), "pooled shade");
        per_scene([&](yrc_render_scene* s) {
            return d < s->dev.max_depth ? BounceSubsurface(s, QueuesAt(s, d), d, s->stream) : Ok();
        });
        pooled(d, true);
        per_scene([&](yrc_render_scene* s) {
            if (d >= s->dev.max_depth) return Ok();
            const Queues q = QueuesAt(s, d);
            int* error = AccelErrorWord(s->accel);
            const ShadowKind kind = ShadowKindOf(s);
            if (kind == ShadowKind::kExact) {
                const cudaError_t e = ShadowStage(s, q, s->capacity, error, s->stream);
                if (e != cudaSuccess) return CudaError(e, "shadow trace");
            } else if (kind == ShadowKind::kTransmittance) {
                ShadowOverflow(s, q, s->capacity, error, s->stream);
            }
            return BounceResolve(s, q, d, s->stream);
        });
    }
    per_scene([&](yrc_render_scene* s) { return BatchEpilogue(s, s->graph_max_batch, s->stream); });
    cudaGraph_t graph = nullptr;
    err = cudaStreamEndCapture(main, &graph);
    if (status == YRC_OK && err != cudaSuccess) status = CudaError(err, "pooled batch capture");
    if (status == YRC_OK) {
        err = cudaGraphInstantiate(&pb.exec, graph, 0);
        if (err != cudaSuccess) status = CudaError(err, "pooled batch instantiate");
    }
    if (graph) cudaGraphDestroy(graph);
    return status;
}

// yrc_render_many / yrc_render_pooled: every step launches one graph for
// the scenes still rendering, rebuilt when a scene finishes.
yrc_status RenderMany(yrc_render_scene* const* scenes, int32_t count, const yrc_render_request* requests,
                      yrc_film_pixel* const* films_out, uint64_t* bad_samples_out, yrc_render_stats* stats,
                      double* device_seconds, bool pooled, const char* name) {
    if (count < 0 || (count > 0 && (!scenes || !films_out))) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, std::string(name) + ": bad argument");
    }
    if (count == 0) return Ok();
    if (pooled && count > kMaxPoolJobs) {
        return Fail(YRC_ERR_INVALID_ARGUMENT,
                    std::string(name) + ": at most " + std::to_string(kMaxPoolJobs) + " scenes per call");
    }
    // One lock per scene, taken in address order; every scene on one device.
    std::vector<yrc_render_scene*> order(scenes, scenes + count);
    for (int32_t i = 0; i < count; ++i) {
        if (!order[static_cast<size_t>(i)] || !films_out[i]) {
            return Fail(YRC_ERR_INVALID_ARGUMENT, std::string(name) + ": null scene or film");
        }
        for (int32_t j = 0; j < i; ++j) {
            if (order[static_cast<size_t>(j)] == order[static_cast<size_t>(i)]) {
                return Fail(YRC_ERR_INVALID_ARGUMENT, std::string(name) + ": a scene appears twice");
            }
        }
        if (order[static_cast<size_t>(i)]->device != order[0]->device) {
            return Fail(YRC_ERR_INVALID_ARGUMENT, std::string(name) + ": scenes on different devices");
        }
        if (requests && requests[i].progress) {
            return Fail(YRC_ERR_INVALID_ARGUMENT, std::string(name) + ": progress callbacks are not supported");
        }
        for (int32_t j = 0; j < i; ++j) {
            if (scenes[i]->cache && scenes[i]->cache == scenes[j]->cache) {
                return Fail(YRC_ERR_INVALID_ARGUMENT, std::string(name) + ": two scenes share a radiance cache");
            }
        }
    }
    std::sort(order.begin(), order.end());
    std::vector<std::unique_lock<std::mutex>> locks;
    for (yrc_render_scene* s : order) locks.emplace_back(s->mutex);
    cudaSetDevice(scenes[0]->device);
    std::vector<RenderRun> runs(static_cast<size_t>(count));
    for (int32_t i = 0; i < count; ++i) {
        RenderRun& run = runs[static_cast<size_t>(i)];
        run.s = scenes[i];
        if (requests) run.r = requests[i];
        run.film_out = films_out[i];
        run.bad_out = bad_samples_out ? bad_samples_out + i : nullptr;
        run.stats = stats ? stats + i : nullptr;
        const yrc_status status = BeginRender(run);
        if (status != YRC_OK) return status;
    }
    cudaStream_t stream = nullptr;
    cudaError_t err = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    if (err != cudaSuccess) return CudaError(err, "render stream");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, stream);
    cudaGraphExec_t exec = nullptr;  // child-graph form
    PooledBatch pb;                  // pooled form
    std::vector<int32_t> members;
    yrc_status status = YRC_OK;
    for (;;) {
        std::vector<int32_t> live;
        for (int32_t i = 0; i < count; ++i) {
            if (runs[static_cast<size_t>(i)].active()) live.push_back(i);
        }
        if (live.empty()) break;
        bool cancelled = false;
        for (int32_t i : live) {
            const yrc_render_request& r = runs[static_cast<size_t>(i)].r;
            if (r.stop_flag && *r.stop_flag) cancelled = true;
        }
        if (cancelled) {
            status = Fail(YRC_ERR_CANCELLED, "render cancelled");
            break;
        }
        if (live != members) {
            if (pooled) {
                std::vector<yrc_render_scene*> ss;
                for (int32_t i : live) ss.push_back(runs[static_cast<size_t>(i)].s);
                status = CapturePooledBatch(ss, stream, pb);
                if (status != YRC_OK) break;
            } else {
                if (exec) cudaGraphExecDestroy(exec);
                exec = nullptr;
                cudaGraph_t combined = nullptr;
                err = cudaGraphCreate(&combined, 0);
                for (int32_t i : live) {
                    cudaGraphNode_t node = nullptr;
                    if (err == cudaSuccess) {
                        err = cudaGraphAddChildGraphNode(&node, combined, nullptr, 0,
                                                         runs[static_cast<size_t>(i)].s->graph_template);
                    }
                }
                if (err == cudaSuccess) err = cudaGraphInstantiate(&exec, combined, 0);
                if (combined) cudaGraphDestroy(combined);
                if (err != cudaSuccess) {
                    status = CudaError(err, "combined batch graph");
                    break;
                }
            }
            members = live;
        }
        for (int32_t i : live) QueueBatchPrologue(runs[static_cast<size_t>(i)], stream);
        err = cudaGraphLaunch(pooled ? pb.exec : exec, stream);
        if (err != cudaSuccess) {
            status = CudaError(err, "combined batch launch");
            break;
        }
        for (int32_t i : live) QueueBatchReadback(runs[static_cast<size_t>(i)], stream);
        err = cudaStreamSynchronize(stream);
        if (err != cudaSuccess) {
            status = CudaError(err, "combined batch");
            break;
        }
        for (int32_t i : live) CollectBatch(runs[static_cast<size_t>(i)]);
    }
    cudaEventRecord(e1, stream);
    cudaEventSynchronize(e1);
    float device_ms = 0.0f;
    cudaEventElapsedTime(&device_ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (exec) cudaGraphExecDestroy(exec);
    pb.Release();
    cudaStreamDestroy(stream);
    if (status != YRC_OK) return status;
    if (device_seconds) *device_seconds = device_ms / 1e3;
    for (int32_t i = 0; i < count && status == YRC_OK; ++i) {
        status = FinishRender(runs[static_cast<size_t>(i)], device_ms / 1e3);
    }
    return status;
}

}  // namespace
}  // namespace yrc

extern "C" yrc_status yrc_render_many(yrc_render_scene* const* scenes, int32_t count,
                                      const yrc_render_request* requests, yrc_film_pixel* const* films_out,
                                      uint64_t* bad_samples_out, yrc_render_stats* stats, double* device_seconds) {
    return yrc::RenderMany(scenes, count, requests, films_out, bad_samples_out, stats, device_seconds, false,
                           "yrc_render_many");
}

extern "C" yrc_status yrc_render_pooled(yrc_render_scene* const* scenes, int32_t count,
                                        const yrc_render_request* requests, yrc_film_pixel* const* films_out,
                                        uint64_t* bad_samples_out, yrc_render_stats* stats, double* device_seconds) {
    return yrc::RenderMany(scenes, count, requests, films_out, bad_samples_out, stats, device_seconds, true,
                           "yrc_render_pooled");
}

extern "C" yrc_status yrc_render_scene_set_capacity(yrc_render_scene* s, int64_t capacity) {
    using namespace yrc;
    if (!s || capacity < 0) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_render_scene_set_capacity: bad argument");
    std::lock_guard<std::mutex> lock(s->mutex);
    s->capacity_choice = capacity;
    return Ok();
}

extern "C" int64_t yrc_render_scene_capacity(const yrc_render_scene* s) {
    return s ? yrc::RenderCapacity(s) : 0;
}

extern "C" yrc_status yrc_render_autotune(yrc_render_scene* s, int32_t flags, yrc_render_tuning* result) {
    using namespace yrc;
    if (!s || (flags & ~(YRC_TUNE_CAPACITY | YRC_TUNE_TRACE_SHAPE)) != 0) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_render_autotune: bad argument");
    }
    std::lock_guard<std::mutex> lock(s->mutex);
    cudaSetDevice(s->device);
    const int64_t pixels = static_cast<int64_t>(s->settings.width) * s->settings.height;
    const int spp = std::max(1, s->settings.spp);
    const int most_passes = std::min(spp, kMaxBatch);
    // Candidate capacities: whole passes of the image, 2^17 .. 2^23 paths
    // (the smallest and largest whole-pass counts always included).
    std::vector<int64_t> caps;
    for (int k = 1; k <= most_passes; k *= 2) {
        const int64_t c = pixels * k;
        if ((c >= (int64_t{1} << 17) || k * 2 > most_passes) && (c <= (int64_t{1} << 23) || k == 1)) caps.push_back(c);
    }
    if (caps.empty()) caps.push_back(pixels);
    // Every probe renders the same passes: two batches of the largest candidate.
    const int32_t passes =
        static_cast<int32_t>(std::min<int64_t>(spp, std::max<int64_t>(1, 2 * caps.back() / pixels)));
    // Probes run without the radiance cache, so that they do not train it.
    yrc_nrc* cache = s->cache;
    s->cache = nullptr;
    DropGraph(s);
    EnsureCache(s);
    const int64_t saved_choice = s->capacity_choice;
    const int saved_shape = yrc_accel_get_trace_shape(s->accel, 0);
    const int saved_any_shape = yrc_accel_get_trace_shape(s->accel, 1);
    int tried = 0;
    double best = 0.0;
    int64_t best_cap = RenderCapacity(s);
    int best_shape = saved_shape;
    yrc_status status = YRC_OK;
    // One launch shape for the extend (closest-hit) and shadow (any-hit and
    // transmittance) traversals.
    auto time_config = [&](int64_t cap, int shape, double* sec) -> yrc_status {
        s->capacity_choice = cap;
        yrc_accel_set_trace_shape(s->accel, 0, shape);
        yrc_accel_set_trace_shape(s->accel, 1, shape);
        DropGraph(s);
        double first = 0.0;
        yrc_status st = ProbeRender(s, passes, &first);  // allocation, graph capture, warm-up
        if (st == YRC_OK) st = ProbeRender(s, passes, sec);
        ++tried;
        return st;
    };
    if (flags & YRC_TUNE_CAPACITY) {
        for (const int64_t cap : caps) {
            double sec = 0.0;
            status = time_config(cap, saved_shape, &sec);
            if (status != YRC_OK) break;
            if (best == 0.0 || sec < best) {
                best = sec;
                best_cap = cap;
            }
        }
    }
    // Traversal launch shapes of the extend stage.
    if (status == YRC_OK && (flags & YRC_TUNE_TRACE_SHAPE)) {
        for (int shape = 0; shape < YRC_TRACE_SHAPES; ++shape) {
            double sec = 0.0;
            status = time_config(best_cap, shape, &sec);
            if (status != YRC_OK) break;
            if (best == 0.0 || sec < best) {
                best = sec;
                best_shape = shape;
            }
        }
    }
    if (status == YRC_OK && best == 0.0) {  // nothing tuned: time the current configuration
        status = time_config(best_cap, best_shape, &best);
    }
    s->capacity_choice = status == YRC_OK ? best_cap : saved_choice;
    yrc_accel_set_trace_shape(s->accel, 0, status == YRC_OK ? best_shape : saved_shape);
    yrc_accel_set_trace_shape(s->accel, 1, status == YRC_OK ? best_shape : saved_any_shape);
    DropGraph(s);
    s->cache = cache;
    s->cache_capacity = 0;  // re-allocated for the chosen capacity on the next render
    if (status != YRC_OK) return status;
    if (result) {
        result->capacity = best_cap;
        result->trace_shape = best_shape;
        result->candidates = tried;
        result->seconds_per_sample = best / (static_cast<double>(pixels) * passes);
    }
    return Ok();
}

extern "C" yrc_status yrc_render_scene_set_tuning(yrc_render_scene* s, const yrc_render_tuning* tuning) {
    using namespace yrc;
    if (!s || !tuning || tuning->capacity < 0 || tuning->trace_shape < 0 || tuning->trace_shape >= YRC_TRACE_SHAPES) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_render_scene_set_tuning: bad argument");
    }
    std::lock_guard<std::mutex> lock(s->mutex);
    cudaSetDevice(s->device);
    s->capacity_choice = tuning->capacity;
    yrc_status st = yrc_accel_set_trace_shape(s->accel, 0, tuning->trace_shape);
    if (st == YRC_OK) st = yrc_accel_set_trace_shape(s->accel, 1, tuning->trace_shape);
    if (st != YRC_OK) return st;
    DropGraph(s);
    return Ok();
}

// TraceShadowVisibility (src/integrators/path_direct_lighting.cpp:23-113) for
// caller rays, through the scene's own shadow stage: the single-pass
// transmittance kernel with its exact-loop overflow, the exact loop for
// scenes with cut-outs, or the any-hit kernel for scenes without surfaces
// that pass light.
extern "C" yrc_status yrc_render_scene_shadow_eval(yrc_render_scene* s, const yrc_ray* rays, int64_t n,
                                                   float* transmittance) {
    using namespace yrc;
    if (!s || n < 0 || n > (int64_t{1} << 30) || (n > 0 && (!rays || !transmittance))) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_render_scene_shadow_eval: bad argument");
    }
    if (n == 0) return Ok();
    std::lock_guard<std::mutex> lock(s->mutex);
    cudaSetDevice(s->device);
    const size_t un = static_cast<size_t>(n);
    const DevScene& sc = s->dev;
    DeviceArena a;
    Queues q{};
    q.shadow_ray = a.Upload(reinterpret_cast<const float4*>(rays), 2 * un);
    std::vector<int32_t> slot(un);
    for (size_t i = 0; i < un; ++i) slot[i] = static_cast<int32_t>(i);
    q.shadow_slot = a.Upload(slot);
    q.shadow_overflow = a.Alloc<int32_t>(un);
    q.shadow_occluded = a.Alloc<uint8_t>(un);
    q.counters = a.Alloc<unsigned long long>(kCtrCount);
    float4* tr = a.Alloc<float4>(un);
    std::vector<unsigned long long> counters(kCtrCount, 0);
    counters[kCtrShadow] = static_cast<unsigned long long>(n);
    cudaError_t err = a.err;
    if (err == cudaSuccess) {
        err = cudaMemcpy(q.counters, counters.data(), sizeof(unsigned long long) * kCtrCount, cudaMemcpyHostToDevice);
    }
    int* error = AccelErrorWord(s->accel);
    const cudaStream_t st = nullptr;
    const bool opaque = !sc.exact_shadows && !sc.any_transparent;
    if (err == cudaSuccess) {
        if (sc.exact_shadows) {
            LaunchShadowExact(sc, q, tr, q.counters + kCtrStatsBase + 2, n, s->sm_count, error, st);
            err = cudaGetLastError();
        } else if (sc.any_transparent) {
            ShadowArgs sa{};
            sa.accel = sc.accel;
            sa.rays = q.shadow_ray;
            sa.count_ptr = q.counters + kCtrShadow;
            sa.capacity = n;
            sa.out_index = q.shadow_slot;
            sa.transmittance = tr;
            sa.tri_prim = sc.tri_prim;
            sa.prim_material = sc.prim_material;
            sa.sphere_material = sc.sphere_material;
            sa.materials = sc.materials;
            sa.tri_clear = sc.tri_clear;
            sa.sphere_clear = sc.sphere_clear;
            sa.counter = q.counters + kCtrShadowTrace;
            sa.occluded_count = q.counters + kCtrStatsBase + 2;
            sa.overflow = q.shadow_overflow;
            sa.overflow_count = q.counters + kCtrShadowOverflow;
            sa.error = error;
            sa.leaf_batch = LeafBatchOfShape(TraceShapeOf(s->accel, 1));
            err = LaunchShadowTransmittance(sa, st, s->sm_count);
            if (err == cudaSuccess) {
                LaunchShadowExact(sc, q, tr, q.counters + kCtrStatsBase + 2, n, s->sm_count, error, st,
                                  q.shadow_overflow);
                err = cudaGetLastError();
            }
        } else {
            TraceArgs sh{};
            sh.accel = sc.accel;
            sh.rays = q.shadow_ray;
            sh.count = n;
            sh.count_ptr = q.counters + kCtrShadow;
            sh.occluded = q.shadow_occluded;
            sh.out_index = q.shadow_slot;
            sh.counter = q.counters + kCtrShadowTrace;
            sh.occluded_count = q.counters + kCtrStatsBase + 2;
            sh.error = error;
            err = LaunchTrace(sh, true, false, TraceShapeOf(s->accel, 1), st, s->sm_count);
        }
    }
    if (err == cudaSuccess) err = cudaDeviceSynchronize();
    if (err == cudaSuccess && opaque) {
        std::vector<uint8_t> occ(un);
        err = cudaMemcpy(occ.data(), q.shadow_occluded, un, cudaMemcpyDeviceToHost);
        for (size_t i = 0; err == cudaSuccess && i < un; ++i) {
            const float v = occ[i] ? 0.0f : 1.0f;
            for (int c = 0; c < 4; ++c) transmittance[4 * i + c] = v;
        }
    } else if (err == cudaSuccess) {
        err = cudaMemcpy(transmittance, tr, sizeof(float4) * un, cudaMemcpyDeviceToHost);
    }
    a.Release();
    if (err != cudaSuccess) return CudaError(err, "yrc_render_scene_shadow_eval");
    return CheckDeviceError(s->accel);
}

// A new camera and sampler seed for a resident scene (a camera path, frames
// of an animation): one small copy into the scene's view record. The scene's
// working memory and captured batch stay as they are, so the next render
// pays neither allocation nor capture. No counterpart in the reference (its
// RenderJob is immutable once prepared).
extern "C" yrc_status yrc_render_scene_set_view(yrc_render_scene* s, const yrc_camera* camera, uint64_t seed) {
    using namespace yrc;
    if (!s || !camera) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_render_scene_set_view: bad argument");
    std::lock_guard<std::mutex> lock(s->mutex);
    cudaSetDevice(s->device);
    const DevView v = MakeView(*camera, seed);
    const cudaError_t err = cudaMemcpy(s->view, &v, sizeof(v), cudaMemcpyHostToDevice);
    if (err != cudaSuccess) return CudaError(err, "yrc_render_scene_set_view");
    s->settings.seed = seed;
    return Ok();
}
