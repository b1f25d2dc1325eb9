// Wavefront path-tracing stages: the bounce loop of IntegratePathSample
// (src/integrators/path_integrator.cpp:23-197) split into
//   generate  camera rays + per-path sampler/RNG state   (cpu_path_tracer.cpp:120-150)
//   extend    closest-hit traversal of the ray queue     (trace_kernels.cu)
//   shade     surface resolve, emission + MIS, next-event estimation samples,
//             BSDF sampling, Russian roulette             (path_integrator.cpp:46-192)
//   shadow    any-hit or transparent-shadow traversal    (path_direct_lighting.cpp:23-113)
//   resolve   adds the visible next-event contributions  (path_direct_lighting.cpp:170-283)
//   film      in-order Film::AddSample per pixel          (film.cpp:160-183)
// The bounce depth is a launch parameter (every path in flight is at the same
// depth), queue sizes live on the device so a whole batch can be replayed as
// one CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>

#include "bsdf.cuh"
#include "bssrdf.cuh"
#include "render_kernels.hpp"
#include "render_types.hpp"
#include "sampler.cuh"
#include "shading.cuh"
#include "traversal.cuh"

namespace yrc {
namespace {

constexpr float kMinShadowBias = 1.0e-4f;
constexpr float kShadowBiasScale = 1.0e-5f;
constexpr float kMaxShadowBiasFraction = 1.0e-2f;

__device__ __forceinline__ float MaxAbs(V3 p) { return fmaxf(fabsf(p.x), fmaxf(fabsf(p.y), fabsf(p.z))); }

// SurfaceBias / ShadowBias (src/integrators/path_integrator_common.cpp:129-138).
__device__ __forceinline__ float SurfaceBias(V3 p) { return fmaxf(kMinShadowBias, MaxAbs(p) * kShadowBiasScale); }
__device__ __forceinline__ float ShadowBias(V3 o, V3 t, float dist) {
    const float scaled = fmaxf(MaxAbs(o), MaxAbs(t)) * kShadowBiasScale;
    return fminf(fmaxf(kMinShadowBias, scaled), dist * kMaxShadowBiasFraction);
}

__device__ __forceinline__ V3 F4(const float4& v) { return V3{v.x, v.y, v.z}; }
__device__ __forceinline__ float4 ToF4(V3 v, float w = 0.0f) { return make_float4(v.x, v.y, v.z, w); }

// Warp-aggregated append to a device queue; returns this lane's slot. The
// lanes that append to the same queue are aggregated together (in a pooled
// launch the lanes of a warp may serve different jobs' queues).
__device__ __forceinline__ unsigned long long QueueAppend(unsigned long long* counter) {
    const unsigned mask = __match_any_sync(__activemask(), reinterpret_cast<unsigned long long>(counter));
    const int leader = __ffs(mask) - 1;
    const unsigned lane = threadIdx.x & 31u;
    unsigned long long base = 0;
    if (static_cast<int>(lane) == leader) base = atomicAdd(counter, static_cast<unsigned long long>(__popc(mask)));
    base = __shfl_sync(mask, base, leader);
    return base + __popc(mask & ((1u << lane) - 1u));
}

__device__ __forceinline__ void CountStat(unsigned long long* counters, int which) {
    const unsigned mask = __match_any_sync(__activemask(), reinterpret_cast<unsigned long long>(counters));
    if ((threadIdx.x & 31u) == static_cast<unsigned>(__ffs(mask) - 1)) {
        atomicAdd(counters + kCtrStatsBase + which, static_cast<unsigned long long>(__popc(mask)));
    }
}

enum StatIndex { kStatRays = 0, kStatShadow = 1, kStatOccluded = 2, kStatHits = 3, kStatMisses = 4 };

// PerspectiveDirection (src/scene/camera.cpp:9-16); tan(fov/2) comes from the host.
__device__ inline V3 CameraDirection(const DevScene& sc, float fx, float fy) {
    const float w = static_cast<float>(sc.width < 1 ? 1 : sc.width);
    const float h = static_cast<float>(sc.height < 1 ? 1 : sc.height);
    const float aspect = w / h;
    const DevView& v = *sc.view;
    const float sx = (2.0f * fx / w - 1.0f) * aspect * v.cam_half_height;
    const float sy = (1.0f - 2.0f * fy / h) * v.cam_half_height;
    return Normalize(Ld3(v.cam_forward) + Ld3(v.cam_right) * sx + Ld3(v.cam_up) * sy);
}

}  // namespace

// ------------------------------------------------------------------ generate

// Radiance cache: 1 in `train_one_in` paths (by a hash of pixel and sample)
// takes a training slot while slots last; the others may end at the cache.
__device__ __forceinline__ uint32_t CacheHash(uint32_t a, uint32_t b) {
    uint32_t h = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u) * 0x85EBCA77u;
    h ^= h >> 15;
    h *= 0x2C1B3C6Du;
    h ^= h >> 12;
    return h;
}

__global__ void GenerateKernel(DevScene sc, PathState ps, Queues q, BatchArgs b, CacheArgs cache) {
    const int64_t n_active = static_cast<int64_t>(*b.active_count);
    const int32_t batch = *b.batch;
    const int64_t total = n_active * batch;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t p = i % n_active;
        const int32_t j = static_cast<int32_t>(i / n_active);
        const int32_t pixel = b.active[p];
        const int x = pixel % sc.width, y = pixel / sc.width;
        const int32_t sample = static_cast<int32_t>(b.film[pixel].samples) + j;
        PixelSampler smp;
        smp.Init(sc.sampler, sc.view->seed, x, y, sample, sc.spp);
        float sx, sy;
        smp.Sample2D(kDimPixel, 0, sx, sy);
        const float fx = static_cast<float>(x) + sx;
        const float fy = static_cast<float>(y) + sy;
        const V3 d = CameraDirection(sc, fx, fy);
        Pcg32 rng;
        rng.Seed(SeedForPixelSample(sc.view->seed, x, y, sample) ^ kDefaultSeed);
        ps.pixel[i] = pixel;
        ps.sample[i] = sample;
        ps.throughput[i] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
        ps.radiance[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        ps.flags[i] = 0;
        ps.rng_state[i] = rng.state;
        ps.rng_inc[i] = rng.inc;
        ps.aov_albedo[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        ps.aov_normal[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        ps.nee[3 * i] = ps.nee[3 * i + 1] = ps.nee[3 * i + 2] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        q.ray_in[2 * i] = make_float4(sc.view->cam_origin[0], sc.view->cam_origin[1], sc.view->cam_origin[2], 1.0e-5f);
        q.ray_in[2 * i + 1] = make_float4(d.x, d.y, d.z, __int_as_float(0x7f800000));
        q.path_in[i] = static_cast<int32_t>(i);
        if (cache.enabled) {
            int32_t slot = -1;
            if (CacheHash(static_cast<uint32_t>(pixel), static_cast<uint32_t>(sample)) %
                    static_cast<uint32_t>(cache.train_one_in) == 0) {
                const unsigned long long k = atomicAdd(cache.counters + 1, 1ull);
                if (k < static_cast<unsigned long long>(cache.train_paths)) {
                    slot = static_cast<int32_t>(k);
                    cache.slot_path[slot] = static_cast<int32_t>(i);
                    cache.slot_len[slot] = 0;
                }
            }
            cache.train_slot[i] = slot;
            ps.spread[i] = make_float2(0.0f, 0.0f);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) q.counters[kCtrIn] = static_cast<unsigned long long>(total);
}

// Resets the per-bounce queue counters (so the bounce loop can be captured).
__global__ void ResetCountersKernel(Queues q) {
    if (threadIdx.x == 0) {
        q.counters[kCtrOut] = 0;
        q.counters[kCtrShadow] = 0;
        q.counters[kCtrNee] = 0;
        q.counters[kCtrTrace] = 0;
        q.counters[kCtrShadowTrace] = 0;
        q.counters[kCtrShadowOverflow] = 0;
        q.counters[kCtrProbe] = 0;
        q.counters[kCtrDefer] = 0;
        q.counters[kCtrDefer2] = 0;
        for (int c = 0; c < kShadeClasses; ++c) {
            q.counters[kCtrClass0 + c] = 0;
            q.counters[kCtrCursor0 + c] = 0;
        }
    }
}

// Makes the next-bounce queue the current one.
__global__ void AdvanceQueueKernel(Queues q) {
    if (threadIdx.x == 0) q.counters[kCtrIn] = q.counters[kCtrOut];
}

// ------------------------------------------------------------ class sort

// Shading class of one extend-queue entry (its hit's material kind).
__device__ inline int ShadeClassOf(const DevScene& sc, float4 hit) {
    const int32_t id = __float_as_int(hit.y);
    if (id == -1) return kClassMiss;
    int32_t material;
    if (id <= -2) {
        material = sc.sphere_material[-2 - id];
        if (material < 0) return kClassDiffuse;  // default RenderMaterial
    } else {
        material = sc.prim_material[sc.tri_prim[id]];
        if (material < 0) return kClassGeneric;  // invalid material marker
    }
    switch (sc.materials[material].kind) {
        case kDiffuse: return kClassDiffuse;
        case kConductor: return kClassConductor;
        case kDielectric: return kClassDielectric;
        case kCoatedDiffuse: return kClassCoatedDiffuse;
        default: return kClassGeneric;
    }
}

// Per-entry class plus per-class counts (block-aggregated in shared memory).
__global__ void ClassifyKernel(DevScene sc, Queues q) {
    __shared__ unsigned int s_count[kShadeClasses];
    if (threadIdx.x < kShadeClasses) s_count[threadIdx.x] = 0;
    __syncthreads();
    const int64_t count = static_cast<int64_t>(q.counters[kCtrIn]);
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < count;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int c = ShadeClassOf(sc, q.hits[e]);
        q.shade_class[e] = static_cast<uint8_t>(c);
        atomicAdd(&s_count[c], 1u);
    }
    __syncthreads();
    if (threadIdx.x < kShadeClasses && s_count[threadIdx.x] > 0) {
        atomicAdd(q.counters + kCtrClass0 + threadIdx.x, static_cast<unsigned long long>(s_count[threadIdx.x]));
    }
}

// Writes the entries into `order` grouped by class (class c occupies
// [sum of the counts of classes < c, + count of c)); order within a class is
// unspecified, which changes no result: every path's state is indexed by path.
__global__ void ScatterByClassKernel(Queues q) {
    __shared__ unsigned long long s_begin[kShadeClasses];
    __shared__ unsigned int s_count[kShadeClasses];
    __shared__ unsigned long long s_base[kShadeClasses];
    if (threadIdx.x == 0) {
        unsigned long long b = 0;
        for (int c = 0; c < kShadeClasses; ++c) {
            s_begin[c] = b;
            b += q.counters[kCtrClass0 + c];
        }
    }
    const int64_t count = static_cast<int64_t>(q.counters[kCtrIn]);
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t base = blockIdx.x * static_cast<int64_t>(blockDim.x); base < count; base += stride) {
        if (threadIdx.x < kShadeClasses) s_count[threadIdx.x] = 0;
        __syncthreads();
        const int64_t e = base + threadIdx.x;
        int c = -1;
        unsigned int local = 0;
        if (e < count) {
            c = q.shade_class[e];
            local = atomicAdd(&s_count[c], 1u);
        }
        __syncthreads();
        if (threadIdx.x < kShadeClasses && s_count[threadIdx.x] > 0) {
            s_base[threadIdx.x] = atomicAdd(q.counters + kCtrCursor0 + threadIdx.x,
                                            static_cast<unsigned long long>(s_count[threadIdx.x]));
        }
        __syncthreads();
        if (c >= 0) q.order[s_begin[c] + s_base[c] + local] = static_cast<int32_t>(e);
        __syncthreads();
    }
}

// ------------------------------------------------------------------- shade

namespace {

struct Surface {
    V3 p;        // hit point
    V3 n;        // shading normal (face-forwarded as the reference does)
    V3 ng_obj;   // object-space geometric normal of a triangle (emission MIS)
    V3 reflectance_scale;  // reflectance texture lookup (1, 1, 1 when untextured)
    int32_t material;
    int32_t prim;  // mesh primitive, -1 for spheres
    bool triangle;
};

__device__ inline V3 VertexPos(const DevScene& sc, int32_t v) { return F4(sc.positions[v]); }

// TransformNormal (src/core/transform.cpp:46-74).
__device__ inline V3 TransformNormal(const float* m, V3 n) {
    const float a = m[0], b = m[4], c = m[8], d = m[1], e = m[5], f = m[9], g = m[2], h = m[6], i = m[10];
    const float det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
    if (fabsf(det) <= 1.0e-12f) {
        const V3 tv = V3{m[0] * n.x + m[4] * n.y + m[8] * n.z, m[1] * n.x + m[5] * n.y + m[9] * n.z,
                         m[2] * n.x + m[6] * n.y + m[10] * n.z};
        const V3 fb = Normalize(tv);
        return LengthSq(fb) > 0.0f ? fb : Normalize(n);
    }
    const float inv = 1.0f / det;
    return Normalize(V3{((e * i - f * h) * n.x + (f * g - d * i) * n.y + (d * h - e * g) * n.z) * inv,
                        ((c * h - b * i) * n.x + (a * i - c * g) * n.y + (b * g - a * h) * n.z) * inv,
                        ((b * f - c * e) * n.x + (c * d - a * f) * n.y + (a * e - b * d) * n.z) * inv});
}

// ResolveShadingNormal (src/geometry/intersection.cpp:84-106).
__device__ inline V3 ResolveShadingNormal(const DevScene& sc, int32_t prim, int4 tv, float u, float v, V3 gn) {
    V3 n = Normalize(gn);
    if (sc.normals && (sc.prim_flags[prim] & 1u)) {
        const float w = 1.0f - u - v;
        const V3 n0 = F4(sc.normals[tv.x]), n1 = F4(sc.normals[tv.y]), n2 = F4(sc.normals[tv.z]);
        const V3 in = Normalize(V3{n0.x * w + n1.x * u + n2.x * v, n0.y * w + n1.y * u + n2.y * v,
                                   n0.z * w + n1.z * u + n2.z * v});
        if (LengthSq(in) > 0.0f) n = in;
    }
    if (Dot(n, gn) < 0.0f) n = -n;
    if (LengthSq(n) == 0.0f) return Normalize(gn);
    return n;
}

// ------------------------------------------------------ textured shading

__device__ __forceinline__ bool TextureValid(const DevScene& sc, int32_t t) { return t >= 0 && t < sc.texture_count; }

__device__ __forceinline__ V3 TransformPointV(const float* m, V3 p) {
    const float in[3] = {p.x, p.y, p.z};
    float out[3];
    TransformPointRef(m, in, out);
    return V3{out[0], out[1], out[2]};
}

__device__ __forceinline__ V3 TransformVectorV(const float* m, V3 v) {
    const float in[3] = {v.x, v.y, v.z};
    float out[3];
    TransformVectorRef(m, in, out);
    return V3{out[0], out[1], out[2]};
}

// The pixel-step differentials of a camera ray (GeneratePerspectiveCameraRay,
// src/scene/camera.cpp:33-37): both start at the camera origin and pass
// through (film_x + 1, film_y) and (film_x, film_y + 1).
__device__ inline void CameraDifferentials(const DevScene& sc, int32_t pixel, int32_t sample, V3& dx, V3& dy) {
    const int x = pixel % sc.width, y = pixel / sc.width;
    PixelSampler smp;
    smp.Init(sc.sampler, sc.view->seed, x, y, sample, sc.spp);
    float sx, sy;
    smp.Sample2D(kDimPixel, 0, sx, sy);
    const float fx = static_cast<float>(x) + sx;
    const float fy = static_cast<float>(y) + sy;
    dx = CameraDirection(sc, fx + 1.0f, fy);
    dy = CameraDirection(sc, fx, fy + 1.0f);
}

// ComputeTextureFootprint (src/integrators/surface_query.cpp:35-97) for a
// camera ray from `origin` with pixel differentials dx, dy; o2w is the
// instance transform (null for world-space geometry).
__device__ inline TexFootprint ComputeFootprint(const DevScene& sc, int4 tv, const float* o2w, V3 hit_point, V3 gn,
                                                V3 origin, V3 dx, V3 dy) {
    const TexFootprint zero{0.0f, 0.0f, 0.0f, 0.0f};
    V3 p0 = VertexPos(sc, tv.x), p1 = VertexPos(sc, tv.y), p2 = VertexPos(sc, tv.z);
    if (o2w) {
        p0 = TransformPointV(o2w, p0);
        p1 = TransformPointV(o2w, p1);
        p2 = TransformPointV(o2w, p2);
    }
    const float2 uv0 = sc.uvs[tv.x], uv1 = sc.uvs[tv.y], uv2 = sc.uvs[tv.z];
    const float du1 = uv1.x - uv0.x;
    const float dv1 = uv1.y - uv0.y;
    const float du2 = uv2.x - uv0.x;
    const float dv2 = uv2.y - uv0.y;
    const float uv_det = du1 * dv2 - dv1 * du2;
    if (fabsf(uv_det) < 1.0e-12f) return zero;
    const float inverse_uv_det = 1.0f / uv_det;
    const V3 dp1 = p1 - p0;
    const V3 dp2 = p2 - p0;
    const V3 dpdu = (dp1 * dv2 - dp2 * dv1) * inverse_uv_det;
    const V3 dpdv = (dp2 * du1 - dp1 * du2) * inverse_uv_det;
    auto differential_point = [&](V3 direction) {
        const float denominator = Dot(gn, direction);
        if (fabsf(denominator) < 1.0e-12f) return hit_point;
        const float t = Dot(gn, hit_point - origin) / denominator;
        return origin + direction * t;
    };
    const V3 dpdx = differential_point(dx) - hit_point;
    const V3 dpdy = differential_point(dy) - hit_point;
    const float a = Dot(dpdu, dpdu);
    const float b = Dot(dpdu, dpdv);
    const float c = Dot(dpdv, dpdv);
    const float gram_det = a * c - b * b;
    if (fabsf(gram_det) < 1.0e-20f) return zero;
    const float inverse_gram_det = 1.0f / gram_det;
    auto solve = [&](V3 dp) {
        const float u_rhs = Dot(dp, dpdu);
        const float v_rhs = Dot(dp, dpdv);
        return make_float2((u_rhs * c - v_rhs * b) * inverse_gram_det, (v_rhs * a - u_rhs * b) * inverse_gram_det);
    };
    const float2 fdx = solve(dpdx);
    const float2 fdy = solve(dpdy);
    if (!isfinite(fdx.x) || !isfinite(fdx.y) || !isfinite(fdy.x) || !isfinite(fdy.y)) return zero;
    return TexFootprint{fdx.x, fdx.y, fdy.x, fdy.y};
}

// The textured part of EvaluateMaterialAtSurface
// (src/shading/material_evaluator.cpp:131-176) for a triangle with uvs:
// the reflectance texture (multiplied into the reflectance) and the normal
// map (ResolveNormalMap, :35-96) applied to the shading normal `n`, before
// the final face-forward. At a camera-ray hit (depth 0) the lookups use the
// ray-differential footprint; other rays have none.
__device__ __forceinline__ void ApplySurfaceTextures(const DevScene& sc, const DevMaterial& dm, int32_t prim, int4 tv,
                                                  float u, float v, const float* o2w, V3 o, V3 hit_point, V3 gn,
                                                  int depth, int32_t pixel, int32_t sample, V3& n, V3& refl_scale) {
    const bool refl = TextureValid(sc, dm.reflectance_texture);
    const bool nmap = TextureValid(sc, dm.normal_map) && (sc.prim_flags[prim] & 4u) && sc.tangents;
    if (!refl && !nmap) return;
    // InterpolateUv (src/geometry/intersection.cpp:20-32).
    const float w = 1.0f - u - v;
    const float2 a = sc.uvs[tv.x], b = sc.uvs[tv.y], c = sc.uvs[tv.z];
    const float tu = a.x * w + b.x * u + c.x * v;
    const float tv2 = a.y * w + b.y * u + c.y * v;
    TexFootprint fp{0.0f, 0.0f, 0.0f, 0.0f};
    if (depth == 0) {
        V3 dx, dy;
        CameraDifferentials(sc, pixel, sample, dx, dy);
        fp = ComputeFootprint(sc, tv, o2w, hit_point, gn, o, dx, dy);
    }
    if (refl) {
        const float4 t = SampleTexture4(sc.textures[dm.reflectance_texture], tu, tv2, fp, sc.ewa_weights);
        refl_scale = V3{t.x, t.y, t.z};
    }
    if (!nmap) return;
    const float4 enc = SampleTexture4(sc.textures[dm.normal_map], tu, tv2, fp, sc.ewa_weights);
    V3 ts{enc.x * 2.0f - 1.0f, enc.y * 2.0f - 1.0f, enc.z * 2.0f - 1.0f};
    ts.x = ts.x * dm.normal_scale;
    ts.y = ts.y * dm.normal_scale;
    ts = Normalize(ts);
    if (LengthSq(ts) == 0.0f) return;
    // InterpolateTangent / InterpolateHandedness (intersection.cpp:49-73).
    const float4 t0 = sc.tangents[tv.x], t1 = sc.tangents[tv.y], t2 = sc.tangents[tv.z];
    V3 tangent = Normalize(V3{t0.x * w + t1.x * u + t2.x * v, t0.y * w + t1.y * u + t2.y * v,
                              t0.z * w + t1.z * u + t2.z * v});
    if (o2w) tangent = TransformVectorV(o2w, tangent);
    // OrthogonalizeTangent (material_evaluator.cpp:27-33).
    const V3 projected = tangent - n * Dot(tangent, n);
    if (LengthSq(projected) <= 1.0e-12f) return;
    tangent = Normalize(projected);
    if (LengthSq(tangent) == 0.0f) return;
    float orientation = 1.0f;
    if (o2w) {
        const float* m = o2w;
        const float det = m[0] * (m[5] * m[10] - m[9] * m[6]) - m[4] * (m[1] * m[10] - m[9] * m[2]) +
                          m[8] * (m[1] * m[6] - m[5] * m[2]);
        orientation = det < 0.0f ? -1.0f : 1.0f;
    }
    const float handedness = (t0.w * w + t1.w * u + t2.w * v) * orientation;
    const V3 bitangent = Cross(n, tangent) * handedness;
    const V3 mapped = Normalize(tangent * ts.x + bitangent * ts.y + n * ts.z);
    if (LengthSq(mapped) > 0.0f) n = mapped;
}

// TraceVisibleSurface's surface resolve (src/integrators/surface_query.cpp:129-187)
// and EvaluateMaterialAtSurface (src/shading/material_evaluator.cpp:112-180).
// Returns false for a hit on an invalid triangle material. kTextured adds
// the texture lookups (the texture stage); depth, pixel and sample locate
// the camera ray of a depth-0 hit (texture footprints).
template <bool kTextured>
__device__ inline bool ResolveSurface(const DevScene& sc, V3 o, V3 d, float4 hit, int32_t inst, Surface& s,
                                      int depth, int32_t pixel, int32_t sample) {
    s.reflectance_scale = V3{1.0f, 1.0f, 1.0f};
    const int32_t id = __float_as_int(hit.y);
    s.p = o + d * hit.x;
    if (id <= -2) {
        const int32_t sphere = -2 - id;
        const float4 c = sc.spheres[sphere];
        const V3 gn = Normalize(V3{s.p.x - c.x, s.p.y - c.y, s.p.z - c.z});
        s.n = sc.sphere_flip[sphere] ? -gn : gn;
        s.material = sc.sphere_material[sphere];
        s.prim = -1;
        s.triangle = false;
        if (s.material < 0) {  // default RenderMaterial with the default (0, 0, 1) normal
            s.n = V3{0.0f, 0.0f, 1.0f};
        }
        return true;
    }
    const int32_t prim = sc.tri_prim[id];
    const int4 tv = sc.tri_vertices[id];
    s.prim = prim;
    s.triangle = true;
    s.material = sc.prim_material[prim];
    if (s.material < 0) return false;
    const V3 p0 = VertexPos(sc, tv.x), p1 = VertexPos(sc, tv.y), p2 = VertexPos(sc, tv.z);
    const V3 raw = Normalize(Cross(p1 - p0, p2 - p0));
    s.ng_obj = raw;
    const float u = hit.z, v = hit.w;
    const V3 wo = -d;
    const bool textured = kTextured && sc.texture_count > 0 && sc.uvs && (sc.prim_flags[prim] & 2u);
    if (inst >= 0) {
        const float* m = sc.instance_o2w + 16 * inst;
        const V3 wraw = TransformNormal(m, raw);
        const V3 gn = Dot(wraw, wo) < 0.0f ? -wraw : wraw;
        V3 n = TransformNormal(m, ResolveShadingNormal(sc, prim, tv, u, v, raw));
        if (Dot(n, gn) < 0.0f) n = -n;
        if (textured) {
            ApplySurfaceTextures(sc, sc.materials[s.material], prim, tv, u, v, m, o, s.p, gn, depth, pixel, sample,
                                 n, s.reflectance_scale);
        }
        s.n = Dot(n, wo) < 0.0f ? -n : n;
    } else {
        const V3 gn = Dot(raw, wo) < 0.0f ? -raw : raw;
        V3 n = ResolveShadingNormal(sc, prim, tv, u, v, gn);
        if (textured) {
            ApplySurfaceTextures(sc, sc.materials[s.material], prim, tv, u, v, nullptr, o, s.p, gn, depth, pixel,
                                 sample, n, s.reflectance_scale);
        }
        s.n = Dot(n, wo) < 0.0f ? -n : n;
    }
    return true;
}

// SampleAliasTable (src/lighting/light_sampling.cpp:185-204).
__device__ inline int SampleAlias(const float* prob, const int32_t* alias, const float* pmf, int count, float u,
                                  float& out_pmf, float& remapped) {
    const float hi = 0.99999994f;
    const float su = isfinite(u) ? Clampf(u, 0.0f, 1.0f) : 0.0f;
    const float scaled = fminf(su, hi) * static_cast<float>(count);
    const int column = min(static_cast<int>(scaled), count - 1);
    const float frac = scaled - static_cast<float>(column);
    const float p = prob[column];
    int index = column;
    float r = 0.0f;
    if (frac < p) {
        r = p > 0.0f ? frac / p : 0.0f;
    } else {
        index = alias[column];
        r = p < 1.0f ? (frac - p) / (1.0f - p) : 0.0f;
    }
    out_pmf = pmf[index];
    remapped = Clampf(r, 0.0f, hi);
    return index;
}

__device__ __forceinline__ float EmissiveArea(const DevScene& sc, int e) {
    const float a = sc.emissive_area[e];
    return isfinite(a) && a > 0.0f ? a : 0.0f;
}

__device__ __forceinline__ float Luminance(V3 c) { return fmaxf(0.0f, 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z); }

struct LightSample {
    V3 point, normal, radiance;
    float pdf;
    int32_t emissive;
    bool valid;
};

// SampleEmissiveLights / SampleEmissivePrimitive (light_sampling.cpp:275-355).
__device__ inline LightSample SampleEmissive(const DevScene& sc, float u_select, float tx, float ty) {
    LightSample out{};
    out.valid = false;
    if (sc.emissive_count == 0) return out;
    int e = -1;
    float pmf = 0.0f, local = 0.0f;
    if (sc.alias_count == sc.emissive_count) {
        e = SampleAlias(sc.alias_prob, sc.alias_index, sc.alias_pmf, sc.alias_count, u_select, pmf, local);
        if (e < 0 || pmf <= 0.0f) return out;
    } else {
        const float total = sc.total_emissive_power;
        if (!isfinite(total) || total <= 0.0f) return out;
        const float su = isfinite(u_select) ? Clampf(u_select, 0.0f, 1.0f) : 0.0f;
        const float target = su * total;
        float cum = 0.0f;
        for (int i = 0; i < sc.emissive_count; ++i) {
            const float power = EmissiveArea(sc, i) * Luminance(Ld3(sc.emissive_radiance + 3 * i));
            if (power <= 0.0f) continue;
            const float prev = cum;
            cum += power;
            e = i;
            pmf = power / total;
            local = 1.0f;
            if (target < cum) {
                local = (target - prev) / power;
                break;
            }
        }
        if (e < 0) return out;
    }
    const float area = EmissiveArea(sc, e);
    if (area <= 0.0f) return out;
    const int32_t prim = sc.emissive_prim[e];
    if (prim < 0 || prim >= sc.primitive_count) return out;
    // SelectTriangleByArea: first triangle whose cumulative area exceeds the
    // target (zero-area triangles never raise the cumulative sum).
    const int32_t off = sc.emissive_tri_offset[e], cnt = sc.emissive_tri_count[e];
    const float parea = sc.emissive_prim_area[e];
    if (cnt == 0 || !isfinite(parea) || parea <= 0.0f) return out;
    const float su = isfinite(local) ? Clampf(local, 0.0f, 1.0f) : 0.0f;
    const float target = su * parea;
    int lo = 0, hi = cnt;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (sc.tri_cdf[off + mid] <= target) lo = mid + 1;
        else hi = mid;
    }
    if (lo == cnt) lo = cnt - 1;  // the last positive-area triangle
    const int32_t flat = sc.tri_local[off + lo];
    const int4 tv = sc.tri_vertices[flat];
    const V3 p0 = VertexPos(sc, tv.x), p1 = VertexPos(sc, tv.y), p2 = VertexPos(sc, tv.z);
    const float sq = sqrtf(tx);
    const float u = 1.0f - sq;
    const float v = ty * sq;
    out.point = p0 * (1.0f - u - v) + p1 * u + p2 * v;
    const V3 e1 = p1 - p0, e2 = p2 - p0;
    const V3 cr = Cross(e1, e2);
    out.normal = Normalize(cr);
    const float tri_area = sqrtf(LengthSq(cr)) * 0.5f;
    if (!(isfinite(tri_area) && tri_area > 0.0f) || LengthSq(out.normal) == 0.0f) return out;
    out.radiance = Ld3(sc.emissive_radiance + 3 * e);
    out.pdf = (1.0f / area) * pmf;
    out.emissive = e;
    out.valid = true;
    return out;
}

// PdfEmissiveLightSolidAngle (light_sampling.cpp:357-396).
__device__ inline float PdfEmissiveSolidAngle(const DevScene& sc, V3 shading, V3 light, V3 ln, int e) {
    if (sc.emissive_count == 0) return 0.0f;
    float area_pdf = 0.0f;
    if (e >= 0 && e < sc.emissive_count) {
        const float area = EmissiveArea(sc, e);
        if (area <= 0.0f) return 0.0f;
        float pmf = 0.0f;
        if (sc.alias_count == sc.emissive_count) {
            pmf = sc.alias_pmf[e];
        } else {
            const float total = sc.total_emissive_power;
            pmf = total > 0.0f ? (area * Luminance(Ld3(sc.emissive_radiance + 3 * e))) / total : 0.0f;
        }
        area_pdf = pmf / area;
    } else {
        float total_area = 0.0f;
        for (int i = 0; i < sc.emissive_count; ++i) total_area += EmissiveArea(sc, i);
        if (!isfinite(total_area) || total_area <= 0.0f) return 0.0f;
        area_pdf = 1.0f / total_area;
    }
    const V3 dir = light - shading;
    const float dsq = LengthSq(dir);
    if (dsq <= 0.0f) return 0.0f;
    const float c = fabsf(Dot(ln, Normalize(shading - light)));
    if (c <= 0.0f) return 0.0f;
    return area_pdf * dsq / c;
}

__device__ __forceinline__ void PushShadow(Queues& q, V3 o, V3 d, float tmax, int32_t slot) {
    const unsigned long long k = QueueAppend(q.counters + kCtrShadow);
    q.shadow_ray[2 * k] = make_float4(o.x, o.y, o.z, 1.0e-5f);
    q.shadow_ray[2 * k + 1] = make_float4(d.x, d.y, d.z, tmax);
    q.shadow_slot[k] = slot;
}

}  // namespace

// --------------------------------------------------------- analytic lights

struct AnalyticSample {
    V3 wi, radiance;
    float distance, selection_pdf;
    bool valid;
};

// DistanceSquaredToBounds / TreeImportance
// (src/lighting/analytic_light_sampling.cpp:8-20).
__device__ __forceinline__ float StdMax3(float a, float b, float c) {
    float r = a;
    if (r < b) r = b;
    if (r < c) r = c;
    return r;
}
__device__ inline float TreeImportance(const DevLightNode& n, V3 p) {
    const float dx = StdMax3(n.lo[0] - p.x, 0.0f, p.x - n.hi[0]);
    const float dy = StdMax3(n.lo[1] - p.y, 0.0f, p.y - n.hi[1]);
    const float dz = StdMax3(n.lo[2] - p.z, 0.0f, p.z - n.hi[2]);
    const float d2 = dx * dx + dy * dy + dz * dz;
    return n.power / fmaxf(1.0e-4f, d2);
}

// SampleAnalyticLight (src/lighting/analytic_light_sampling.cpp:22-142):
// the light chosen by the tree walk (power over distance), else the power
// alias table, else uniformly; then the point / spot / distant sample.
// Not inlined, and given pointers rather than the scene, so that the shade
// kernels do not carry its registers when a scene has no analytic lights.
__device__ __noinline__ AnalyticSample SampleAnalyticLight(const DevAnalytic* analytic, int32_t analytic_count,
                                                           const float* alias_prob, const int32_t* alias_index,
                                                           const float* alias_pmf, const DevLightNode* tree,
                                                           int32_t tree_root, V3 p, float select) {
    struct {
        const DevAnalytic* analytic;
        int32_t analytic_count;
        const float* analytic_alias_prob;
        const int32_t* analytic_alias_index;
        const float* analytic_alias_pmf;
        const DevLightNode* analytic_tree;
        int32_t analytic_tree_root;
    } sc{analytic, analytic_count, alias_prob, alias_index, alias_pmf, tree, tree_root};
    AnalyticSample out{{0, 0, 0}, {0, 0, 0}, 0.0f, 0.0f, false};
    int light = -1;
    float pdf = 1.0f;
    float u = select < 0.0f ? 0.0f : (0.99999994f < select ? 0.99999994f : select);
    if (sc.analytic_tree_root >= 0) {
        int node = sc.analytic_tree_root;
        for (int guard = 0; node >= 0 && guard < 64; ++guard) {
            const DevLightNode& n = sc.analytic_tree[node];
            if (n.light_index >= 0) {
                light = n.light_index;
                break;
            }
            if (n.left < 0 || n.right < 0) return out;
            const float lw = TreeImportance(sc.analytic_tree[n.left], p);
            const float rw = TreeImportance(sc.analytic_tree[n.right], p);
            const float total = lw + rw;
            const float lp = total > 0.0f ? lw / total : 0.5f;
            if (u < lp) {
                pdf *= lp;
                u = lp > 0.0f ? u / lp : 0.0f;
                node = n.left;
            } else {
                const float rp = 1.0f - lp;
                pdf *= rp;
                u = rp > 0.0f ? (u - lp) / rp : 0.0f;
                node = n.right;
            }
        }
    } else if (sc.analytic_alias_pmf) {
        float r;
        light = SampleAlias(sc.analytic_alias_prob, sc.analytic_alias_index, sc.analytic_alias_pmf, sc.analytic_count,
                            u, pdf, r);
    } else {
        light = min(static_cast<int>(u * static_cast<float>(sc.analytic_count)), sc.analytic_count - 1);
        pdf = 1.0f / static_cast<float>(sc.analytic_count);
    }
    if (light < 0 || light >= sc.analytic_count || pdf <= 0.0f) return out;
    const DevAnalytic& l = sc.analytic[light];
    const V3 intensity = Ld3(l.intensity);
    if (l.kind == 2) {  // distant
        const V3 to_light = -Ld3(l.direction);
        if (LengthSq(to_light) == 0.0f) return out;
        out.wi = Normalize(to_light);
        out.distance = 1.0e6f;
        out.radiance = intensity;
    } else {
        const V3 delta = Ld3(l.position) - p;
        const float dsq = Dot(delta, delta);
        if (dsq <= 0.0f) return out;
        const float dist = sqrtf(dsq);
        if (l.kind == 0) {  // point
            out.wi = Normalize(delta);
            out.radiance = intensity / dsq;
        } else {  // spot
            const V3 wi = delta / dist;
            const V3 ld = Ld3(l.direction);
            const V3 axis = LengthSq(ld) > 0.0f ? Normalize(ld) : V3{0.0f, 0.0f, 1.0f};
            const float cc = -Dot(wi, axis);
            float falloff = 0.0f;
            if (cc >= l.cone_cos_inner) {
                falloff = 1.0f;
            } else if (cc > l.cone_angle) {
                const float t = (cc - l.cone_angle) / (l.cone_cos_inner - l.cone_angle);
                falloff = t * t * (3.0f - 2.0f * t);
            }
            out.wi = wi;
            out.radiance = intensity * (falloff / dsq);
        }
        out.distance = dist;
    }
    out.valid = true;
    out.selection_pdf = pdf;
    return out;
}

// EstimateDirectLight (src/integrators/path_direct_lighting.cpp:170-283) with
// visibility deferred: draws the light samples of vertex p (normal n, towards
// the viewer wo), stores each contribution without visibility in the path's
// NEE slots and queues the shadow rays; the shadow stage and NeeResolveKernel
// finish the estimate.
//
// kEmissiveOnly: the scene has neither analytic lights nor a sampleable
// environment (checked on the host), so those two branches are left out of
// the instance.
template <bool kEmissiveOnly = false>
__device__ inline void NextEvent(const DevScene& sc, PathState& ps, Queues& q, int32_t path, PixelSampler& smp,
                                 Pcg32& rng, int depth, const Mat& m, V3 p, V3 n, V3 wo, V3 tp, uint32_t& flags) {
    bool any = false;
    if (sc.emissive_count > 0) {
        const float us = smp.Sample1D(kDimDirectLightSelect, depth);
        float tx, ty;
        smp.Sample2D(kDimDirectLightSurface, depth, tx, ty);
        const LightSample ls = SampleEmissive(sc, us, tx, ty);
        if (ls.valid && ls.pdf > 0.0f && !IsBlack(ls.radiance)) {
            const V3 to_light = ls.point - p;
            const float dsq = LengthSq(to_light);
            if (dsq > kMinShadowBias * kMinShadowBias) {
                const float dist = sqrtf(dsq);
                const float sb = ShadowBias(p, ls.point, dist);
                if (dist > sb) {
                    const V3 so = p + n * sb;
                    const V3 stl = ls.point - so;
                    const float sdsq = LengthSq(stl);
                    if (sdsq > kMinShadowBias * kMinShadowBias) {
                        const float sd = sqrtf(sdsq);
                        const V3 wi = stl / sd;
                        const float cs = fmaxf(0.0f, Dot(n, wi));
                        if (cs > 0.0f) {
                            const float pl = PdfEmissiveSolidAngle(sc, p, ls.point, ls.normal, ls.emissive);
                            if (pl > 0.0f) {
                                CountStat(q.counters, kStatShadow);
                                const V3 f = EvalBsdf(m, wo, wi, n, rng);
                                if (!IsBlack(f)) {
                                    const float pb = PdfBsdf(m, wo, wi, n, rng);
                                    const float mis = PowerHeuristic(1, pl, 1, pb);
                                    ps.nee[3 * path + 0] = ToF4(Mul(f, ls.radiance) * (cs * mis / pl));
                                    PushShadow(q, so, wi, sd - sb, 3 * path + 0);
                                    any = true;
                                } else {
                                    ps.nee[3 * path + 0] = make_float4(0, 0, 0, 0);
                                }
                            }
                        }
                    }
                }
            }
        }
    }
    if (!kEmissiveOnly && sc.analytic_count > 0) {  // delta lights: no MIS against the BSDF
        const AnalyticSample as = SampleAnalyticLight(sc.analytic, sc.analytic_count, sc.analytic_alias_prob,
                                                      sc.analytic_alias_index, sc.analytic_alias_pmf,
                                                      sc.analytic_tree, sc.analytic_tree_root, p,
                                                      smp.Sample1D(kDimAnalyticLightSelect, depth));
        if (as.valid && as.selection_pdf > 0.0f && !IsBlack(as.radiance)) {
            const float cs = fmaxf(0.0f, Dot(n, as.wi));
            if (cs > 0.0f) {
                const V3 f = EvalBsdf(m, wo, as.wi, n, rng);
                if (!IsBlack(f)) {
                    CountStat(q.counters, kStatShadow);
                    const float sb = SurfaceBias(p);
                    ps.nee[3 * path + 1] = ToF4(Mul(f, as.radiance) * (cs / as.selection_pdf));
                    PushShadow(q, p + n * sb, as.wi, as.distance - sb, 3 * path + 1);
                    any = true;
                }
            }
        }
    }
    if (!kEmissiveOnly && EnvSampleable(sc.env)) {
        float tx, ty;
        smp.Sample2D(kDimDirectLightSurface, depth, tx, ty);
        const EnvSample es = SampleEnvironment(sc.env, tx, ty);
        if (es.valid && es.pdf > 0.0f && !IsBlack(es.radiance)) {
            const float cs = fmaxf(0.0f, Dot(n, es.dir));
            if (cs > 0.0f) {
                const V3 f = EvalBsdf(m, wo, es.dir, n, rng);
                if (!IsBlack(f)) {
                    CountStat(q.counters, kStatShadow);
                    const float pb = PdfBsdf(m, wo, es.dir, n, rng);
                    const float mis = PowerHeuristic(1, es.pdf, 1, pb);
                    ps.nee[3 * path + 2] = ToF4(Mul(f, es.radiance) * (cs * mis / es.pdf));
                    PushShadow(q, p + n * SurfaceBias(p), es.dir, __int_as_float(0x7f800000),
                               3 * path + 2);
                    any = true;
                }
            }
        }
    }
    if (any) {
        flags |= kPathNee;
        ps.nee_tp[path] = ToF4(tp);
        const unsigned long long k = QueueAppend(q.counters + kCtrNee);
        q.nee_paths[k] = path;
    }
}

// A coated (layered) vertex, whose BSDF evaluations draw from the path's
// PCG32 stream. EstimateDirectLight (src/integrators/path_direct_lighting.cpp:
// 170-283) evaluates the BSDF for an emissive light sample only after its
// shadow ray came back visible, then evaluates it for the analytic and the
// environment samples before their shadow rays, draws the environment pdf
// after its ray, and the continuation is sampled after all of that
// (path_integrator.cpp:93-173). To draw in that order the vertex is kept
// (PathState::defer) and finished in two later stages: here only the
// emissive light sample and its shadow ray, which need no BSDF; then
// LayeredNeeKernel after the shadow stage, and LayeredContinueKernel after a
// second shadow stage for the analytic and environment rays.
__device__ inline void DeferLayeredVertex(const DevScene& sc, PathState& ps, Queues& q, int32_t path,
                                          PixelSampler& smp, int depth, const Mat& m, int32_t material, V3 p, V3 n,
                                          V3 wo, uint32_t& flags) {
    float4* v = ps.defer + 5 * static_cast<int64_t>(path);
    v[0] = ToF4(p, __int_as_float(material));
    v[1] = ToF4(n, __int_as_float(m.kind));
    v[2] = ToF4(wo, 0.0f);
    v[3] = ToF4(m.reflectance, 0.0f);
    flags &= ~(kPathDeferEmissive | kPathDeferAnalytic | kPathDeferEnvironment);
    if (sc.emissive_count > 0) {
        const float us = smp.Sample1D(kDimDirectLightSelect, depth);
        float tx, ty;
        smp.Sample2D(kDimDirectLightSurface, depth, tx, ty);
        const LightSample ls = SampleEmissive(sc, us, tx, ty);
        if (ls.valid && ls.pdf > 0.0f && !IsBlack(ls.radiance)) {
            const V3 to_light = ls.point - p;
            const float dsq = LengthSq(to_light);
            if (dsq > kMinShadowBias * kMinShadowBias) {
                const float dist = sqrtf(dsq);
                const float sb = ShadowBias(p, ls.point, dist);
                if (dist > sb) {
                    const V3 so = p + n * sb;
                    const V3 stl = ls.point - so;
                    const float sdsq = LengthSq(stl);
                    if (sdsq > kMinShadowBias * kMinShadowBias) {
                        const float sd = sqrtf(sdsq);
                        const V3 wi = stl / sd;
                        const float cs = fmaxf(0.0f, Dot(n, wi));
                        if (cs > 0.0f) {
                            const float pl = PdfEmissiveSolidAngle(sc, p, ls.point, ls.normal, ls.emissive);
                            if (pl > 0.0f) {
                                CountStat(q.counters, kStatShadow);
                                ps.nee[3 * path + 0] = ToF4(ls.radiance, cs);
                                v[4] = ToF4(wi, pl);
                                PushShadow(q, so, wi, sd - sb, 3 * path + 0);
                                flags |= kPathDeferEmissive;
                            }
                        }
                    }
                }
            }
        }
    }
    const unsigned long long k = QueueAppend(q.counters + kCtrDefer);
    q.defer_paths[k] = path;
}

// Radiance-cache query of a surface vertex (the 16-float layout of
// yrc_nrc_infer): position, roughness, direction towards the viewer,
// shading normal, diffuse and specular albedo.
__device__ __forceinline__ void WriteCacheQuery(float* out, V3 p, V3 wo, V3 n, const Mat& m) {
    const bool diffuse_like = m.kind == kDiffuse || m.kind == kCoatedDiffuse || m.kind == kDiffuseTransmission;
    const bool specular_like = m.kind != kDiffuse && m.kind != kDiffuseTransmission;
    const V3 kd = diffuse_like ? m.reflectance : V3{0.0f, 0.0f, 0.0f};
    const float ks = specular_like ? 1.0f : 0.0f;
    float4* o = reinterpret_cast<float4*>(out);
    o[0] = make_float4(p.x, p.y, p.z, m.ur);
    o[1] = make_float4(wo.x, wo.y, wo.z, n.x);
    o[2] = make_float4(n.y, n.z, kd.x, kd.y);
    o[3] = make_float4(kd.z, ks, ks, ks);
}

// The end of a surface vertex of IntegratePathSample (src/integrators/
// path_integrator.cpp:171-192): the continuation sampled from the BSDF,
// Russian roulette from depth 3, the medium state after a thick-dielectric
// transmission and the next bounce's ray queued; then the path's throughput,
// radiance, flags and PCG32 state are stored.
__device__ inline void ContinuePath(const DevScene& sc, PathState& ps, Queues& q, int32_t path, int depth,
                                    const Mat& m, int32_t material, V3 p, V3 n, V3 wo, V3 tp, V3 rad,
                                    uint32_t flags, PixelSampler& smp, Pcg32& rng) {
    bool cont = depth + 1 < sc.max_depth;
    BsdfSample bs = NoSample();
    if (cont) {
        float bx, by;
        smp.Sample2D(kDimBsdf, depth, bx, by);
        bs = SampleBsdf(m, wo, n, bx, by, rng);
        cont = bs.valid && !IsBlack(bs.weight);
    }
    if (cont) {
        tp = Mul(tp, bs.weight);
        // SurviveRussianRoulette (path_integrator_common.cpp:185-201)
        if (depth >= 3) {
            const float survival = Clampf(MaxComp(tp), 0.05f, 0.95f);
            if (smp.Sample1D(kDimRussianRoulette, depth) >= survival) {
                cont = false;
            } else {
                tp = tp / survival;
            }
        }
    }
    if (cont) {
        // UpdateMediumStateAfterBsdf (path_integrator_common.cpp:108-123)
        if (m.kind == kDielectric && Dot(bs.wi, n) < 0.0f) {
            if (flags & kPathMedium) {
                flags &= ~kPathMedium;
            } else {
                flags |= kPathMedium;
                const DevMaterial& dm = sc.materials[material];
                ps.medium[path] = make_float4(dm.absorption_color[0], dm.absorption_color[1],
                                              dm.absorption_color[2], dm.absorption_distance);
            }
        }
        flags |= kPathPrevValid;
        flags = bs.specular ? (flags | kPathPrevDelta) : (flags & ~kPathPrevDelta);
        ps.prev[path] = ToF4(p, bs.pdf);
        const V3 bn = Dot(bs.wi, n) >= 0.0f ? n : -n;
        const V3 no = p + bn * SurfaceBias(p);
        const unsigned long long k = QueueAppend(q.counters + kCtrOut);
        q.ray_out[2 * k] = make_float4(no.x, no.y, no.z, 1.0e-5f);
        q.ray_out[2 * k + 1] = make_float4(bs.wi.x, bs.wi.y, bs.wi.z, __int_as_float(0x7f800000));
        q.path_out[k] = path;
    }
    ps.throughput[path] = ToF4(tp);
    ps.radiance[path] = ToF4(rad);
    ps.flags[path] = flags;
    ps.rng_state[path] = rng.state;
}

// The material kind a shading class folds to (-1: any kind).
template <int kClass>
__device__ constexpr int32_t ClassKind() {
    return kClass == kClassDiffuse ? kDiffuse
         : kClass == kClassConductor ? kConductor
         : kClass == kClassDielectric ? kDielectric
         : kClass == kClassCoatedDiffuse ? kCoatedDiffuse : -1;
}

// Texture stage of a bounce: for every extend-queue entry that hit a
// triangle with uvs whose material has a reflectance texture or a normal
// map, the textured surface resolve (EvaluateMaterialAtSurface,
// src/shading/material_evaluator.cpp:112-180): the reflectance scale and
// the final shading normal, w = 1; other entries get w = 0. Kept apart from
// the shade kernels so that their register budget does not carry the
// texture filters.
__global__ void __launch_bounds__(256, 4) SurfaceTextureKernel(DevScene sc, PathState ps, Queues q, int depth) {
    const int64_t n = static_cast<int64_t>(q.counters[kCtrIn]);
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < n;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const float4 hit = q.hits[e];
        const int32_t id = __float_as_int(hit.y);
        bool textured = false;
        if (id >= 0) {
            const int32_t prim = sc.tri_prim[id];
            const int32_t mi = sc.prim_material[prim];
            if (mi >= 0 && (sc.prim_flags[prim] & 2u)) {
                const DevMaterial& dm = sc.materials[mi];
                textured = TextureValid(sc, dm.reflectance_texture) ||
                           (TextureValid(sc, dm.normal_map) && (sc.prim_flags[prim] & 4u) && sc.tangents);
            }
        }
        if (!textured) {
            q.tex_normal[e] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            continue;
        }
        const int32_t path = q.path_in[e];
        const V3 o = F4(q.ray_in[2 * e]), d = F4(q.ray_in[2 * e + 1]);
        Surface s;
        ResolveSurface<true>(sc, o, d, hit, q.inst[e], s, depth, ps.pixel[path], ps.sample[path]);
        q.tex_normal[e] = make_float4(s.n.x, s.n.y, s.n.z, 1.0f);
        q.tex_scale[e] = make_float4(s.reflectance_scale.x, s.reflectance_scale.y, s.reflectance_scale.z, 0.0f);
    }
}

// ----------------------------------------------------------- alpha cut-outs

constexpr int kMaxAlphaSkips = 64;          // MaxAlphaSkippedHits (surface_query.cpp:12)
constexpr float kAlphaSkipOffset = 1.0e-4f;  // AlphaSkipTOffset (surface_query.cpp:13)

struct TraceHit {
    float4 h;      // t, id bits (-1 miss), u, v
    int32_t inst;
};

// Closest hit of (o, d) over [tmin, tmax], one ray per thread (IntersectBvh /
// IntersectTwoLevelBvh); col is the thread's shared-memory stack column.
template <bool kTwo, int kTotal>
__device__ inline TraceHit ClosestHit(const AccelParams& a, V3 o, V3 d, float tmin, float tmax,
                                      StackStore<kTotal>& st, int2* col, int* error) {
    Traversal t;
    const float of[3] = {o.x, o.y, o.z};
    const float df[3] = {d.x, d.y, d.z};
    bool alive = BeginRay(a, of, df, tmin, tmax, t);
    while (alive) alive = Step<false, false, kTwo>(a, nullptr, 0, t, st, col, error);
    TraceHit r;
    r.h = make_float4(t.best.t, __int_as_float(t.best.hit ? t.best.id : -1), t.best.u, t.best.v);
    r.inst = t.best.hit ? t.best_inst : -1;
    return r;
}

// The resolved alpha of a triangle hit (EvaluateMaterialAtSurface,
// src/shading/material_evaluator.cpp:130-149) compared with IsAlphaVisible's
// 0.5 (:182-184). Spheres and hits on invalid materials are visible. At a
// camera-ray hit (depth 0) the alpha texture uses the ray-differential
// footprint.
__device__ inline bool AlphaVisible(const DevScene& sc, V3 o, V3 d, float4 hit, int32_t inst, int depth, int32_t pixel,
                                    int32_t sample) {
    const int32_t id = __float_as_int(hit.y);
    if (id < 0) return true;
    const int32_t prim = sc.tri_prim[id];
    const int32_t mi = sc.prim_material[prim];
    if (mi < 0) return true;
    const DevMaterial& dm = sc.materials[mi];
    float alpha = dm.alpha;
    if (sc.uvs && (sc.prim_flags[prim] & 2u) && TextureValid(sc, dm.alpha_texture)) {
        const int4 tv = sc.tri_vertices[id];
        const float u = hit.z, v = hit.w;
        const float w = 1.0f - u - v;
        const float2 a = sc.uvs[tv.x], b = sc.uvs[tv.y], c = sc.uvs[tv.z];
        const float tu = a.x * w + b.x * u + c.x * v;
        const float tw = a.y * w + b.y * u + c.y * v;
        TexFootprint fp{0.0f, 0.0f, 0.0f, 0.0f};
        if (depth == 0) {
            const float* m = inst >= 0 ? sc.instance_o2w + 16 * inst : nullptr;
            const V3 p0 = VertexPos(sc, tv.x), p1 = VertexPos(sc, tv.y), p2 = VertexPos(sc, tv.z);
            V3 raw = Normalize(Cross(p1 - p0, p2 - p0));
            if (m) raw = TransformNormal(m, raw);
            const V3 gn = Dot(raw, -d) < 0.0f ? -raw : raw;
            V3 dx, dy;
            CameraDifferentials(sc, pixel, sample, dx, dy);
            fp = ComputeFootprint(sc, tv, m, o + d * hit.x, gn, o, dx, dy);
        }
        alpha = alpha * SampleTexture4(sc.textures[dm.alpha_texture], tu, tw, fp, sc.ewa_weights).x;
    }
    return alpha >= 0.5f;
}

// TraceVisibleSurface's skip loop (src/integrators/surface_query.cpp:108-199)
// after a first closest hit `first`: while the hit surface is cut out, trace
// again from just past it, at most kMaxAlphaSkips traces in all. Returns the
// visible hit, or a miss (exhausted = true when the trace budget ran out).
template <bool kTwo, int kTotal>
__device__ inline TraceHit SkipCutOuts(const DevScene& sc, V3 o, V3 d, float tmax, TraceHit first, int depth,
                                       int32_t pixel, int32_t sample, StackStore<kTotal>& st, int2* col, int* error,
                                       bool& exhausted) {
    exhausted = false;
    TraceHit h = first;
    const TraceHit miss{make_float4(tmax, __int_as_float(-1), 0.0f, 0.0f), -1};
    for (int traces = 1;; ++traces) {
        if (__float_as_int(h.h.y) == -1) return miss;
        if (AlphaVisible(sc, o, d, h.h, h.inst, depth, pixel, sample)) return h;
        const float tmin = h.h.x + kAlphaSkipOffset;
        if (tmin >= tmax) return miss;
        if (traces >= kMaxAlphaSkips) {
            exhausted = true;
            return miss;
        }
        h = ClosestHit<kTwo, kTotal>(sc.accel, o, d, tmin, tmax, st, col, error);
    }
}

// Extend-stage fix-up for scenes with cut-out materials: every entry whose
// closest hit is cut out continues past it (an exhausted skip loop counts as
// a miss, as the path integrator treats it).
template <bool kTwo, int kTotal>
__global__ void __launch_bounds__(kTraceBlock) AlphaExtendKernel(DevScene sc, PathState ps, Queues q, int depth,
                                                                 int* error) {
    __shared__ int2 s_stack[kShortStack * kTraceBlock];
    int2* col = s_stack + threadIdx.x;
    StackStore<kTotal> st;
    const int64_t n = static_cast<int64_t>(q.counters[kCtrIn]);
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < n;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const float4 hit = q.hits[e];
        const V3 o = F4(q.ray_in[2 * e]);
        const float4 rb = q.ray_in[2 * e + 1];
        const V3 d = F4(rb);
        const int32_t path = q.path_in[e];
        const int32_t inst = q.inst[e];
        if (__float_as_int(hit.y) == -1) continue;
        const int32_t pixel = depth == 0 ? ps.pixel[path] : 0;
        const int32_t sample = depth == 0 ? ps.sample[path] : 0;
        if (AlphaVisible(sc, o, d, hit, inst, depth, pixel, sample)) continue;
        bool exhausted;
        const TraceHit r = SkipCutOuts<kTwo, kTotal>(sc, o, d, rb.w, TraceHit{hit, inst}, depth, pixel, sample, st,
                                                     col, error, exhausted);
        q.hits[e] = r.h;
        q.inst[e] = r.inst;
    }
}

// TraceShadowVisibility (src/integrators/path_direct_lighting.cpp:23-113)
// one shadow ray per thread, each query a closest hit with the cut-out skip
// loop, for scenes where the single-pass shadow kernel does not apply (cut-out
// materials, or thin dielectrics whose reflectance is textured), and for the
// rays that kernel leaves to it (`list`: shadow entries past more than 16
// clear surfaces, counted in kCtrShadowOverflow). Writes the transmittance
// (w = 1 visible, all 0 occluded) to the ray's slot.
template <bool kTwo, int kTotal>
__global__ void __launch_bounds__(kTraceBlock) ShadowExactKernel(DevScene sc, Queues q, const int32_t* list,
                                                                 float4* transmittance,
                                                                 unsigned long long* occluded_count, int* error) {
    __shared__ int2 s_stack[kShortStack * kTraceBlock];
    int2* col = s_stack + threadIdx.x;
    StackStore<kTotal> st;
    const int64_t n = static_cast<int64_t>(list ? q.counters[kCtrShadowOverflow] : q.counters[kCtrShadow]);
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t k = list ? static_cast<int64_t>(list[i]) : i;
        const float4 ra = q.shadow_ray[2 * k], rb = q.shadow_ray[2 * k + 1];
        V3 o = F4(ra);
        const V3 d = F4(rb);
        float remaining = rb.w;
        float qmin = ra.w;
        V3 T{1.0f, 1.0f, 1.0f}, mc{1.0f, 1.0f, 1.0f};
        float md = 1.0f;
        bool medium = false;
        auto black = [&]() { return fmaxf(T.x, fmaxf(T.y, T.z)) <= 1.0e-6f; };
        auto beer = [&](float dist) {
            if (dist <= 0.0f || md <= 0.0f) return;
            const float inv = 1.0f / md;
            const float c0 = fminf(fmaxf(mc.x, 1.0e-6f), 1.0f), c1 = fminf(fmaxf(mc.y, 1.0e-6f), 1.0f),
                        c2 = fminf(fmaxf(mc.z, 1.0e-6f), 1.0f);
            T = V3{T.x * expf(logf(c0) * dist * inv), T.y * expf(logf(c1) * dist * inv),
                   T.z * expf(logf(c2) * dist * inv)};
        };
        float4 result = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        for (int query = 0; query < kClearHits; ++query) {
            const bool finite = isfinite(remaining);
            const TraceHit first = ClosestHit<kTwo, kTotal>(sc.accel, o, d, qmin, remaining, st, col, error);
            bool exhausted;
            const TraceHit h =
                SkipCutOuts<kTwo, kTotal>(sc, o, d, remaining, first, 1, 0, 0, st, col, error, exhausted);
            if (exhausted) break;
            const int32_t id = __float_as_int(h.h.y);
            if (id == -1) {
                if (medium) {
                    if (!finite) break;
                    beer(remaining);
                }
                if (!black()) result = make_float4(T.x, T.y, T.z, 1.0f);
                break;
            }
            const float t = h.h.x;
            if (medium) {
                beer(t);
                if (black()) break;
            }
            const int32_t prim = id >= 0 ? sc.tri_prim[id] : -1;
            const int32_t material = id >= 0 ? sc.prim_material[prim] : sc.sphere_material[-2 - id];
            if (material < 0) break;
            const DevMaterial& m = sc.materials[material];
            if (m.kind != kDielectric && m.kind != kThinDielectric) break;
            const V3 hp = o + d * t;
            if (m.kind == kThinDielectric) {
                V3 refl = Ld3(m.reflectance);
                if (id >= 0 && sc.uvs && (sc.prim_flags[prim] & 2u) && TextureValid(sc, m.reflectance_texture)) {
                    const int4 tv = sc.tri_vertices[id];
                    const float u = h.h.z, v = h.h.w;
                    const float w = 1.0f - u - v;
                    const float2 a = sc.uvs[tv.x], b = sc.uvs[tv.y], c = sc.uvs[tv.z];
                    const float4 tx = SampleTexture4(sc.textures[m.reflectance_texture], a.x * w + b.x * u + c.x * v,
                                                     a.y * w + b.y * u + c.y * v,
                                                     TexFootprint{0.0f, 0.0f, 0.0f, 0.0f}, sc.ewa_weights);
                    refl = Mul(refl, V3{tx.x, tx.y, tx.z});
                }
                T = V3{T.x * Clampf(refl.x, 0.0f, 1.0f), T.y * Clampf(refl.y, 0.0f, 1.0f),
                       T.z * Clampf(refl.z, 0.0f, 1.0f)};
                if (black()) break;
            } else if (medium) {
                medium = false;
                mc = V3{1.0f, 1.0f, 1.0f};
                md = 1.0f;
            } else {
                medium = true;
                mc = Ld3(m.absorption_color);
                md = m.absorption_distance;
            }
            const float bias = SurfaceBias(hp);
            if (finite) {
                remaining = remaining - (t + bias);
                if (remaining <= 0.0f) {
                    if (!black()) result = make_float4(T.x, T.y, T.z, 1.0f);
                    break;
                }
            }
            o = hp + d * bias;
            qmin = 1.0e-5f;
        }
        transmittance[q.shadow_slot[k]] = result;
        if (result.w == 0.0f) atomicAdd(occluded_count, 1ull);
    }
}

// IntegratePathSample's per-bounce body (src/integrators/path_integrator.cpp:23-197)
// for the entries of one shading class.
// One extend-queue entry `e` of shading class kClass.
template <int kClass, bool kLean = false>
__device__ __forceinline__ void ShadeEntry(const DevScene& sc, PathState& ps, Queues& q, int depth,
                                           const CacheArgs& cache, int64_t e) {
    const int32_t path = q.path_in[e];
    const float4 ra = q.ray_in[2 * e], rb = q.ray_in[2 * e + 1];
    const V3 o = F4(ra), d = F4(rb);
    const float4 hit = q.hits[e];
    const int32_t inst = q.inst[e];
    const int32_t id = __float_as_int(hit.y);
    V3 tp = F4(ps.throughput[path]);
    V3 rad = F4(ps.radiance[path]);
    uint32_t flags = ps.flags[path];
    const float4 prev = ps.prev[path];
    CountStat(q.counters, kStatRays);

    // --- miss: environment with the BSDF-sampling MIS weight
    if (kClass == kClassMiss || id == -1) {
        CountStat(q.counters, kStatMisses);
        float w = 1.0f;
        if ((flags & kPathPrevValid) && !(flags & kPathPrevDelta)) {
            w = PowerHeuristic(1, prev.w, 1, PdfEnvironment(sc.env, d));
        }
        rad = rad + Mul(tp, EvalEnvironment(sc.env, d)) * w;
        ps.radiance[path] = ToF4(rad);
        return;
    }
    CountStat(q.counters, kStatHits);

    // --- medium attenuation (Beer-Lambert inside a thick dielectric)
    if (flags & kPathMedium) {
        const float4 md = ps.medium[path];
        if (hit.x > 0.0f && md.w > 0.0f) {
            const float inv = 1.0f / md.w;
            const float c[3] = {Clampf(md.x, 1.0e-6f, 1.0f), Clampf(md.y, 1.0e-6f, 1.0f), Clampf(md.z, 1.0e-6f, 1.0f)};
            tp = V3{tp.x * expf(logf(c[0]) * hit.x * inv), tp.y * expf(logf(c[1]) * hit.x * inv),
                    tp.z * expf(logf(c[2]) * hit.x * inv)};
        }
    }
    if (IsBlack(tp)) {
        ps.throughput[path] = ToF4(tp);
        return;
    }

    Surface s;
    if (!ResolveSurface<false>(sc, o, d, hit, inst, s, depth, 0, 0)) {
        rad = rad + Mul(tp, V3{1.0f, 0.0f, 1.0f});  // invalid material marker
        ps.radiance[path] = ToF4(rad);
        return;
    }
    if (sc.texture_count > 0 && s.triangle) {  // the texture stage's result for this entry
        const float4 tn = q.tex_normal[e];
        if (tn.w != 0.0f) {
            s.n = F4(tn);
            s.reflectance_scale = F4(q.tex_scale[e]);
        }
    }
    Mat m;
    V3 emission{0.0f, 0.0f, 0.0f};
    if (s.material >= 0) {
        const DevMaterial& dm = sc.materials[s.material];
        m = LoadMat(dm);
        m.reflectance = Mul(m.reflectance, s.reflectance_scale);
        m.measured = dm.measured_index >= 0 ? sc.measured + dm.measured_index : nullptr;
        emission = Ld3(dm.emission);
    } else {  // default RenderMaterial: diffuse 0.5
        m = Mat{kDiffuse, {0.5f, 0.5f, 0.5f}, 1.5f, 0.0f, 0.0f, 1.5f, 0.01f, {0, 0, 0}, 10, 1};
    }
    if constexpr (ClassKind<kClass>() >= 0) m.kind = ClassKind<kClass>();  // the class fixes the kind
    const V3 wo = -d;
    if (depth == 0) {
        flags |= kPathPrimary;
        ps.aov_albedo[path] = ToF4(m.reflectance, hit.x);
        ps.aov_normal[path] = ToF4(s.n);
    }

    // --- emission with the BSDF-sampling MIS weight (triangle lights only)
    if (!IsBlack(emission) && s.triangle) {
        float w = 1.0f;
        if ((flags & kPathPrevValid) && !(flags & kPathPrevDelta)) {
            const int32_t ei = sc.prim_emissive[s.prim];
            const float pl = PdfEmissiveSolidAngle(sc, F4(prev), s.p, s.ng_obj, ei);
            w = PowerHeuristic(1, prev.w, 1, pl);
        }
        rad = rad + Mul(tp, emission) * w;
    }

    // --- radiance cache: path spread (footprint heuristic), training
    // records, early termination into the cache
    if (!kLean && cache.enabled) {
        const float cv = fmaxf(fabsf(Dot(d, s.n)), 1.0e-4f);
        float2 sp = ps.spread[path];
        if (depth == 0) {
            sp.x = hit.x * hit.x / (4.0f * kPi * cv);
            sp.y = 0.0f;
        } else if (!(flags & kPathPrevDelta)) {
            sp.y += sqrtf(hit.x * hit.x / (fmaxf(prev.w, 1.0e-12f) * cv));
        }
        ps.spread[path] = sp;
        const int32_t slot = cache.train_slot[path];
        if (slot >= 0) {
            const int32_t k = cache.slot_len[slot];
            if (k < cache.max_depth) {
                const int64_t v = static_cast<int64_t>(slot) * cache.max_depth + k;
                WriteCacheQuery(cache.slot_q + 16 * v, s.p, wo, s.n, m);
                cache.slot_lt[2 * v] = ToF4(rad);
                cache.slot_lt[2 * v + 1] = ToF4(tp);
                cache.slot_len[slot] = k + 1;
            }
        }
        const bool fires = depth >= 1 && !(flags & kPathCacheQueued) && (cache.delta_vertices || !IsDelta(m)) &&
                           sp.y * sp.y > cache.spread_c * sp.x;
        if (fires) {
            // The image estimate of the path ends here: radiance so far
            // plus throughput x cache. A training path goes on as an
            // unbiased suffix whose radiance only trains the cache.
            const unsigned long long k = QueueAppend(cache.counters + 0);
            WriteCacheQuery(cache.queries + 16 * k, s.p, wo, s.n, m);
            cache.query_path[k] = path;
            cache.query_tp[k] = ToF4(tp);
            cache.query_base[k] = ToF4(rad);
            if (slot < 0) {
                ps.throughput[path] = ToF4(tp);
                ps.radiance[path] = ToF4(rad);
                ps.flags[path] = flags;
                return;
            }
            flags |= kPathCacheQueued;
        }
    }

    PixelSampler smp;
    const int32_t pixel = ps.pixel[path];
    smp.Init(sc.sampler, sc.view->seed, pixel % sc.width, pixel / sc.width, ps.sample[path], sc.spp);
    Pcg32 rng{ps.rng_state[path], ps.rng_inc[path]};

    // --- coated vertex: next events and continuation in the reference's
    // PCG32 order, after the shadow stages (DeferLayeredVertex)
    if ((kClass == kClassCoatedDiffuse || kClass == kClassGeneric) && IsLayered(m.kind) && !IsDelta(m)) {
        DeferLayeredVertex(sc, ps, q, path, smp, depth, m, s.material, s.p, s.n, wo, flags);
        ps.throughput[path] = ToF4(tp);
        ps.radiance[path] = ToF4(rad);
        ps.flags[path] = flags;
        return;
    }

    // --- next-event estimation: samples now, visibility in the shadow stage
    if (!IsDelta(m)) NextEvent<kLean>(sc, ps, q, path, smp, rng, depth, m, s.p, s.n, wo, tp, flags);

    // --- subsurface entry (path_integrator.cpp:103-135): Fresnel split at
    // the interface; the transmitted part becomes a probe ray that the
    // subsurface stage traces and closes (SubsurfaceExitKernel).
    if (kClass == kClassGeneric && m.kind == kSubsurface && s.material >= 0 &&
        sc.materials[s.material].bssrdf_index >= 0 && sc.materials[s.material].bssrdf_index < sc.bssrdf_count) {
        if (depth + 1 < sc.max_depth) {
            const DevMaterial& dm = sc.materials[s.material];
            const V3 ns = s.n;
            V3 ss, ts;
            BssrdfFrame(ns, ss, ts);
            const float fr = FrDielectric(fabsf(Dot(wo, ns)), dm.bssrdf_eta);
            if (smp.Sample1D(kDimBssrdfReflect, depth) < fr) {
                // Specular reflection (the selection probability cancels Fresnel).
                const V3 wr = ns * (2.0f * Dot(wo, ns)) - wo;
                flags |= kPathPrevValid | kPathPrevDelta;
                ps.prev[path] = ToF4(s.p, 1.0f);
                const V3 bn = Dot(wr, ns) >= 0.0f ? ns : -ns;
                const V3 no = s.p + bn * SurfaceBias(s.p);
                const unsigned long long k = QueueAppend(q.counters + kCtrOut);
                q.ray_out[2 * k] = make_float4(no.x, no.y, no.z, 1.0e-5f);
                q.ray_out[2 * k + 1] = make_float4(wr.x, wr.y, wr.z, __int_as_float(0x7f800000));
                q.path_out[k] = path;
            } else {
                // SampleBssrdfProbe (src/integrators/bssrdf_probe.cpp:17-60): projection
                // axis, colour channel, radius, and the probe segment through the disk.
                const TabBssrdf tab = MakeTabBssrdf(dm, sc.bssrdf[dm.bssrdf_index]);
                float u1 = smp.Sample1D(kDimBssrdfAxis, depth);
                float ux, uy;
                smp.Sample2D(kDimBssrdfDisk, depth, ux, uy);
                V3 vx, vy, vz;
                if (u1 < 0.5f) {
                    vx = ss, vy = ts, vz = ns;
                    u1 *= 2.0f;
                } else if (u1 < 0.75f) {
                    vx = ts, vy = ns, vz = ss;
                    u1 = (u1 - 0.5f) * 4.0f;
                } else {
                    vx = ns, vy = ss, vz = ts;
                    u1 = (u1 - 0.75f) * 4.0f;
                }
                const int channel = min(max(static_cast<int>(u1 * 3.0f), 0), 2);
                u1 = u1 * 3.0f - static_cast<float>(channel);
                const float radius = BssrdfSampleSr(tab, channel, ux);
                if (radius >= 0.0f) {
                    const float phi = 2.0f * kPi * uy;
                    const float max_radius = BssrdfSampleSr(tab, channel, 0.999f);
                    if (radius < max_radius) {
                        const float length = 2.0f * sqrtf(fmaxf(0.0f, max_radius * max_radius - radius * radius));
                        // cos/sin rounded from double precision: the correctly rounded
                        // float values, as the host libm's float cos/sin return them.
                        const float cphi = static_cast<float>(cos(static_cast<double>(phi)));
                        const float sphi = static_cast<float>(sin(static_cast<double>(phi)));
                        const V3 disk = vx * (radius * cphi) + vy * (radius * sphi);
                        const V3 base = s.p + disk - vz * (length * 0.5f);
                        const unsigned long long k = QueueAppend(q.counters + kCtrProbe);
                        q.probe_ray[2 * k] = make_float4(base.x, base.y, base.z, 1.0e-5f);
                        q.probe_ray[2 * k + 1] = make_float4(vz.x, vz.y, vz.z, length);
                        q.probe_target[k] = make_int4(s.triangle ? s.prim : -1, s.triangle ? inst : -1,
                                                      s.triangle ? -1 : -2 - id, path);
                        q.probe_entry[2 * k] = ToF4(s.p, u1);
                        q.probe_entry[2 * k + 1] = ToF4(ns, __int_as_float(s.material));
                    }
                }
            }
        }
        ps.throughput[path] = ToF4(tp);
        ps.radiance[path] = ToF4(rad);
        ps.flags[path] = flags;
        ps.rng_state[path] = rng.state;
        return;
    }

    ContinuePath(sc, ps, q, path, depth, m, s.material, s.p, s.n, wo, tp, rad, flags, smp, rng);
}

// kLean: the scene has only emissive-surface lights and no radiance cache
// (ShadeLean, on the host); the instance leaves the other light kinds' and
// the cache's code out, which frees registers for the rest.
template <int kClass, bool kLean>
__global__ void __launch_bounds__(256, 2) ShadeKernel(DevScene sc, PathState ps, Queues q, int depth,
                                                       CacheArgs cache) {
    unsigned long long begin = 0;
#pragma unroll
    for (int c = 0; c < kClass; ++c) begin += q.counters[kCtrClass0 + c];
    const int64_t count = static_cast<int64_t>(q.counters[kCtrClass0 + kClass]);
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        ShadeEntry<kClass, kLean>(sc, ps, q, depth, cache, q.order[begin + i]);
    }
}

// ShadeKernel over the class-kClass entries of several jobs' extend queues
// at once (ShadeJob table): each thread takes an entry from the jobs'
// class ranges laid end to end and shades it with its job's scene, path
// state and queues.
template <int kClass>
__global__ void __launch_bounds__(256, 2) PooledShadeKernel(const ShadeJob* __restrict__ jobs, int njobs) {
    __shared__ unsigned long long s_ends[kMaxPoolJobs];
    __shared__ unsigned long long s_begin[kMaxPoolJobs];
    for (int j = threadIdx.x; j < njobs; j += blockDim.x) {
        const unsigned long long* c = jobs[j].q.counters;
        unsigned long long b = 0;
#pragma unroll
        for (int k = 0; k < kClass; ++k) b += c[kCtrClass0 + k];
        s_begin[j] = b;
        s_ends[j] = c[kCtrClass0 + kClass];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int j = 1; j < njobs; ++j) s_ends[j] += s_ends[j - 1];
    }
    __syncthreads();
    const unsigned long long total = njobs > 0 ? s_ends[njobs - 1] : 0ull;
    for (unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
        const int j = PoolJobOf(s_ends, njobs, i);
        const ShadeJob& job = jobs[j];
        PathState ps = job.ps;
        Queues q = job.q;
        const unsigned long long local = i - (j ? s_ends[j - 1] : 0ull);
        ShadeEntry<kClass>(job.sc, ps, q, job.depth, job.cache, q.order[s_begin[j] + local]);
    }
}

// Adds each path's visible next-event contributions:
// radiance += throughput_at_vertex * ((emissive + analytic) + environment).
// Each thread resolves kNeePerThread entries (e, e + stride, ...) with all
// of their paths' loads issued before any store: the accesses follow the
// shading order through the path state, so the kernel waits on latency, and
// independent paths per thread multiply the loads in flight.
constexpr int kNeePerThread = 2;

template <bool kTransmittance>
__global__ void NeeResolveKernel(PathState ps, Queues q, const float4* transmittance) {
    const int64_t count = static_cast<int64_t>(q.counters[kCtrNee]);
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t e0 = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e0 < count;
         e0 += kNeePerThread * stride) {
        int32_t path[kNeePerThread];
        bool live[kNeePerThread];
#pragma unroll
        for (int j = 0; j < kNeePerThread; ++j) {
            const int64_t e = e0 + j * stride;
            live[j] = e < count;
            path[j] = live[j] ? q.nee_paths[e] : q.nee_paths[e0];
        }
        float4 c[kNeePerThread][3], vis[kNeePerThread][3], tp[kNeePerThread], rad[kNeePerThread];
        uint32_t fl[kNeePerThread];
#pragma unroll
        for (int j = 0; j < kNeePerThread; ++j) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int32_t slot = 3 * path[j] + k;
                c[j][k] = ps.nee[slot];
                if (kTransmittance) {
                    vis[j][k] = transmittance[slot];
                } else {
                    const float v = q.shadow_occluded[slot] ? 0.0f : 1.0f;
                    vis[j][k] = make_float4(v, v, v, 0.0f);
                }
            }
            tp[j] = ps.nee_tp[path[j]];
            rad[j] = ps.radiance[path[j]];
            fl[j] = ps.flags[path[j]];
        }
#pragma unroll
        for (int j = 0; j < kNeePerThread; ++j) {
            if (!live[j]) continue;
            V3 sum{0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                sum = sum + Mul(F4(c[j][k]), F4(vis[j][k]));
                ps.nee[3 * path[j] + k] = make_float4(0, 0, 0, 0);
            }
            ps.radiance[path[j]] = ToF4(F4(rad[j]) + Mul(F4(tp[j]), sum));
            ps.flags[path[j]] = fl[j] & ~kPathNee;
        }
    }
}

// ------------------------------------------------------ coated vertices

// A queued shadow ray's outcome by its slot: the transmittance (w = 1
// visible, all 0 occluded) or, in scenes without surfaces that pass light,
// the any-hit flag.
template <bool kTransmittance>
__device__ __forceinline__ float4 SlotVisibility(const Queues& q, const float4* transmittance, int32_t slot) {
    if (kTransmittance) return transmittance[slot];
    const float v = q.shadow_occluded[slot] ? 0.0f : 1.0f;
    return make_float4(v, v, v, v);
}

// The BSDF of a deferred coated vertex (the shade kernel's Mat).
__device__ inline Mat DeferredMat(const DevScene& sc, const float4* v) {
    Mat m = LoadMat(sc.materials[__float_as_int(v[0].w)]);
    m.kind = __float_as_int(v[1].w);
    m.reflectance = F4(v[3]);
    m.measured = nullptr;
    return m;
}

// After the shadow stage: the emissive next event of each deferred coated
// vertex (BSDF value and pdf drawn only when its shadow ray was visible),
// then the analytic and environment samples with their BSDF values and
// shadow rays (queued for a second shadow stage), as EstimateDirectLight
// orders them (path_direct_lighting.cpp:185-262, 115-168). A vertex with no
// second-stage ray samples its continuation right away.
template <bool kTransmittance>
__global__ void __launch_bounds__(256, 2) LayeredNeeKernel(DevScene sc, PathState ps, Queues q,
                                                            const float4* transmittance, int depth) {
    const int64_t count = static_cast<int64_t>(q.counters[kCtrDefer]);
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t path = q.defer_paths[i];
        float4* v = ps.defer + 5 * static_cast<int64_t>(path);
        const V3 p = F4(v[0]), n = F4(v[1]), wo = F4(v[2]);
        const int32_t material = __float_as_int(v[0].w);
        const Mat m = DeferredMat(sc, v);
        uint32_t flags = ps.flags[path];
        Pcg32 rng{ps.rng_state[path], ps.rng_inc[path]};
        PixelSampler smp;
        const int32_t pixel = ps.pixel[path];
        smp.Init(sc.sampler, sc.view->seed, pixel % sc.width, pixel / sc.width, ps.sample[path], sc.spp);
        V3 sum{0.0f, 0.0f, 0.0f};
        if (flags & kPathDeferEmissive) {
            const float4 vis = SlotVisibility<kTransmittance>(q, transmittance, 3 * path + 0);
            if (vis.w == 1.0f) {
                const float4 lc = ps.nee[3 * path + 0];  // radiance, cosine
                const float4 wl = v[4];                  // direction, light pdf
                const V3 wi = F4(wl);
                const V3 f = EvalBsdf(m, wo, wi, n, rng);
                if (!IsBlack(f)) {
                    const float pb = PdfBsdf(m, wo, wi, n, rng);
                    const float mis = PowerHeuristic(1, wl.w, 1, pb);
                    sum = sum + Mul(f, Mul(F4(vis), F4(lc))) * (lc.w * mis / wl.w);
                }
            }
            ps.nee[3 * path + 0] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        flags &= ~(kPathDeferEmissive | kPathDeferAnalytic | kPathDeferEnvironment);
        if (sc.analytic_count > 0) {  // delta lights: no MIS against the BSDF
            const AnalyticSample as = SampleAnalyticLight(sc.analytic, sc.analytic_count, sc.analytic_alias_prob,
                                                          sc.analytic_alias_index, sc.analytic_alias_pmf,
                                                          sc.analytic_tree, sc.analytic_tree_root, p,
                                                          smp.Sample1D(kDimAnalyticLightSelect, depth));
            if (as.valid && as.selection_pdf > 0.0f && !IsBlack(as.radiance)) {
                const float cs = fmaxf(0.0f, Dot(n, as.wi));
                if (cs > 0.0f) {
                    const V3 f = EvalBsdf(m, wo, as.wi, n, rng);
                    if (!IsBlack(f)) {
                        CountStat(q.counters, kStatShadow);
                        const float sb = SurfaceBias(p);
                        ps.nee[3 * path + 1] = ToF4(Mul(f, as.radiance) * (cs / as.selection_pdf));
                        PushShadow(q, p + n * sb, as.wi, as.distance - sb, 3 * path + 1);
                        flags |= kPathDeferAnalytic;
                    }
                }
            }
        }
        if (EnvSampleable(sc.env)) {
            float tx, ty;
            smp.Sample2D(kDimDirectLightSurface, depth, tx, ty);
            const EnvSample es = SampleEnvironment(sc.env, tx, ty);
            if (es.valid && es.pdf > 0.0f && !IsBlack(es.radiance)) {
                const float cs = fmaxf(0.0f, Dot(n, es.dir));
                if (cs > 0.0f) {
                    const V3 f = EvalBsdf(m, wo, es.dir, n, rng);
                    if (!IsBlack(f)) {
                        CountStat(q.counters, kStatShadow);
                        ps.nee[3 * path + 2] = ToF4(Mul(f, es.radiance), es.pdf);
                        v[4] = ToF4(es.dir, cs);
                        PushShadow(q, p + n * SurfaceBias(p), es.dir, __int_as_float(0x7f800000), 3 * path + 2);
                        flags |= kPathDeferEnvironment;
                    }
                }
            }
        }
        const V3 tp = F4(ps.throughput[path]);
        const V3 rad = F4(ps.radiance[path]) + Mul(tp, sum);
        if (flags & (kPathDeferAnalytic | kPathDeferEnvironment)) {
            ps.radiance[path] = ToF4(rad);
            ps.flags[path] = flags;
            ps.rng_state[path] = rng.state;
            const unsigned long long k = QueueAppend(q.counters + kCtrDefer2);
            q.defer_paths2[k] = path;
            continue;
        }
        ContinuePath(sc, ps, q, path, depth, m, material, p, n, wo, tp, rad, flags, smp, rng);
    }
}

// After the second shadow stage: the analytic contribution, the environment
// pdf (drawn only when its shadow ray was visible) and MIS weight, then the
// continuation of each deferred coated vertex.
template <bool kTransmittance>
__global__ void __launch_bounds__(256, 2) LayeredContinueKernel(DevScene sc, PathState ps, Queues q,
                                                                 const float4* transmittance, int depth) {
    const int64_t count = static_cast<int64_t>(q.counters[kCtrDefer2]);
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t path = q.defer_paths2[i];
        const float4* v = ps.defer + 5 * static_cast<int64_t>(path);
        const V3 p = F4(v[0]), n = F4(v[1]), wo = F4(v[2]);
        const int32_t material = __float_as_int(v[0].w);
        const Mat m = DeferredMat(sc, v);
        uint32_t flags = ps.flags[path];
        Pcg32 rng{ps.rng_state[path], ps.rng_inc[path]};
        PixelSampler smp;
        const int32_t pixel = ps.pixel[path];
        smp.Init(sc.sampler, sc.view->seed, pixel % sc.width, pixel / sc.width, ps.sample[path], sc.spp);
        V3 sum{0.0f, 0.0f, 0.0f};
        if (flags & kPathDeferAnalytic) {
            const float4 vis = SlotVisibility<kTransmittance>(q, transmittance, 3 * path + 1);
            if (vis.w == 1.0f) sum = sum + Mul(F4(ps.nee[3 * path + 1]), F4(vis));
            ps.nee[3 * path + 1] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        if (flags & kPathDeferEnvironment) {
            const float4 vis = SlotVisibility<kTransmittance>(q, transmittance, 3 * path + 2);
            if (vis.w == 1.0f) {
                const float4 fl = ps.nee[3 * path + 2];  // BSDF x radiance, environment pdf
                const float4 dc = v[4];                  // direction, cosine
                const float pb = PdfBsdf(m, wo, F4(dc), n, rng);
                const float mis = PowerHeuristic(1, fl.w, 1, pb);
                sum = sum + Mul(F4(fl), F4(vis)) * (dc.w * mis / fl.w);
            }
            ps.nee[3 * path + 2] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        flags &= ~(kPathDeferAnalytic | kPathDeferEnvironment);
        const V3 tp = F4(ps.throughput[path]);
        const V3 rad = F4(ps.radiance[path]) + Mul(tp, sum);
        ContinuePath(sc, ps, q, path, depth, m, material, p, n, wo, tp, rad, flags, smp, rng);
    }
}

// Empties the shadow queue between the two shadow stages of a bounce (the
// first stage's results stay in their slots).
__global__ void ResetShadowQueueKernel(Queues q) {
    if (threadIdx.x == 0) {
        q.counters[kCtrShadow] = 0;
        q.counters[kCtrShadowTrace] = 0;
        q.counters[kCtrShadowOverflow] = 0;
    }
}

// ---------------------------------------------------------- subsurface

// The exit half of the subsurface branch (path_integrator.cpp:136-170,
// bssrdf_probe.cpp:61-90): for each probe, the exit point among the target
// hits the probe stage selected, Sp / pdf, next-event estimation at the exit
// through the normalised Fresnel-weighted cosine lobe (Sw), and the
// continuation sampled from that lobe.
__global__ void __launch_bounds__(256, 2) SubsurfaceExitKernel(DevScene sc, PathState ps, Queues q, int depth) {
    const int64_t n = static_cast<int64_t>(q.counters[kCtrProbe]);
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t hits = q.probe_count[k];
        if (hits <= 0) continue;  // no exit: the path ends
        const int32_t path = q.probe_target[k].w;
        const float4 h = q.probe_hit[k];
        const int32_t id = __float_as_int(h.y);
        const V3 base = F4(q.probe_ray[2 * k]), vz = F4(q.probe_ray[2 * k + 1]);
        const V3 pi = base + vz * h.x;
        V3 ni;
        if (id >= 0) {  // GeometricNormal of the triangle, object space (intersection.cpp:75-82)
            const int4 tv = sc.tri_vertices[id];
            const V3 p0 = VertexPos(sc, tv.x), p1 = VertexPos(sc, tv.y), p2 = VertexPos(sc, tv.z);
            ni = Normalize(Cross(p1 - p0, p2 - p0));
        } else {  // SphereNormal (intersection.cpp:136-143)
            const float4 c = sc.spheres[-2 - id];
            ni = Normalize(V3{pi.x - c.x, pi.y - c.y, pi.z - c.z});
        }
        const float4 e0 = q.probe_entry[2 * k], e1 = q.probe_entry[2 * k + 1];
        const V3 po = F4(e0), ns = F4(e1);
        const DevMaterial& dm = sc.materials[__float_as_int(e1.w)];
        V3 ss, ts;
        BssrdfFrame(ns, ss, ts);
        const TabBssrdf tab = MakeTabBssrdf(dm, sc.bssrdf[dm.bssrdf_index]);
        const V3 sp = BssrdfSr(tab, sqrtf(LengthSq(po - pi)));
        const float pdf = BssrdfPdfSp(tab, po, ss, ts, ns, pi, ni) / static_cast<float>(hits);
        if (!(pdf > 0.0f)) continue;
        V3 tp = F4(ps.throughput[path]);
        tp = Mul(tp, V3{sp.x / pdf, sp.y / pdf, sp.z / pdf});
        if (IsBlack(tp)) {
            ps.throughput[path] = ToF4(tp);
            continue;
        }
        Mat mx{};
        mx.kind = kSubsurfaceExit;
        mx.ior = dm.bssrdf_eta;
        uint32_t flags = ps.flags[path];
        PixelSampler smp;
        const int32_t pixel = ps.pixel[path];
        smp.Init(sc.sampler, sc.view->seed, pixel % sc.width, pixel / sc.width, ps.sample[path], sc.spp);
        Pcg32 rng{ps.rng_state[path], ps.rng_inc[path]};
        NextEvent(sc, ps, q, path, smp, rng, depth, mx, pi, ni, ni, tp, flags);
        float bx, by;
        smp.Sample2D(kDimBssrdfExitBsdf, depth, bx, by);
        const BsdfSample bs = SampleBsdf(mx, ni, ni, bx, by, rng);
        bool cont = bs.valid && !IsBlack(bs.weight);
        if (cont) {
            tp = Mul(tp, bs.weight);
            if (depth >= 3) {  // SurviveRussianRoulette
                const float survival = Clampf(MaxComp(tp), 0.05f, 0.95f);
                if (smp.Sample1D(kDimRussianRoulette, depth) >= survival) {
                    cont = false;
                } else {
                    tp = tp / survival;
                }
            }
        }
        if (cont) {
            flags = (flags | kPathPrevValid) & ~kPathPrevDelta;
            ps.prev[path] = ToF4(pi, bs.pdf);
            const V3 bn = Dot(bs.wi, ni) >= 0.0f ? ni : -ni;
            const V3 no = pi + bn * SurfaceBias(pi);
            const unsigned long long o = QueueAppend(q.counters + kCtrOut);
            q.ray_out[2 * o] = make_float4(no.x, no.y, no.z, 1.0e-5f);
            q.ray_out[2 * o + 1] = make_float4(bs.wi.x, bs.wi.y, bs.wi.z, __int_as_float(0x7f800000));
            q.path_out[o] = path;
        }
        ps.throughput[path] = ToF4(tp);
        ps.flags[path] = flags;
        ps.rng_state[path] = rng.state;
    }
}

// ------------------------------------------------------- radiance cache

// The image estimate of every path that ended at the cache: its radiance up
// to the query vertex plus throughput x cached radiance. Runs after the
// training targets were taken from the training paths' full radiance.
__global__ void CacheResolveKernel(PathState ps, CacheArgs cache) {
    const int64_t n = static_cast<int64_t>(cache.counters[0]);
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t path = cache.query_path[k];
        V3 c = F4(cache.query_rgb[k]);
        if (!(isfinite(c.x) && isfinite(c.y) && isfinite(c.z))) c = V3{0.0f, 0.0f, 0.0f};
        ps.radiance[path] = ToF4(F4(cache.query_base[k]) + Mul(F4(cache.query_tp[k]), c));
    }
}

// Training records of the unbiased training paths: for each recorded vertex,
// target = (final path radiance - radiance before the vertex's reflected
// light) / throughput at the vertex, i.e. a one-sample estimate of the
// radiance the vertex reflects towards the previous one.
__global__ void CacheTargetsKernel(PathState ps, CacheArgs cache) {
    const int64_t slots = static_cast<int64_t>(
        min(cache.counters[1], static_cast<unsigned long long>(cache.train_paths)));
    for (int64_t slot = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; slot < slots;
         slot += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t path = cache.slot_path[slot];
        const V3 L = F4(ps.radiance[path]);
        const int32_t len = cache.slot_len[slot];
        for (int32_t k = 0; k < len; ++k) {
            const int64_t v = slot * cache.max_depth + k;
            const V3 lb = F4(cache.slot_lt[2 * v]);
            const V3 t = F4(cache.slot_lt[2 * v + 1]);
            V3 target{t.x > 1.0e-8f ? fmaxf(L.x - lb.x, 0.0f) / t.x : 0.0f,
                      t.y > 1.0e-8f ? fmaxf(L.y - lb.y, 0.0f) / t.y : 0.0f,
                      t.z > 1.0e-8f ? fmaxf(L.z - lb.z, 0.0f) / t.z : 0.0f};
            // Rare numerically extreme samples would dominate the optimiser's
            // moment estimates: bound each target's largest component.
            const float mc = MaxComp(target);
            if (mc > cache.target_max) target = target * (cache.target_max / mc);
            if (!(isfinite(target.x) && isfinite(target.y) && isfinite(target.z))) continue;
            const unsigned long long r = atomicAdd(cache.counters + 2, 1ull);
            if (r >= static_cast<unsigned long long>(cache.train_records)) break;
            const float4* src = reinterpret_cast<const float4*>(cache.slot_q + 16 * v);
            float4* dst = reinterpret_cast<float4*>(cache.rec_q + 16 * r);
            dst[0] = src[0];
            dst[1] = src[1];
            dst[2] = src[2];
            dst[3] = src[3];
            cache.rec_t[r] = ToF4(target);
        }
    }
}

// ------------------------------------------------------------------- film

// Film::AddSample in sample order for each active pixel (film.cpp:160-183),
// with the radiance clamp of IntegratePathSample (path_integrator.cpp:195).
// A batch rendered `batch` consecutive sample indices per pixel on the
// assumption that every sample is finite; accepting stops at the first
// non-finite one (the reference re-uses that sample index on its next pass)
// or when adaptive sampling declares the pixel converged.
// The film's sample count summed over the pixels (RenderStats::samples_rendered)
// into *out, one atomic per warp.
__global__ void SumSamplesKernel(const yrc_film_pixel* film, int64_t pixels, unsigned long long* out) {
    unsigned long long n = 0;
    for (int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; p < pixels;
         p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        n += film[p].samples;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31u) == 0 && n) atomicAdd(out, n);
}

__global__ void FilmKernel(DevScene sc, PathState ps, BatchArgs b, FilmArgs f) {
    const int64_t n_active = static_cast<int64_t>(*b.active_count);
    const int32_t batch = *b.batch;
    for (int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; p < n_active;
         p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t pixel = b.active[p];
        yrc_film_pixel px = b.film[pixel];
        int32_t attempts = f.attempts_left[pixel];
        for (int32_t j = 0; j < batch && attempts > 0; ++j) {
            const int64_t slot = j * n_active + p;
            V3 beauty = F4(ps.radiance[slot]);
            // ClampMaxComponent (path_integrator_common.cpp:37-46)
            if (sc.radiance_clamp > 0.0f) {
                const float mc = MaxComp(beauty);
                if (!(mc <= sc.radiance_clamp || mc <= 0.0f)) beauty = beauty * (sc.radiance_clamp / mc);
            }
            --attempts;
            if (!(isfinite(beauty.x) && isfinite(beauty.y) && isfinite(beauty.z))) {
                atomicAdd(f.bad_samples, 1ull);
                break;
            }
            px.sum[0] = px.sum[0] + beauty.x;
            px.sum[1] = px.sum[1] + beauty.y;
            px.sum[2] = px.sum[2] + beauty.z;
            ++px.samples;
            const float lum = 0.2126f * beauty.x + 0.7152f * beauty.y + 0.0722f * beauty.z;
            const float delta = lum - px.luminance_mean;
            px.luminance_mean += delta / static_cast<float>(px.samples);
            const float delta2 = lum - px.luminance_mean;
            px.luminance_m2 += delta * delta2;
            if (ps.flags[slot] & kPathPrimary) {
                const float4 al = ps.aov_albedo[slot];
                const float4 nm = ps.aov_normal[slot];
                const float depth = al.w;
                if (isfinite(al.x) && isfinite(al.y) && isfinite(al.z) && isfinite(nm.x) && isfinite(nm.y) &&
                    isfinite(nm.z) && isfinite(depth) && depth >= 0.0f) {
                    px.albedo_sum[0] = px.albedo_sum[0] + al.x;
                    px.albedo_sum[1] = px.albedo_sum[1] + al.y;
                    px.albedo_sum[2] = px.albedo_sum[2] + al.z;
                    px.normal_sum[0] = px.normal_sum[0] + nm.x;
                    px.normal_sum[1] = px.normal_sum[1] + nm.y;
                    px.normal_sum[2] = px.normal_sum[2] + nm.z;
                    px.depth_sum += depth;
                    ++px.aov_samples;
                }
            }
            if (px.samples >= static_cast<uint32_t>(sc.spp)) break;
            if (f.adaptive && px.samples >= static_cast<uint32_t>(max(2, f.min_spp))) {
                // Film::IsConverged (film.cpp:113-121)
                const float var = px.samples > 1 ? px.luminance_m2 / static_cast<float>(px.samples - 1) : 0.0f;
                const float se = px.samples > 1 ? sqrtf(fmaxf(0.0f, var) / static_cast<float>(px.samples))
                                                : __int_as_float(0x7f800000);
                const float bound = fmaxf(0.0f, f.confidence) * se;
                const float tol = fmaxf(0.0f, f.absolute_error) + fmaxf(0.0f, f.relative_error) * fabsf(px.luminance_mean);
                if (isfinite(bound) && bound <= tol) break;
            }
        }
        b.film[pixel] = px;
        f.attempts_left[pixel] = attempts;
    }
}

// Rebuilds the active-pixel list: pixels with attempts left, fewer than spp
// samples and (with adaptive sampling) not converged; also counts converged
// pixels. Order is irrelevant: every pixel's samples are independent.
__global__ void ActivePixelsKernel(DevScene sc, BatchArgs b, FilmArgs f, int64_t pixels) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < pixels;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const yrc_film_pixel px = b.film[i];
        bool converged = false;
        if (f.adaptive && px.samples >= static_cast<uint32_t>(max(2, f.min_spp))) {
            const float var = px.samples > 1 ? px.luminance_m2 / static_cast<float>(px.samples - 1) : 0.0f;
            const float se = px.samples > 1 ? sqrtf(fmaxf(0.0f, var) / static_cast<float>(px.samples))
                                            : __int_as_float(0x7f800000);
            const float bound = fmaxf(0.0f, f.confidence) * se;
            const float tol = fmaxf(0.0f, f.absolute_error) + fmaxf(0.0f, f.relative_error) * fabsf(px.luminance_mean);
            converged = isfinite(bound) && bound <= tol;
        }
        if (converged) atomicAdd(f.converged, 1ull);
        if (!converged && px.samples < static_cast<uint32_t>(sc.spp) && f.attempts_left[i] > 0) {
            const unsigned long long k = QueueAppend(b.active_count_next);
            b.active[k] = static_cast<int32_t>(i);
        }
    }
}

// Publishes the rebuilt active list and sizes the next batch: as many sample
// attempts per active pixel as fit in the path-state capacity (at least 1).
__global__ void FinishActiveKernel(unsigned long long* active_count, unsigned long long* next, int32_t* batch,
                                   int32_t max_batch, int64_t capacity) {
    if (threadIdx.x == 0) {
        const unsigned long long n = *next;
        *active_count = n;
        *next = 0;
        int64_t b = n > 0 ? capacity / static_cast<int64_t>(n) : 1;
        if (b > max_batch) b = max_batch;
        if (b < 1) b = 1;
        *batch = static_cast<int32_t>(b);
    }
}

namespace {
constexpr int kThreads = 256;
unsigned Grid(int64_t work, int sm_count, int per_sm = 8) {
    int64_t blocks = (work + kThreads - 1) / kThreads;
    const int64_t cap = static_cast<int64_t>(sm_count) * per_sm;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    return static_cast<unsigned>(blocks);
}
}  // namespace

void LaunchGenerate(const DevScene& sc, const PathState& ps, const Queues& q, const BatchArgs& b,
                    const CacheArgs& cache, int64_t capacity, int sm_count, cudaStream_t st) {
    GenerateKernel<<<Grid(capacity, sm_count), kThreads, 0, st>>>(sc, ps, q, b, cache);
}
void LaunchResetCounters(const Queues& q, cudaStream_t st) { ResetCountersKernel<<<1, 32, 0, st>>>(q); }
void LaunchAdvanceQueue(const Queues& q, cudaStream_t st) { AdvanceQueueKernel<<<1, 32, 0, st>>>(q); }
void LaunchShade(const DevScene& sc, const PathState& ps, const Queues& q, const CacheArgs& cache, int depth,
                 int64_t capacity, int sm_count, cudaStream_t st) {
    LaunchShadeSort(sc, ps, q, depth, capacity, sm_count, st);
    LaunchShadeClasses(sc, ps, q, cache, depth, capacity, sm_count, st);
}
void LaunchShadeSort(const DevScene& sc, const PathState& ps, const Queues& q, int depth, int64_t capacity,
                     int sm_count, cudaStream_t st) {
    if (sc.texture_count > 0) SurfaceTextureKernel<<<Grid(capacity, sm_count), kThreads, 0, st>>>(sc, ps, q, depth);
    ClassifyKernel<<<Grid(capacity, sm_count), kThreads, 0, st>>>(sc, q);
    ScatterByClassKernel<<<Grid(capacity, sm_count), kThreads, 0, st>>>(q);
}
void LaunchPooledShade(const ShadeJob* jobs, int njobs, int64_t capacity, int sm_count, cudaStream_t st) {
    if (njobs <= 0) return;
    const unsigned grid = Grid(capacity, sm_count);
    PooledShadeKernel<kClassMiss><<<grid, kThreads, 0, st>>>(jobs, njobs);
    PooledShadeKernel<kClassDiffuse><<<grid, kThreads, 0, st>>>(jobs, njobs);
    PooledShadeKernel<kClassConductor><<<grid, kThreads, 0, st>>>(jobs, njobs);
    PooledShadeKernel<kClassDielectric><<<grid, kThreads, 0, st>>>(jobs, njobs);
    PooledShadeKernel<kClassCoatedDiffuse><<<grid, kThreads, 0, st>>>(jobs, njobs);
    PooledShadeKernel<kClassGeneric><<<grid, kThreads, 0, st>>>(jobs, njobs);
}
// Host mirror of the device checks that the lean shading instances drop:
// no analytic light, no sampleable environment (EnvSampleable), no cache.
static bool ShadeLean(const DevScene& sc, const CacheArgs& cache) {
    const bool env = sc.env.active && sc.env.strength > 0.0f && sc.env.texels && sc.env.texel_weights;
    return sc.analytic_count == 0 && !env && !cache.enabled;
}
template <bool kLean>
static void LaunchShadeClassesOf(const DevScene& sc, const PathState& ps, const Queues& q, const CacheArgs& cache,
                                 int depth, int64_t capacity, int sm_count, cudaStream_t st) {
    const unsigned grid = Grid(capacity, sm_count);
    ShadeKernel<kClassMiss, kLean><<<grid, kThreads, 0, st>>>(sc, ps, q, depth, cache);
    ShadeKernel<kClassDiffuse, kLean><<<grid, kThreads, 0, st>>>(sc, ps, q, depth, cache);
    ShadeKernel<kClassConductor, kLean><<<grid, kThreads, 0, st>>>(sc, ps, q, depth, cache);
    ShadeKernel<kClassDielectric, kLean><<<grid, kThreads, 0, st>>>(sc, ps, q, depth, cache);
    ShadeKernel<kClassCoatedDiffuse, kLean><<<grid, kThreads, 0, st>>>(sc, ps, q, depth, cache);
    ShadeKernel<kClassGeneric, kLean><<<grid, kThreads, 0, st>>>(sc, ps, q, depth, cache);
}
void LaunchShadeClasses(const DevScene& sc, const PathState& ps, const Queues& q, const CacheArgs& cache, int depth,
                        int64_t capacity, int sm_count, cudaStream_t st) {
    if (ShadeLean(sc, cache)) {
        LaunchShadeClassesOf<true>(sc, ps, q, cache, depth, capacity, sm_count, st);
    } else {
        LaunchShadeClassesOf<false>(sc, ps, q, cache, depth, capacity, sm_count, st);
    }
}
template <bool kTwo, int kTotal>
void LaunchAlphaOne(const DevScene& sc, const PathState& ps, const Queues& q, int depth, int64_t capacity,
                    int sm_count, int* error, float4* transmittance, unsigned long long* occluded_count,
                    bool shadows, const int32_t* list, cudaStream_t st) {
    const unsigned blocks = static_cast<unsigned>(std::min<int64_t>((capacity + kTraceBlock - 1) / kTraceBlock,
                                                                    static_cast<int64_t>(sm_count) * 16));
    if (shadows) {
        // An overflow list is rare and short: one block per SM covers it.
        const unsigned grid = list ? static_cast<unsigned>(sm_count) : blocks * 2;
        ShadowExactKernel<kTwo, kTotal><<<grid, kTraceBlock, 0, st>>>(sc, q, list, transmittance, occluded_count, error);
    } else {
        AlphaExtendKernel<kTwo, kTotal><<<blocks, kTraceBlock, 0, st>>>(sc, ps, q, depth, error);
    }
}

void LaunchAlpha(const DevScene& sc, const PathState& ps, const Queues& q, int depth, int64_t capacity, int sm_count,
                 int* error, float4* transmittance, unsigned long long* occluded_count, bool shadows,
                 const int32_t* list, cudaStream_t st) {
    const bool two = sc.accel.two_level != 0;
    const bool deep = sc.accel.stack_limit > 64;
    if (two) {
        if (deep) LaunchAlphaOne<true, kMaxTraceStack>(sc, ps, q, depth, capacity, sm_count, error, transmittance, occluded_count, shadows, list, st);
        else LaunchAlphaOne<true, 64>(sc, ps, q, depth, capacity, sm_count, error, transmittance, occluded_count, shadows, list, st);
    } else {
        if (deep) LaunchAlphaOne<false, kMaxTraceStack>(sc, ps, q, depth, capacity, sm_count, error, transmittance, occluded_count, shadows, list, st);
        else LaunchAlphaOne<false, 64>(sc, ps, q, depth, capacity, sm_count, error, transmittance, occluded_count, shadows, list, st);
    }
}

void LaunchAlphaExtend(const DevScene& sc, const PathState& ps, const Queues& q, int depth, int64_t capacity,
                       int sm_count, int* error, cudaStream_t st) {
    LaunchAlpha(sc, ps, q, depth, capacity, sm_count, error, nullptr, nullptr, false, nullptr, st);
}

void LaunchShadowExact(const DevScene& sc, const Queues& q, float4* transmittance, unsigned long long* occluded_count,
                       int64_t capacity, int sm_count, int* error, cudaStream_t st, const int32_t* list) {
    LaunchAlpha(sc, PathState{}, q, 0, capacity, sm_count, error, transmittance, occluded_count, true, list, st);
}

void LaunchSubsurfaceExit(const DevScene& sc, const PathState& ps, const Queues& q, int depth, int64_t capacity,
                          int sm_count, cudaStream_t st) {
    SubsurfaceExitKernel<<<Grid(capacity, sm_count), kThreads, 0, st>>>(sc, ps, q, depth);
}
void LaunchCacheResolve(const PathState& ps, const CacheArgs& cache, int64_t capacity, int sm_count,
                        cudaStream_t st) {
    CacheResolveKernel<<<Grid(capacity, sm_count), kThreads, 0, st>>>(ps, cache);
}
void LaunchCacheTargets(const PathState& ps, const CacheArgs& cache, int sm_count, cudaStream_t st) {
    CacheTargetsKernel<<<Grid(cache.train_paths, sm_count), kThreads, 0, st>>>(ps, cache);
}
void LaunchLayeredNee(const DevScene& sc, const PathState& ps, const Queues& q, const float4* transmittance,
                      int depth, int64_t capacity, int sm_count, cudaStream_t st) {
    ResetShadowQueueKernel<<<1, 32, 0, st>>>(q);
    if (transmittance) {
        LayeredNeeKernel<true><<<Grid(capacity, sm_count), kThreads, 0, st>>>(sc, ps, q, transmittance, depth);
    } else {
        LayeredNeeKernel<false><<<Grid(capacity, sm_count), kThreads, 0, st>>>(sc, ps, q, transmittance, depth);
    }
}
void LaunchLayeredContinue(const DevScene& sc, const PathState& ps, const Queues& q, const float4* transmittance,
                           int depth, int64_t capacity, int sm_count, cudaStream_t st) {
    if (transmittance) {
        LayeredContinueKernel<true><<<Grid(capacity, sm_count), kThreads, 0, st>>>(sc, ps, q, transmittance, depth);
    } else {
        LayeredContinueKernel<false><<<Grid(capacity, sm_count), kThreads, 0, st>>>(sc, ps, q, transmittance, depth);
    }
}
void LaunchNeeResolve(const PathState& ps, const Queues& q, const float4* transmittance, int64_t capacity,
                      int sm_count, cudaStream_t st) {
    if (transmittance) {
        NeeResolveKernel<true><<<Grid(capacity, sm_count), kThreads, 0, st>>>(ps, q, transmittance);
    } else {
        NeeResolveKernel<false><<<Grid(capacity, sm_count), kThreads, 0, st>>>(ps, q, nullptr);
    }
}
void LaunchFilm(const DevScene& sc, const PathState& ps, const BatchArgs& b, const FilmArgs& f, int64_t pixels,
                int sm_count, cudaStream_t st) {
    FilmKernel<<<Grid(pixels, sm_count), kThreads, 0, st>>>(sc, ps, b, f);
}
__global__ void FillInt32Kernel(int32_t* dst, int64_t n, int32_t value) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        dst[i] = value;
    }
}
void LaunchFillInt32(int32_t* dst, int64_t n, int32_t value, int sm_count, cudaStream_t st) {
    FillInt32Kernel<<<Grid(n, sm_count), kThreads, 0, st>>>(dst, n, value);
}
void LaunchActivePixels(const DevScene& sc, const BatchArgs& b, const FilmArgs& f, int64_t pixels, int sm_count,
                        cudaStream_t st) {
    ActivePixelsKernel<<<Grid(pixels, sm_count), kThreads, 0, st>>>(sc, b, f, pixels);
}
void LaunchFinishActive(unsigned long long* active_count, unsigned long long* active_count_next, int32_t* batch,
                        int32_t max_batch, int64_t capacity, cudaStream_t st) {
    FinishActiveKernel<<<1, 32, 0, st>>>(active_count, active_count_next, batch, max_batch, capacity);
}

void LaunchSumSamples(const yrc_film_pixel* film, int64_t pixels, unsigned long long* out, int sm_count,
                      cudaStream_t st) {
    SumSamplesKernel<<<Grid(pixels, sm_count), kThreads, 0, st>>>(film, pixels, out);
}

}  // namespace yrc
