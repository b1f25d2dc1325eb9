// Device BSDF, light-sampling and environment math of the reference path
// tracer, used by the wavefront shade stages. This translation unit is
// compiled with -fmad=false so every a*b+c rounds twice as in the reference's
// SSE2 build; sqrt and division are IEEE. Transcendentals (cos, sin, exp,
// log, pow, acos, atan2, tan) are CUDA's, whose last-ulp results differ from
// the host libm, so renders match the CPU backend statistically (per-pixel
// relMSE), not bit for bit.
#pragma once

#include <cstdint>

#include "render_types.hpp"

namespace yrc {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kTwoPi = 2.0f * kPi;
constexpr float kDeltaRoughness = 1.0e-3f;

struct V3 {
    float x, y, z;
};

__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ V3 Mul(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ float Dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 Cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float LengthSq(V3 v) { return Dot(v, v); }
// Normalize (vec.hpp:175-178): v / |v|, zero vector when |v| == 0.
__device__ __forceinline__ V3 Normalize(V3 v) {
    const float len = sqrtf(LengthSq(v));
    return len > 0.0f ? v / len : V3{0.0f, 0.0f, 0.0f};
}
__device__ __forceinline__ bool IsBlack(V3 c) { return c.x <= 0.0f && c.y <= 0.0f && c.z <= 0.0f; }
__device__ __forceinline__ float MaxComp(V3 c) { return fmaxf(c.x, fmaxf(c.y, c.z)); }
__device__ __forceinline__ float Clampf(float v, float lo, float hi) { return v < lo ? lo : (hi < v ? hi : v); }
__device__ __forceinline__ V3 Ld3(const float* p) { return {p[0], p[1], p[2]}; }

// ------------------------------------------------------------ BSDF helpers
// (src/shading/bsdf_common.cpp, bsdf_microfacet.cpp)

__device__ __forceinline__ bool IsAbove(V3 d, V3 n) { return Dot(d, n) > 0.0f; }

__device__ __forceinline__ V3 Reflect(V3 d, V3 n) { return Normalize(d - n * (2.0f * Dot(d, n))); }

__device__ inline float FresnelDielectric(float cos_i, float eta_i, float eta_t) {
    cos_i = Clampf(cos_i, -1.0f, 1.0f);
    if (cos_i <= 0.0f) {
        const float tmp = eta_i;
        eta_i = eta_t;
        eta_t = tmp;
        cos_i = fabsf(cos_i);
    }
    const float sin_i = sqrtf(fmaxf(0.0f, 1.0f - cos_i * cos_i));
    const float sin_t = eta_i / eta_t * sin_i;
    if (sin_t >= 1.0f) return 1.0f;
    const float cos_t = sqrtf(fmaxf(0.0f, 1.0f - sin_t * sin_t));
    const float rpar = ((eta_t * cos_i) - (eta_i * cos_t)) / ((eta_t * cos_i) + (eta_i * cos_t));
    const float rper = ((eta_i * cos_i) - (eta_t * cos_t)) / ((eta_i * cos_i) + (eta_t * cos_t));
    return 0.5f * (rpar * rpar + rper * rper);
}

__device__ inline bool Refract(V3 wo, V3 n, float eta, V3& wi) {
    const float cos_i = Dot(n, wo);
    const float sin2_i = fmaxf(0.0f, 1.0f - cos_i * cos_i);
    const float sin2_t = eta * eta * sin2_i;
    if (sin2_t >= 1.0f) return false;
    const float cos_t = sqrtf(fmaxf(0.0f, 1.0f - sin2_t));
    wi = Normalize(-wo * eta + n * (eta * cos_i - cos_t));
    return true;
}

__device__ __forceinline__ float AbsDot(V3 a, V3 b) { return fabsf(Dot(a, b)); }

// Orthonormal basis used by the hemisphere samplers.
__device__ __forceinline__ void Basis(V3 n, V3& t, V3& b) {
    const V3 helper = fabsf(n.z) < 0.999f ? V3{0.0f, 0.0f, 1.0f} : V3{1.0f, 0.0f, 0.0f};
    t = Normalize(Cross(helper, n));
    b = Cross(n, t);
}

// SampleCosineHemisphere (bsdf_microfacet.cpp:91-104): Malley's method.
__device__ inline V3 SampleCosineHemisphere(V3 n, float sx, float sy) {
    const float u1 = Clampf(sx, 0.0f, 1.0f);
    const float u2 = Clampf(sy, 0.0f, 1.0f);
    const float r = sqrtf(u1);
    const float theta = 2.0f * kPi * u2;
    float s, c;
    sincosf(theta, &s, &c);
    const float lx = r * c, ly = r * s, lz = sqrtf(fmaxf(0.0f, 1.0f - u1));
    V3 t, b;
    Basis(n, t, b);
    return Normalize(t * lx + b * ly + n * lz);
}

__device__ __forceinline__ float RoughnessToAlpha(float r) {
    const float c = fmaxf(kDeltaRoughness, r);
    return c * c;
}

__device__ __forceinline__ float GgxD(float cos_h, float alpha) {
    const float cos2 = cos_h * cos_h;
    const float a2 = alpha * alpha;
    const float denom = cos2 * (a2 - 1.0f) + 1.0f;
    return a2 / (kPi * denom * denom);
}

__device__ __forceinline__ float SmithG1(float cos_t, float alpha) {
    const float cos2 = cos_t * cos_t;
    if (cos2 <= 0.0f) return 0.0f;
    const float tan2 = (1.0f - cos2) / cos2;
    return 2.0f / (1.0f + sqrtf(1.0f + alpha * alpha * tan2));
}

// SchlickFresnel (bsdf_microfacet.cpp:143-146): Lerp(f0, 1, (1-cos)^5).
__device__ __forceinline__ V3 Schlick(V3 f0, float cos_t) {
    const float t = powf(1.0f - Clampf(cos_t, 0.0f, 1.0f), 5.0f);
    return f0 * (1.0f - t) + V3{1.0f, 1.0f, 1.0f} * t;
}

__device__ inline V3 GgxSpecularBrdf(V3 f0, float roughness, V3 wo, V3 wi, V3 n) {
    if (!IsAbove(wo, n) || !IsAbove(wi, n)) return {0, 0, 0};
    const V3 h = Normalize(wo + wi);
    if (LengthSq(h) <= 0.0f || !IsAbove(h, n)) return {0, 0, 0};
    const float co = fmaxf(0.0f, Dot(n, wo)), ci = fmaxf(0.0f, Dot(n, wi));
    const float ch = fmaxf(0.0f, Dot(n, h)), coh = fmaxf(0.0f, Dot(wo, h));
    if (co <= 0.0f || ci <= 0.0f || coh <= 0.0f) return {0, 0, 0};
    const float alpha = RoughnessToAlpha(roughness);
    const float d = GgxD(ch, alpha);
    const float g = SmithG1(co, alpha) * SmithG1(ci, alpha);
    return Schlick(f0, coh) * (d * g / (4.0f * co * ci));
}

__device__ inline float GgxReflectionPdf(float roughness, V3 wo, V3 wi, V3 n) {
    if (!IsAbove(wo, n) || !IsAbove(wi, n)) return 0.0f;
    const V3 h = Normalize(wo + wi);
    if (LengthSq(h) <= 0.0f || !IsAbove(h, n)) return 0.0f;
    const float ch = fmaxf(0.0f, Dot(n, h)), coh = fmaxf(0.0f, Dot(wo, h));
    if (ch <= 0.0f || coh <= 0.0f) return 0.0f;
    return GgxD(ch, RoughnessToAlpha(roughness)) * ch / (4.0f * coh);
}

__device__ __forceinline__ bool SameHemisphere(V3 a, V3 b, V3 n) { return Dot(a, n) * Dot(b, n) > 0.0f; }

__device__ inline V3 GgxDielectricReflection(V3 albedo, float ior, float roughness, V3 wo, V3 wi, V3 n) {
    if (!SameHemisphere(wo, wi, n)) return {0, 0, 0};
    const V3 on = Dot(n, wo) >= 0.0f ? n : -n;
    const V3 h = Normalize(wo + wi);
    if (LengthSq(h) <= 0.0f || Dot(h, on) <= 0.0f) return {0, 0, 0};
    const float co = AbsDot(on, wo), ci = AbsDot(on, wi), ch = AbsDot(on, h), coh = AbsDot(wo, h);
    if (co <= 0.0f || ci <= 0.0f || coh <= 0.0f) return {0, 0, 0};
    const float alpha = RoughnessToAlpha(roughness);
    const float d = GgxD(ch, alpha);
    const float g = SmithG1(co, alpha) * SmithG1(ci, alpha);
    const float f = FresnelDielectric(coh, 1.0f, fmaxf(1.0f, ior));
    return albedo * (f * d * g / (4.0f * co * ci));
}

__device__ inline float GgxDielectricReflectionPdf(float ior, float roughness, V3 wo, V3 wi, V3 n) {
    if (!SameHemisphere(wo, wi, n)) return 0.0f;
    const V3 on = Dot(n, wo) >= 0.0f ? n : -n;
    const V3 h = Normalize(wo + wi);
    if (LengthSq(h) <= 0.0f || Dot(h, on) <= 0.0f) return 0.0f;
    const float ch = AbsDot(on, h), coh = AbsDot(wo, h);
    if (ch <= 0.0f || coh <= 0.0f) return 0.0f;
    const float f = FresnelDielectric(coh, 1.0f, fmaxf(1.0f, ior));
    return f * GgxD(ch, RoughnessToAlpha(roughness)) * ch / (4.0f * coh);
}

__device__ inline V3 TransmissionHalf(V3 wo, V3 wi, V3 n, float ior) {
    const bool entering = Dot(n, wo) >= 0.0f;
    const float ei = entering ? 1.0f : fmaxf(1.0f, ior);
    const float et = entering ? fmaxf(1.0f, ior) : 1.0f;
    const float eta = et / ei;
    V3 h = Normalize(wo + wi * eta);
    if (Dot(h, n) < 0.0f) h = -h;
    return h;
}

__device__ inline V3 GgxDielectricTransmission(V3 albedo, float ior, float roughness, V3 wo, V3 wi, V3 n) {
    if (SameHemisphere(wo, wi, n)) return {0, 0, 0};
    const bool entering = Dot(n, wo) >= 0.0f;
    const V3 on = entering ? n : -n;
    const float ei = entering ? 1.0f : fmaxf(1.0f, ior);
    const float et = entering ? fmaxf(1.0f, ior) : 1.0f;
    const float eta = et / ei;
    const V3 h = TransmissionHalf(wo, wi, on, ior);
    if (LengthSq(h) <= 0.0f || Dot(h, on) <= 0.0f) return {0, 0, 0};
    const float co = AbsDot(on, wo), ci = AbsDot(on, wi), ch = AbsDot(on, h);
    const float woh = Dot(wo, h), wih = Dot(wi, h);
    const float sd = woh + eta * wih;
    if (co <= 0.0f || ci <= 0.0f || ch <= 0.0f || woh <= 0.0f || wih >= 0.0f || sd == 0.0f) return {0, 0, 0};
    const float alpha = RoughnessToAlpha(roughness);
    const float d = GgxD(ch, alpha);
    const float g = SmithG1(co, alpha) * SmithG1(ci, alpha);
    const float f = FresnelDielectric(fabsf(woh), ei, et);
    const float num = fabsf(wih) * fabsf(woh) * eta * eta;
    const float den = co * ci * sd * sd;
    return albedo * ((1.0f - f) * d * g * num / den);
}

__device__ inline float GgxDielectricTransmissionPdf(float ior, float roughness, V3 wo, V3 wi, V3 n) {
    if (SameHemisphere(wo, wi, n)) return 0.0f;
    const bool entering = Dot(n, wo) >= 0.0f;
    const V3 on = entering ? n : -n;
    const float ei = entering ? 1.0f : fmaxf(1.0f, ior);
    const float et = entering ? fmaxf(1.0f, ior) : 1.0f;
    const float eta = et / ei;
    const V3 h = TransmissionHalf(wo, wi, on, ior);
    if (LengthSq(h) <= 0.0f || Dot(h, on) <= 0.0f) return 0.0f;
    const float ch = AbsDot(on, h);
    const float woh = Dot(wo, h), wih = Dot(wi, h);
    const float sd = woh + eta * wih;
    if (ch <= 0.0f || woh <= 0.0f || wih >= 0.0f || sd == 0.0f) return 0.0f;
    const float f = FresnelDielectric(fabsf(woh), ei, et);
    const float dwh = fabsf((eta * eta * wih) / (sd * sd));
    return (1.0f - f) * GgxD(ch, RoughnessToAlpha(roughness)) * ch * dwh;
}

// SampleGgxHalfVector (bsdf_microfacet.cpp:311-328).
__device__ inline V3 SampleGgxHalf(V3 n, float roughness, float sx, float sy) {
    const float u1 = Clampf(sx, 0.0f, 0.999999f);
    const float u2 = Clampf(sy, 0.0f, 1.0f);
    const float alpha = RoughnessToAlpha(roughness);
    const float a2 = alpha * alpha;
    const float tan2 = a2 * u1 / fmaxf(1.0e-6f, 1.0f - u1);
    const float cos_t = 1.0f / sqrtf(1.0f + tan2);
    const float sin_t = sqrtf(fmaxf(0.0f, 1.0f - cos_t * cos_t));
    const float phi = 2.0f * kPi * u2;
    float s, c;
    sincosf(phi, &s, &c);
    V3 t, b;
    Basis(n, t, b);
    return Normalize(t * (sin_t * c) + b * (sin_t * s) + n * cos_t);
}

struct BsdfSample {
    V3 wi;
    V3 weight;
    float pdf;
    bool valid;
    bool specular;
};

__device__ __forceinline__ BsdfSample NoSample() { return BsdfSample{{0, 0, 0}, {0, 0, 0}, 0.0f, false, false}; }

__device__ inline BsdfSample SampleGgxReflection(V3 wo, V3 n, float sx, float sy, V3 f0, float roughness) {
    if (!IsAbove(wo, n) || IsBlack(f0)) return NoSample();
    const V3 h = SampleGgxHalf(n, roughness, sx, sy);
    const V3 wi = Reflect(-wo, h);
    if (!IsAbove(wi, n)) return NoSample();
    const float pdf = GgxReflectionPdf(roughness, wo, wi, n);
    if (pdf <= 0.0f) return NoSample();
    const V3 f = GgxSpecularBrdf(f0, roughness, wo, wi, n);
    const float ci = fmaxf(0.0f, Dot(n, wi));
    return BsdfSample{wi, f * (ci / pdf), pdf, true, false};
}

// ------------------------------------------------------------- environment
// (src/lighting/environment.cpp, bilinear texture lookup texture.cpp:116-130)

__device__ __forceinline__ float Fract(float v) { return v - floorf(v); }

__device__ inline void DirToEnvUv(V3 dir, float rotation, float& u, float& v) {
    const V3 d = Normalize(dir);
    const float phi = atan2f(d.x, d.z);
    u = Fract(0.5f + (phi + rotation) / kTwoPi);
    const float theta = acosf(Clampf(d.y, -1.0f, 1.0f));
    v = Clampf(theta / kPi, 0.0f, 1.0f);
}

__device__ inline V3 EnvUvToDir(float u, float v, float rotation) {
    const float phi = (u - 0.5f) * kTwoPi - rotation;
    const float theta = Clampf(v, 0.0f, 1.0f) * kPi;
    float st, ct, sp, cp;
    sincosf(theta, &st, &ct);
    sincosf(phi, &sp, &cp);
    return Normalize(V3{st * sp, ct, st * cp});
}

// Repeat-wrapped bilinear lookup of the environment texture.
__device__ inline V3 EnvTexture(const DevEnvironment& env, float u, float v) {
    const int w = env.width, h = env.height;
    if (w <= 0 || h <= 0) return {0, 0, 0};
    if (w == 1 && h == 1) return Ld3(env.texels);
    auto wrapf = [](float x) {
        const float f = x - floorf(x);
        return f < 0.0f ? f + 1.0f : f;
    };
    const float s = wrapf(u) * static_cast<float>(w) - 0.5f;
    const float t = wrapf(v) * static_cast<float>(h) - 0.5f;
    const int s0 = static_cast<int>(floorf(s)), t0 = static_cast<int>(floorf(t));
    const float ds = s - static_cast<float>(s0), dt = t - static_cast<float>(t0);
    auto texel = [&](int x, int y) {
        int ix = x % w;
        if (ix < 0) ix += w;
        int iy = y % h;
        if (iy < 0) iy += h;
        return Ld3(env.texels + 4 * (static_cast<int64_t>(iy) * w + ix));
    };
    const V3 c00 = texel(s0, t0), c10 = texel(s0 + 1, t0), c01 = texel(s0, t0 + 1), c11 = texel(s0 + 1, t0 + 1);
    const V3 a = c00 * (1.0f - ds) + c10 * ds;
    const V3 b = c01 * (1.0f - ds) + c11 * ds;
    return a * (1.0f - dt) + b * dt;
}

// EvaluateEnvironment (environment.cpp:125-148).
__device__ inline V3 EvalEnvironment(const DevEnvironment& env, V3 dir) {
    const V3 rad = Ld3(env.radiance);
    if (!env.active) return rad * env.strength;
    if (env.strength <= 0.0f || !env.texels) return {0, 0, 0};
    float u, v;
    DirToEnvUv(dir, env.rotation, u, v);
    const V3 s = EnvTexture(env, u, v);
    return V3{s.x * rad.x, s.y * rad.y, s.z * rad.z} * env.strength;
}

__device__ __forceinline__ bool EnvSampleable(const DevEnvironment& env) {
    return env.active && env.strength > 0.0f && env.texels && env.texel_weights;
}

// PdfEnvironment (environment.cpp:199-219): nearest-texel probability over
// the texel's solid angle.
__device__ inline float PdfEnvironment(const DevEnvironment& env, V3 dir) {
    if (!EnvSampleable(env)) return 0.0f;
    const int w = env.width, h = env.height;
    if (w <= 0 || h <= 0 || env.total_weight <= 0.0f) return 0.0f;
    float u, v;
    DirToEnvUv(dir, env.rotation, u, v);
    const int x = min(max(static_cast<int>(floorf(u * static_cast<float>(w))), 0), w - 1);
    const int y = min(max(static_cast<int>(floorf(v * static_cast<float>(h))), 0), h - 1);
    const float p = env.texel_weights[static_cast<int64_t>(y) * w + x] / env.total_weight;
    const float st = fmaxf(1.0e-6f, sinf((static_cast<float>(y) + 0.5f) * kPi / static_cast<float>(h)));
    const float sa = (kTwoPi / static_cast<float>(w)) * (kPi / static_cast<float>(h)) * st;
    return p / sa;
}

// std::lower_bound over a non-decreasing float array: first i with a[i] >= t.
__device__ __forceinline__ int LowerBound(const float* a, int n, float t) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < t) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

struct EnvSample {
    V3 dir;
    V3 radiance;
    float pdf;
    bool valid;
};

// SampleEnvironment (environment.cpp:157-197): row CDF then the row's
// conditional CDF, both by lower_bound.
__device__ inline EnvSample SampleEnvironment(const DevEnvironment& env, float sx, float sy) {
    EnvSample out{{0, 0, 0}, {0, 0, 0}, 0.0f, false};
    if (!EnvSampleable(env)) return out;
    const int w = env.width, h = env.height;
    if (w <= 0 || h <= 0 || env.total_weight <= 0.0f) return out;
    const float hi1 = 0.99999994f;
    const float row_target = Clampf(sy, 0.0f, hi1) * env.total_weight;
    int y = LowerBound(env.row_cdf, h, row_target);
    if (y == h) y = h - 1;
    const float row_prev = y == 0 ? 0.0f : env.row_cdf[y - 1];
    const float row_w = fmaxf(env.row_weights[y], 1.0e-6f);
    const float row_frac = Clampf((row_target - row_prev) / row_w, 0.0f, 1.0f);
    const float* cdf = env.conditional_cdfs + static_cast<int64_t>(y) * w;
    const float col_target = Clampf(sx, 0.0f, hi1) * row_w;
    int x = LowerBound(cdf, w, col_target);
    if (x == w) x = w - 1;
    const float col_prev = x == 0 ? 0.0f : cdf[x - 1];
    const float tw = fmaxf(env.texel_weights[static_cast<int64_t>(y) * w + x], 1.0e-6f);
    const float col_frac = Clampf((col_target - col_prev) / tw, 0.0f, 1.0f);
    const float u = (static_cast<float>(x) + col_frac) / static_cast<float>(w);
    const float v = (static_cast<float>(y) + row_frac) / static_cast<float>(h);
    const V3 d = EnvUvToDir(u, v, env.rotation);
    const float pdf = PdfEnvironment(env, d);
    if (pdf <= 0.0f) return out;
    out.dir = d;
    out.radiance = EvalEnvironment(env, d);
    out.pdf = pdf;
    out.valid = true;
    return out;
}

// PowerHeuristic (src/integrators/mis.cpp:14-31).
__device__ inline float PowerHeuristic(int na, float pa, int nb, float pb) {
    if (!(na > 0 && pa > 0.0f && isfinite(pa))) return 0.0f;
    if (!(nb > 0 && pb > 0.0f && isfinite(pb))) return 1.0f;
    const float a = static_cast<float>(na) * pa;
    const float b = static_cast<float>(nb) * pb;
    const float a2 = a * a, b2 = b * b;
    const float den = a2 + b2;
    if (!isfinite(den) || den <= 0.0f) return 0.0f;
    return a2 / den;
}

}  // namespace yrc
