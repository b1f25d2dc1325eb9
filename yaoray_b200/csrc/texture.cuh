// RenderTexture sampling (src/shading/texture.cpp:14-322) for device code:
// the reference's wrap rules, texel addressing, mip selection, filters and
// expression order, with explicitly rounded float operations so that the
// result does not depend on the translation unit's contraction setting.
//
// Rounding: nearest and bilinear lookups, the mip chain and the EWA tap
// weights are bit-identical to the reference's. hypot is evaluated as
// sqrt(x*x + y*y) in double (exact products, one rounding per step), which
// is how the C library the reference links evaluates hypotf. The level of
// detail uses log2, which this code evaluates in double and rounds once; the
// C library's log2f differs from that correctly rounded value in its last
// bit for a few percent of arguments, so trilinear and EWA lookups can differ
// from the reference's in the last bits of the blend weight.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "yrc_math_host.hpp"

namespace yrc {

// TextureFilter / TextureWrap (include/yaoray/scene/texture_options.hpp:7-17).
constexpr int32_t kTexNearest = 0;
constexpr int32_t kTexBilinear = 1;
constexpr int32_t kTexTrilinear = 2;
constexpr int32_t kTexEwa = 3;
constexpr int32_t kWrapRepeat = 0;
constexpr int32_t kWrapClamp = 1;
constexpr int32_t kWrapMirror = 2;

// EwaWeights (texture.cpp:140-152): 128 Gaussian taps exp(-2 r^2) - exp(-2).
constexpr int kEwaWeightCount = 128;
// Upper bound on the texels one EWA lookup visits. The reference has none; a
// lookup over more texels than this (a footprint wider than about 1000
// texels on its chosen level) returns the bilinear lookup instead.
constexpr int64_t kEwaMaxTaps = int64_t{1} << 20;

// One level of a texture: level 0 is the image, then the mip chain.
struct DevTexLevel {
    const float4* texels;
    int32_t width;
    int32_t height;
};

struct DevTexture {
    const DevTexLevel* levels;  // level_count entries
    int32_t width;              // RenderTexture::width / height
    int32_t height;
    int32_t level_count;        // 1 + mip levels; 0 = no texel data
    int32_t filter;
    int32_t wrap_s;
    int32_t wrap_t;
};

// TextureFootprint (include/yaoray/shading/texture.hpp:11-20).
struct TexFootprint {
    float dudx, dvdx, dudy, dvdy;
};

__device__ __forceinline__ bool FootprintZero(const TexFootprint& f) {
    return f.dudx == 0.0f && f.dvdx == 0.0f && f.dudy == 0.0f && f.dvdy == 0.0f;
}

// static_cast<int>(float) as the reference's x86-64 build executes it
// (cvttss2si): out-of-range values and NaN give INT_MIN.
__device__ __forceinline__ int TruncToInt(float f) {
    return (f >= -2147483648.0f && f < 2147483648.0f) ? static_cast<int>(f) : static_cast<int>(0x80000000u);
}

// std::max / std::min / std::clamp, NaN behaviour included.
__device__ __forceinline__ float StdMax(float a, float b) { return a < b ? b : a; }
__device__ __forceinline__ float StdMin(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ int StdClampI(int v, int lo, int hi) { return v < lo ? lo : (hi < v ? hi : v); }

// hypotf: sqrt of the double sum of exact double squares, rounded to float.
__device__ __forceinline__ float HypotRef(float x, float y) {
    if (isinf(x) || isinf(y)) return __int_as_float(0x7f800000);
    if (isnan(x) || isnan(y)) return x + y;
    const double xd = static_cast<double>(x), yd = static_cast<double>(y);
    return __double2float_rn(__dsqrt_rn(__dadd_rn(__dmul_rn(xd, xd), __dmul_rn(yd, yd))));
}

__device__ __forceinline__ float Log2Ref(float x) { return __double2float_rn(log2(static_cast<double>(x))); }

__device__ __forceinline__ float4 TexBlack() { return make_float4(0.0f, 0.0f, 0.0f, 1.0f); }  // Color4f{}

__device__ __forceinline__ float4 Add4(float4 a, float4 b) {
    return make_float4(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z), __fadd_rn(a.w, b.w));
}
__device__ __forceinline__ float4 Scale4(float4 a, float s) {
    return make_float4(__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s), __fmul_rn(a.w, s));
}
__device__ __forceinline__ float4 Div4(float4 a, float s) {
    return make_float4(__fdiv_rn(a.x, s), __fdiv_rn(a.y, s), __fdiv_rn(a.z, s), __fdiv_rn(a.w, s));
}
// Lerp (texture.cpp:101-103): a * (1 - t) + b * t.
__device__ __forceinline__ float4 Lerp4(float4 a, float4 b, float t) {
    return Add4(Scale4(a, __fsub_rn(1.0f, t)), Scale4(b, t));
}

// ApplyWrap (texture.cpp:20-28).
__device__ __forceinline__ float ApplyWrap(float v, int32_t wrap) {
    if (wrap == kWrapClamp) return v < 0.0f ? 0.0f : (1.0f < v ? 1.0f : v);
    const float base = floorf(v);
    const float fraction = __fsub_rn(v, base);
    if (wrap == kWrapMirror) return (TruncToInt(base) & 1) == 0 ? fraction : __fsub_rn(1.0f, fraction);
    return fraction < 0.0f ? __fadd_rn(fraction, 1.0f) : fraction;
}

// WrappedTexelIndex (texture.cpp:30-40).
__device__ __forceinline__ int WrappedTexelIndex(int value, int count, int32_t wrap) {
    if (wrap == kWrapClamp) return StdClampI(value, 0, count - 1);
    if (wrap == kWrapMirror) {
        const int period = count * 2;
        int wrapped = value % period;
        if (wrapped < 0) wrapped += period;
        return wrapped < count ? wrapped : period - 1 - wrapped;
    }
    int wrapped = value % count;
    if (wrapped < 0) wrapped += count;
    return wrapped;
}

// Level (texture.cpp:42-60): levels past the chain's end give its last.
__device__ __forceinline__ DevTexLevel TexLevel(const DevTexture& t, int level) {
    const int i = level <= 0 ? 0 : (level < t.level_count - 1 ? level : t.level_count - 1);
    return t.levels[i];
}

// TexelAt (texture.cpp:90-99).
__device__ __forceinline__ float4 TexelAt(const DevTexLevel& L, int x, int y, int32_t ws, int32_t wt) {
    if (L.width <= 0 || L.height <= 0 || !L.texels) return TexBlack();
    const int ix = WrappedTexelIndex(x, L.width, ws);
    const int iy = WrappedTexelIndex(y, L.height, wt);
    return __ldg(L.texels + static_cast<int64_t>(iy) * L.width + ix);
}

// SampleNearest (texture.cpp:105-113).
__device__ inline float4 SampleNearest(const DevTexLevel& L, const DevTexture& t, float u, float v) {
    if (L.width <= 0 || L.height <= 0 || !L.texels) return TexBlack();
    const int x = StdClampI(TruncToInt(floorf(__fmul_rn(ApplyWrap(u, t.wrap_s), static_cast<float>(L.width)))), 0,
                            L.width - 1);
    const int y = StdClampI(TruncToInt(floorf(__fmul_rn(ApplyWrap(v, t.wrap_t), static_cast<float>(L.height)))), 0,
                            L.height - 1);
    return TexelAt(L, x, y, t.wrap_s, t.wrap_t);
}

// SampleBilinear (texture.cpp:115-130).
__device__ inline float4 SampleBilinear(const DevTexLevel& L, const DevTexture& t, float u, float v) {
    if (L.width <= 0 || L.height <= 0 || !L.texels) return TexBlack();
    if (L.width == 1 && L.height == 1) return __ldg(L.texels);
    const float s = __fsub_rn(__fmul_rn(ApplyWrap(u, t.wrap_s), static_cast<float>(L.width)), 0.5f);
    const float tt = __fsub_rn(__fmul_rn(ApplyWrap(v, t.wrap_t), static_cast<float>(L.height)), 0.5f);
    const int s0 = TruncToInt(floorf(s));
    const int t0 = TruncToInt(floorf(tt));
    const float ds = __fsub_rn(s, static_cast<float>(s0));
    const float dt = __fsub_rn(tt, static_cast<float>(t0));
    const float4 c00 = TexelAt(L, s0, t0, t.wrap_s, t.wrap_t);
    const float4 c10 = TexelAt(L, s0 + 1, t0, t.wrap_s, t.wrap_t);
    const float4 c01 = TexelAt(L, s0, t0 + 1, t.wrap_s, t.wrap_t);
    const float4 c11 = TexelAt(L, s0 + 1, t0 + 1, t.wrap_s, t.wrap_t);
    return Lerp4(Lerp4(c00, c10, ds), Lerp4(c01, c11, ds), dt);
}

// LodForFootprint (texture.cpp:132-138).
__device__ inline float LodForFootprint(const DevTexture& t, const TexFootprint& f) {
    const float w = static_cast<float>(t.width > 1 ? t.width : 1);
    const float h = static_cast<float>(t.height > 1 ? t.height : 1);
    const float dx = HypotRef(__fmul_rn(f.dudx, w), __fmul_rn(f.dvdx, h));
    const float dy = HypotRef(__fmul_rn(f.dudy, w), __fmul_rn(f.dvdy, h));
    return StdMax(0.0f, Log2Ref(StdMax(1.0f, StdMax(dx, dy))));
}

// SampleEwaLevel (texture.cpp:154-213). `weights` is EwaWeights().
__device__ inline float4 SampleEwaLevel(const DevTexture& t, float u, float v, const TexFootprint& f, int level,
                                        const float* weights) {
    const DevTexLevel L = TexLevel(t, level);
    if (L.width <= 0 || L.height <= 0 || !L.texels) return TexBlack();
    const float lw = static_cast<float>(L.width), lh = static_cast<float>(L.height);
    float dsdx = __fmul_rn(f.dudx, lw);
    float dtdx = __fmul_rn(f.dvdx, lh);
    float dsdy = __fmul_rn(f.dudy, lw);
    float dtdy = __fmul_rn(f.dvdy, lh);
    if (__fadd_rn(__fmul_rn(dsdx, dsdx), __fmul_rn(dtdx, dtdx)) <
        __fadd_rn(__fmul_rn(dsdy, dsdy), __fmul_rn(dtdy, dtdy))) {
        float tmp = dsdx;
        dsdx = dsdy;
        dsdy = tmp;
        tmp = dtdx;
        dtdx = dtdy;
        dtdy = tmp;
    }
    const float major = HypotRef(dsdx, dtdx);
    float minor = HypotRef(dsdy, dtdy);
    const float max_anisotropy = 8.0f;
    if (minor > 0.0f && major > __fmul_rn(minor, max_anisotropy)) {
        const float scale = __fdiv_rn(major, __fmul_rn(minor, max_anisotropy));
        dsdy = __fmul_rn(dsdy, scale);
        dtdy = __fmul_rn(dtdy, scale);
        minor = __fmul_rn(minor, scale);
    }
    if (minor == 0.0f) return SampleBilinear(L, t, u, v);

    const float s = __fsub_rn(__fmul_rn(ApplyWrap(u, t.wrap_s), lw), 0.5f);
    const float tc = __fsub_rn(__fmul_rn(ApplyWrap(v, t.wrap_t), lh), 0.5f);
    float a = __fadd_rn(__fadd_rn(__fmul_rn(dtdx, dtdx), __fmul_rn(dtdy, dtdy)), 1.0f);
    float b = __fmul_rn(-2.0f, __fadd_rn(__fmul_rn(dsdx, dtdx), __fmul_rn(dsdy, dtdy)));
    float c = __fadd_rn(__fadd_rn(__fmul_rn(dsdx, dsdx), __fmul_rn(dsdy, dsdy)), 1.0f);
    const float inverse = __fdiv_rn(1.0f, __fsub_rn(__fmul_rn(a, c), __fmul_rn(__fmul_rn(0.25f, b), b)));
    a = __fmul_rn(a, inverse);
    b = __fmul_rn(b, inverse);
    c = __fmul_rn(c, inverse);
    const float determinant = __fadd_rn(__fmul_rn(-b, b), __fmul_rn(__fmul_rn(4.0f, a), c));
    if (determinant <= 0.0f) return SampleBilinear(L, t, u, v);
    const float inverse_det = __fdiv_rn(1.0f, determinant);
    const float radius_s = __fmul_rn(2.0f, __fsqrt_rn(__fmul_rn(c, inverse_det)));
    const float radius_t = __fmul_rn(2.0f, __fsqrt_rn(__fmul_rn(a, inverse_det)));
    const int s0 = TruncToInt(ceilf(__fsub_rn(s, radius_s)));
    const int s1 = TruncToInt(floorf(__fadd_rn(s, radius_s)));
    const int t0 = TruncToInt(ceilf(__fsub_rn(tc, radius_t)));
    const int t1 = TruncToInt(floorf(__fadd_rn(tc, radius_t)));
    const int64_t cols = static_cast<int64_t>(s1) - s0 + 1, rows = static_cast<int64_t>(t1) - t0 + 1;
    if (cols > kEwaMaxTaps || rows > kEwaMaxTaps || cols * rows > kEwaMaxTaps) return SampleBilinear(L, t, u, v);

    float4 sum = make_float4(0.0f, 0.0f, 0.0f, 1.0f);  // Color4f{} starts at alpha 1
    float weight_sum = 0.0f;
    for (int it = t0; it <= t1; ++it) {
        for (int is = s0; is <= s1; ++is) {
            const float ss = __fsub_rn(static_cast<float>(is), s);
            const float tt = __fsub_rn(static_cast<float>(it), tc);
            const float r2 = __fadd_rn(__fadd_rn(__fmul_rn(__fmul_rn(a, ss), ss), __fmul_rn(__fmul_rn(b, ss), tt)),
                                       __fmul_rn(__fmul_rn(c, tt), tt));
            if (r2 >= 1.0f) continue;
            // std::min(size - 1, size_t(r2 * size)): r2 is in [0, 1) here, or
            // negative for a degenerate ellipse, where size_t() of the
            // product is out of range; the x86-64 build then yields 0 for
            // products in (-1, 0] and 2^64 - |n| (clamped to 127) below.
            const float scaled = __fmul_rn(r2, static_cast<float>(kEwaWeightCount));
            int wi;
            if (scaled > -1.0f) {
                wi = scaled < static_cast<float>(kEwaWeightCount - 1) ? static_cast<int>(scaled) : kEwaWeightCount - 1;
            } else {
                wi = kEwaWeightCount - 1;
            }
            const float weight = weights[wi];
            sum = Add4(sum, Scale4(TexelAt(L, is, it, t.wrap_s, t.wrap_t), weight));
            weight_sum = __fadd_rn(weight_sum, weight);
        }
    }
    return weight_sum > 0.0f ? Div4(sum, weight_sum) : SampleBilinear(L, t, u, v);
}

// SampleTrilinear (texture.cpp:215-223).
__device__ inline float4 SampleTrilinear(const DevTexture& t, float u, float v, const TexFootprint& f) {
    const float lod = StdMin(LodForFootprint(t, f), static_cast<float>(t.level_count - 1));
    const int level0 = TruncToInt(floorf(lod));
    const int level1 = min(level0 + 1, t.level_count - 1);
    return Lerp4(SampleBilinear(TexLevel(t, level0), t, u, v), SampleBilinear(TexLevel(t, level1), t, u, v),
                 __fsub_rn(lod, static_cast<float>(level0)));
}

// SampleEwa (texture.cpp:225-238).
__device__ inline float4 SampleEwa(const DevTexture& t, float u, float v, const TexFootprint& f,
                                   const float* weights) {
    const float w = static_cast<float>(t.width > 1 ? t.width : 1);
    const float h = static_cast<float>(t.height > 1 ? t.height : 1);
    const float dx = HypotRef(__fmul_rn(f.dudx, w), __fmul_rn(f.dvdx, h));
    const float dy = HypotRef(__fmul_rn(f.dudy, w), __fmul_rn(f.dvdy, h));
    const float minor = StdMax(1.0f, StdMin(dx, dy));
    const float lod = StdMin(StdMax(0.0f, Log2Ref(minor)), static_cast<float>(t.level_count - 1));
    const int level0 = TruncToInt(floorf(lod));
    const int level1 = min(level0 + 1, t.level_count - 1);
    return Lerp4(SampleEwaLevel(t, u, v, f, level0, weights), SampleEwaLevel(t, u, v, f, level1, weights),
                 __fsub_rn(lod, static_cast<float>(level0)));
}

// SampleTexture4 (texture.cpp:297-309).
__device__ inline float4 SampleTexture4(const DevTexture& t, float u, float v, const TexFootprint& f,
                                        const float* weights) {
    if (t.width <= 0 || t.height <= 0 || t.level_count <= 0) return TexBlack();
    if (t.filter == kTexNearest) return SampleNearest(TexLevel(t, 0), t, u, v);
    if (t.filter == kTexTrilinear && !FootprintZero(f) && t.level_count > 1) return SampleTrilinear(t, u, v, f);
    if (t.filter == kTexEwa && !FootprintZero(f) && t.level_count > 1) return SampleEwa(t, u, v, f, weights);
    return SampleBilinear(TexLevel(t, 0), t, u, v);
}

}  // namespace yrc
