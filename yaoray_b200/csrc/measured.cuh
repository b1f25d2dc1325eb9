// Measured (RGL, Dupuy & Jakob 2018) BRDFs on the device: the
// piecewise-bilinear 2-D warp with conditioning parameters
// (include/yaoray/shading/piecewise_linear_2d.hpp, the pbrt-v4 layout) and
// the BRDF's evaluation, pdf and importance sampling
// (src/shading/bsdf_measured.cpp:10-242). Warps are built on the host
// (measured.cu) with the reference's normalisation and CDFs; the device
// reads them. The reference's fused multiply-adds (std::fma) are
// __fmaf_rn here; the angles use CUDA's acosf / atan2f / sincosf, so values
// agree with the reference's within rounding, not bit for bit.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "shading.cuh"
#include "texture.cuh"

namespace yrc {

// One PiecewiseLinear2D<D>: size_x x size_y values per slice, slices over
// the D conditioning parameters (param_size values each, stride 0 for a
// parameter with one value).
struct DevWarp {
    const float* data;
    const float* marginal;     // size_y per slice (sampled warps only)
    const float* conditional;  // size_x * size_y per slice (sampled warps only)
    const float* param_values[3];
    uint32_t param_size[3];
    uint32_t param_stride[3];
    int32_t size_x, size_y;
    float patch_x, patch_y, inv_patch_x, inv_patch_y;
};

struct DevMeasuredBrdf {
    DevWarp ndf, sigma, vndf, luminance, spectra;
    int32_t isotropic;
};

struct WarpSample {
    float x, y, pdf;
};

// FindInterval: the last index i in [0, size - 2] with pred(i) true (binary
// search over 1..size-2 as the reference's).
template <typename Pred>
__device__ __forceinline__ uint32_t WarpFindInterval(uint32_t size, const Pred& pred) {
    int64_t first = 1, len = static_cast<int64_t>(size) - 2;
    while (len > 0) {
        const int64_t half = len >> 1, middle = first + half;
        if (pred(static_cast<uint32_t>(middle))) {
            first = middle + 1;
            len -= half + 1;
        } else {
            len = half;
        }
    }
    int64_t lo = first - 1;
    if (lo < 0) lo = 0;
    int64_t hi = static_cast<int64_t>(size) - 2;
    if (hi < 0) hi = 0;
    if (lo > hi) lo = hi;
    return static_cast<uint32_t>(lo);
}

// lookup<D>: multilinear blend of the slices around the parameters.
template <int D>
__device__ __forceinline__ float WarpLookup(const DevWarp& w, const float* base, uint32_t i0, uint32_t size,
                                            const float* pw) {
    if constexpr (D == 0) {
        return __ldg(base + i0);
    } else {
        const uint32_t i1 = i0 + w.param_stride[D - 1] * size;
        const float v0 = WarpLookup<D - 1>(w, base, i0, size, pw);
        const float v1 = WarpLookup<D - 1>(w, base, i1, size, pw);
        return __fmaf_rn(v0, pw[2 * D - 2], __fmul_rn(v1, pw[2 * D - 1]));
    }
}

// The parameter weights and slice offset shared by Evaluate / Invert / Sample.
template <int D>
__device__ __forceinline__ uint32_t WarpParams(const DevWarp& w, const float* param, float* pw) {
    uint32_t slice_offset = 0;
#pragma unroll
    for (int dim = 0; dim < D; ++dim) {
        if (w.param_size[dim] == 1) {
            pw[2 * dim] = 1.0f;
            pw[2 * dim + 1] = 0.0f;
            continue;
        }
        const float* values = w.param_values[dim];
        const float p = param[dim];
        const uint32_t idx = WarpFindInterval(w.param_size[dim], [&](uint32_t i) { return values[i] <= p; });
        const float p0 = values[idx], p1 = values[idx + 1];
        const float t = __fdiv_rn(__fsub_rn(p, p0), __fsub_rn(p1, p0));
        pw[2 * dim + 1] = t < 0.0f ? 0.0f : (t > 1.0f ? 1.0f : t);
        pw[2 * dim] = __fsub_rn(1.0f, pw[2 * dim + 1]);
        slice_offset += w.param_stride[dim] * idx;
    }
    return slice_offset;
}

// Cell index of a coordinate: (int) truncation, at most size - 2, and at
// least 0 (the reference reads outside its arrays for negative
// coordinates; here they take the first cell).
__device__ __forceinline__ int WarpCell(float v, int size) {
    const int i = TruncToInt(v);
    return i < size - 2 ? (i < 0 ? 0 : i) : size - 2;
}

__device__ __forceinline__ float WarpInvPatch(const DevWarp& w) { return __fmul_rn(w.inv_patch_x, w.inv_patch_y); }

// PiecewiseLinear2D::Evaluate.
template <int D>
__device__ inline float WarpEvaluate(const DevWarp& w, float x, float y, const float* param) {
    float pw[2 * (D > 0 ? D : 1)];
    const uint32_t slice = WarpParams<D>(w, param, pw);
    const float px = __fmul_rn(x, w.inv_patch_x), py = __fmul_rn(y, w.inv_patch_y);
    const int ox = WarpCell(px, w.size_x), oy = WarpCell(py, w.size_y);
    const float w1x = __fsub_rn(px, static_cast<float>(ox)), w1y = __fsub_rn(py, static_cast<float>(oy));
    const float w0x = __fsub_rn(1.0f, w1x), w0y = __fsub_rn(1.0f, w1y);
    const uint32_t size = static_cast<uint32_t>(w.size_x) * static_cast<uint32_t>(w.size_y);
    uint32_t index = static_cast<uint32_t>(ox) + static_cast<uint32_t>(oy) * static_cast<uint32_t>(w.size_x);
    if (D != 0) index += slice * size;
    const float v00 = WarpLookup<D>(w, w.data, index, size, pw);
    const float v10 = WarpLookup<D>(w, w.data + 1, index, size, pw);
    const float v01 = WarpLookup<D>(w, w.data + w.size_x, index, size, pw);
    const float v11 = WarpLookup<D>(w, w.data + w.size_x + 1, index, size, pw);
    const float a = __fmaf_rn(w0x, v00, __fmul_rn(w1x, v10));
    const float b = __fmaf_rn(w0x, v01, __fmul_rn(w1x, v11));
    return __fmul_rn(__fmaf_rn(w0y, a, __fmul_rn(w1y, b)), WarpInvPatch(w));
}

// PiecewiseLinear2D::Invert: sample-space position of (x, y) and its pdf.
template <int D>
__device__ inline WarpSample WarpInvert(const DevWarp& w, float x, float y, const float* param) {
    float pw[2 * (D > 0 ? D : 1)];
    const uint32_t slice = WarpParams<D>(w, param, pw);
    float sx = __fmul_rn(x, w.inv_patch_x), sy = __fmul_rn(y, w.inv_patch_y);
    const int posx = WarpCell(sx, w.size_x), posy = WarpCell(sy, w.size_y);
    sx = __fsub_rn(sx, static_cast<float>(posx));
    sy = __fsub_rn(sy, static_cast<float>(posy));
    const uint32_t sxs = static_cast<uint32_t>(w.size_x);
    const uint32_t slice_size = sxs * static_cast<uint32_t>(w.size_y);
    uint32_t offset = static_cast<uint32_t>(posx) + static_cast<uint32_t>(posy) * sxs;
    if (D != 0) offset += slice * slice_size;
    const float v00 = WarpLookup<D>(w, w.data, offset, slice_size, pw);
    const float v10 = WarpLookup<D>(w, w.data + 1, offset, slice_size, pw);
    const float v01 = WarpLookup<D>(w, w.data + w.size_x, offset, slice_size, pw);
    const float v11 = WarpLookup<D>(w, w.data + w.size_x + 1, offset, slice_size, pw);
    const float w1x = sx, w1y = sy, w0x = __fsub_rn(1.0f, w1x), w0y = __fsub_rn(1.0f, w1y);
    const float c0 = __fmaf_rn(w0y, v00, __fmul_rn(w1y, v01));
    const float c1 = __fmaf_rn(w0y, v10, __fmul_rn(w1y, v11));
    const float pdf = __fmaf_rn(w0x, c0, __fmul_rn(w1x, c1));
    sx = __fmul_rn(sx, __fadd_rn(c0, __fmul_rn(__fmul_rn(0.5f, sx), __fsub_rn(c1, c0))));
    const float vc0 = WarpLookup<D>(w, w.conditional, offset, slice_size, pw);
    const float vc1 = WarpLookup<D>(w, w.conditional + w.size_x, offset, slice_size, pw);
    sx = __fadd_rn(sx, __fadd_rn(__fmul_rn(__fsub_rn(1.0f, sy), vc0), __fmul_rn(sy, vc1)));
    offset = static_cast<uint32_t>(posy) * sxs;
    if (D != 0) offset += slice * slice_size;
    const float r0 = WarpLookup<D>(w, w.conditional, offset + sxs - 1, slice_size, pw);
    const float r1 = WarpLookup<D>(w, w.conditional, offset + (sxs * 2 - 1), slice_size, pw);
    sx = __fdiv_rn(sx, __fadd_rn(__fmul_rn(__fsub_rn(1.0f, sy), r0), __fmul_rn(sy, r1)));
    sy = __fmul_rn(sy, __fadd_rn(r0, __fmul_rn(__fmul_rn(0.5f, sy), __fsub_rn(r1, r0))));
    offset = static_cast<uint32_t>(posy);
    if (D != 0) offset += slice * static_cast<uint32_t>(w.size_y);
    sy = __fadd_rn(sy, WarpLookup<D>(w, w.marginal, offset, static_cast<uint32_t>(w.size_y), pw));
    return WarpSample{sx, sy, __fmul_rn(pdf, WarpInvPatch(w))};
}

__device__ __forceinline__ float WarpSafeSqrt(float v) { return __fsqrt_rn(v > 0.0f ? v : 0.0f); }

// PiecewiseLinear2D::Sample.
template <int D>
__device__ inline WarpSample WarpSampleAt(const DevWarp& w, float ux, float uy, const float* param) {
    const float one_minus_eps = 0x1.fffffep-1f;
    const float lo = __fsub_rn(1.0f, one_minus_eps);
    ux = ux < lo ? lo : (ux > one_minus_eps ? one_minus_eps : ux);
    uy = uy < lo ? lo : (uy > one_minus_eps ? one_minus_eps : uy);
    float pw[2 * (D > 0 ? D : 1)];
    const uint32_t slice = WarpParams<D>(w, param, pw);
    const uint32_t sxs = static_cast<uint32_t>(w.size_x), sys = static_cast<uint32_t>(w.size_y);
    uint32_t offset = D != 0 ? slice * sys : 0u;
    auto fetch_marginal = [&](uint32_t idx) { return WarpLookup<D>(w, w.marginal, offset + idx, sys, pw); };
    const uint32_t row = WarpFindInterval(sys, [&](uint32_t idx) { return fetch_marginal(idx) < uy; });
    uy = __fsub_rn(uy, fetch_marginal(row));
    const uint32_t slice_size = sxs * sys;
    offset = row * sxs;
    if (D != 0) offset += slice * slice_size;
    const float r0 = WarpLookup<D>(w, w.conditional, offset + sxs - 1, slice_size, pw);
    const float r1 = WarpLookup<D>(w, w.conditional, offset + (sxs * 2 - 1), slice_size, pw);
    bool is_const = fabsf(__fsub_rn(r0, r1)) < __fmul_rn(1e-4f, __fadd_rn(r0, r1));
    uy = is_const ? __fmul_rn(2.0f, uy)
                  : __fsub_rn(r0, WarpSafeSqrt(__fsub_rn(__fmul_rn(r0, r0),
                                                         __fmul_rn(__fmul_rn(2.0f, uy), __fsub_rn(r0, r1)))));
    uy = __fdiv_rn(uy, is_const ? __fadd_rn(r0, r1) : __fsub_rn(r0, r1));
    ux = __fmul_rn(ux, __fadd_rn(__fmul_rn(__fsub_rn(1.0f, uy), r0), __fmul_rn(uy, r1)));
    auto fetch_conditional = [&](uint32_t idx) {
        const float v0 = WarpLookup<D>(w, w.conditional, offset + idx, slice_size, pw);
        const float v1 = WarpLookup<D>(w, w.conditional + w.size_x, offset + idx, slice_size, pw);
        return __fadd_rn(__fmul_rn(__fsub_rn(1.0f, uy), v0), __fmul_rn(uy, v1));
    };
    const uint32_t col = WarpFindInterval(sxs, [&](uint32_t idx) { return fetch_conditional(idx) < ux; });
    ux = __fsub_rn(ux, fetch_conditional(col));
    offset += col;
    const float v00 = WarpLookup<D>(w, w.data, offset, slice_size, pw);
    const float v10 = WarpLookup<D>(w, w.data + 1, offset, slice_size, pw);
    const float v01 = WarpLookup<D>(w, w.data + w.size_x, offset, slice_size, pw);
    const float v11 = WarpLookup<D>(w, w.data + w.size_x + 1, offset, slice_size, pw);
    const float c0 = __fmaf_rn(__fsub_rn(1.0f, uy), v00, __fmul_rn(uy, v01));
    const float c1 = __fmaf_rn(__fsub_rn(1.0f, uy), v10, __fmul_rn(uy, v11));
    is_const = fabsf(__fsub_rn(c0, c1)) < __fmul_rn(1e-4f, __fadd_rn(c0, c1));
    ux = is_const ? __fmul_rn(2.0f, ux)
                  : __fsub_rn(c0, WarpSafeSqrt(__fsub_rn(__fmul_rn(c0, c0),
                                                         __fmul_rn(__fmul_rn(2.0f, ux), __fsub_rn(c0, c1)))));
    ux = __fdiv_rn(ux, is_const ? __fadd_rn(c0, c1) : __fsub_rn(c0, c1));
    const float pdf = __fmul_rn(__fadd_rn(__fmul_rn(__fsub_rn(1.0f, ux), c0), __fmul_rn(ux, c1)), WarpInvPatch(w));
    return WarpSample{__fmul_rn(__fadd_rn(static_cast<float>(col), ux), w.patch_x),
                      __fmul_rn(__fadd_rn(static_cast<float>(row), uy), w.patch_y), pdf};
}

// ------------------------------------------------------- the measured BRDF

struct MeasuredFrame {
    V3 t, b, n;
};

__device__ __forceinline__ MeasuredFrame MakeMeasuredFrame(V3 n) {
    const V3 helper = fabsf(n.z) < 0.999f ? V3{0.0f, 0.0f, 1.0f} : V3{1.0f, 0.0f, 0.0f};
    const V3 t = Normalize(Cross(helper, n));
    return MeasuredFrame{t, Cross(n, t), n};
}

__device__ __forceinline__ V3 ToLocal(const MeasuredFrame& f, V3 w) { return V3{Dot(w, f.t), Dot(w, f.b), Dot(w, f.n)}; }

__device__ __forceinline__ float MeasuredTheta2U(float t) { return sqrtf(t * (2.0f / kPi)); }
__device__ __forceinline__ float MeasuredPhi2U(float p) { return p * (1.0f / (2.0f * kPi)) + 0.5f; }
__device__ __forceinline__ float ClampUnit(float v) { return v < -1.0f ? -1.0f : (v > 1.0f ? 1.0f : v); }

// EvaluateMeasured (bsdf_measured.cpp:10-61).
static __device__ __noinline__ V3 EvalMeasured(const DevMeasuredBrdf& m, V3 wo, V3 wi, V3 n) {
    const MeasuredFrame f = MakeMeasuredFrame(n);
    V3 lwo = ToLocal(f, wo), lwi = ToLocal(f, wi);
    if (lwo.z * lwi.z <= 0.0f) return V3{0.0f, 0.0f, 0.0f};
    if (lwo.z < 0.0f) {
        lwo = -lwo;
        lwi = -lwi;
    }
    V3 wm = lwo + lwi;
    if (LengthSq(wm) <= 0.0f) return V3{0.0f, 0.0f, 0.0f};
    wm = Normalize(wm);
    const float theta_o = acosf(ClampUnit(lwo.z)), phi_o = atan2f(lwo.y, lwo.x);
    const float theta_m = acosf(ClampUnit(wm.z)), phi_m = atan2f(wm.y, wm.x);
    const float uwo_x = MeasuredTheta2U(theta_o), uwo_y = MeasuredPhi2U(phi_o);
    const float uwm_x = MeasuredTheta2U(theta_m);
    float uwm_y = MeasuredPhi2U(m.isotropic ? (phi_m - phi_o) : phi_m);
    uwm_y = uwm_y - floorf(uwm_y);
    const float p2[2] = {phi_o, theta_o};
    const WarpSample ui = WarpInvert<2>(m.vndf, uwm_x, uwm_y, p2);
    const float cos_i = lwi.z;
    const float sig = WarpEvaluate<0>(m.sigma, uwo_x, uwo_y, nullptr);
    const float denom = 4.0f * sig * cos_i;
    if (denom <= 0.0f) return V3{0.0f, 0.0f, 0.0f};
    const float ndf = WarpEvaluate<0>(m.ndf, uwm_x, uwm_y, nullptr);
    const float pr[3] = {phi_o, theta_o, 630.0f}, pg[3] = {phi_o, theta_o, 532.0f}, pb[3] = {phi_o, theta_o, 467.0f};
    const float r = fmaxf(0.0f, WarpEvaluate<3>(m.spectra, ui.x, ui.y, pr));
    const float g = fmaxf(0.0f, WarpEvaluate<3>(m.spectra, ui.x, ui.y, pg));
    const float b = fmaxf(0.0f, WarpEvaluate<3>(m.spectra, ui.x, ui.y, pb));
    const float scale = ndf / denom;
    const V3 out{r * scale, g * scale, b * scale};
    if (!isfinite(out.x) || !isfinite(out.y) || !isfinite(out.z)) return V3{0.0f, 0.0f, 0.0f};
    return out;
}

// PdfMeasured (bsdf_measured.cpp:177-238).
static __device__ __noinline__ float PdfMeasuredBrdf(const DevMeasuredBrdf& m, V3 wo, V3 wi, V3 n) {
    const MeasuredFrame f = MakeMeasuredFrame(n);
    V3 lwo = ToLocal(f, wo), lwi = ToLocal(f, wi);
    if (lwo.z * lwi.z <= 0.0f) return 0.0f;
    if (lwo.z < 0.0f) {
        lwo = -lwo;
        lwi = -lwi;
    }
    V3 wm = lwi + lwo;
    if (LengthSq(wm) <= 0.0f) return 0.0f;
    wm = Normalize(wm);
    const float theta_o = acosf(ClampUnit(lwo.z)), phi_o = atan2f(lwo.y, lwo.x);
    const float theta_m = acosf(ClampUnit(wm.z)), phi_m = atan2f(wm.y, wm.x);
    const float uwm_x = MeasuredTheta2U(theta_m);
    float uwm_y = MeasuredPhi2U(m.isotropic ? (phi_m - phi_o) : phi_m);
    uwm_y = uwm_y - floorf(uwm_y);
    const float p2[2] = {phi_o, theta_o};
    const WarpSample ui = WarpInvert<2>(m.vndf, uwm_x, uwm_y, p2);
    const float lum = WarpEvaluate<2>(m.luminance, ui.x, ui.y, p2);
    const float sin_theta_m = sqrtf(wm.x * wm.x + wm.y * wm.y);
    const float jac = 4.0f * Dot(lwo, wm) * fmaxf(2.0f * kPi * kPi * uwm_x * sin_theta_m, 1e-6f);
    return jac > 0.0f ? ui.pdf * lum / jac : 0.0f;
}

// SampleMeasured (bsdf_measured.cpp:67-128). The three entry points are not
// inlined, so that the generic shading class carries their registers only
// inside the call.
static __device__ __noinline__ BsdfSample SampleMeasuredBrdf(const DevMeasuredBrdf& m, V3 wo, V3 n, float sx, float sy) {
    const MeasuredFrame f = MakeMeasuredFrame(n);
    V3 lwo = ToLocal(f, wo);
    const bool flip = lwo.z <= 0.0f;
    if (flip) lwo = -lwo;
    const float theta_o = acosf(ClampUnit(lwo.z)), phi_o = atan2f(lwo.y, lwo.x);
    const float p2[2] = {phi_o, theta_o};
    const WarpSample s1 = WarpSampleAt<2>(m.luminance, sx, sy, p2);
    const WarpSample s2 = WarpSampleAt<2>(m.vndf, s1.x, s1.y, p2);
    float phi_m = (2.0f * s2.y - 1.0f) * kPi;
    const float theta_m = s2.x * s2.x * (kPi / 2.0f);
    if (m.isotropic) phi_m += phi_o;
    const float sin_theta_m = sinf(theta_m), cos_theta_m = cosf(theta_m);
    const V3 wm{sin_theta_m * cosf(phi_m), sin_theta_m * sinf(phi_m), cos_theta_m};
    const float dot_wm = Dot(lwo, wm);
    if (dot_wm <= 0.0f) return NoSample();
    V3 wi_local = wm * (2.0f * dot_wm) - lwo;
    if (wi_local.z <= 0.0f) return NoSample();
    const float jac = 4.0f * dot_wm * fmaxf(2.0f * kPi * kPi * s2.x * sin_theta_m, 1e-6f);
    const float sample_pdf = s2.pdf * s1.pdf / jac;
    if (!(sample_pdf > 0.0f) || !isfinite(sample_pdf)) return NoSample();
    if (flip) wi_local = -wi_local;
    const V3 wi = Normalize(f.t * wi_local.x + f.b * wi_local.y + f.n * wi_local.z);
    const float pdf = PdfMeasuredBrdf(m, wo, wi, n);
    if (!(pdf > 0.0f) || !isfinite(pdf)) return NoSample();
    const V3 fv = EvalMeasured(m, wo, wi, n);
    const float cos_wi = fabsf(Dot(wi, n));
    return BsdfSample{wi, fv * (cos_wi / pdf), pdf, true, false};
}

}  // namespace yrc
