// Device BSDF dispatch: EvaluateBsdf / PdfBsdf / SampleBsdf / IsDeltaBsdf of
// src/shading/bsdf.cpp:17-329 and the stochastic layered walk of
// src/shading/bsdf_layered.cpp:13-349, restated for the device. The layered
// estimators draw from the path's PCG32 stream exactly as the reference does
// within one call.
#pragma once

#include "measured.cuh"
#include "sampler.cuh"
#include "shading.cuh"

namespace yrc {

enum MatKind : int32_t {
    kDiffuse = 0,
    kConductor = 1,
    kDielectric = 2,
    kThinDielectric = 3,
    kCoatedDiffuse = 4,
    kCoatedConductor = 5,
    kDiffuseTransmission = 6,
    kMix = 7,
    kMeasured = 8,
    kSubsurface = 9,
    kSubsurfaceExit = 10,
};

// The part of a material the BSDFs read.
struct Mat {
    int32_t kind;
    V3 reflectance;
    float ior;
    float ur, vr;
    float coating_ior;
    float coat_thickness;
    V3 coat_absorption;
    int32_t coat_maxdepth;
    int32_t coat_nsamples;
    const DevMeasuredBrdf* measured;  // kMeasured with data; null: the conductor fallback
};

__device__ inline Mat LoadMat(const DevMaterial& m) {
    Mat r;
    r.kind = m.kind;
    r.reflectance = Ld3(m.reflectance);
    r.ior = m.ior;
    r.ur = m.uroughness;
    r.vr = m.vroughness;
    r.coating_ior = m.coating_ior;
    r.coat_thickness = m.coat_thickness;
    r.coat_absorption = Ld3(m.coat_absorption);
    r.coat_maxdepth = m.coat_maxdepth;
    r.coat_nsamples = m.coat_nsamples;
    r.measured = nullptr;
    return r;
}

// FresnelMoment1 polynomial (src/shading/bssrdf.cpp) used by SubsurfaceSw;
// FrDielectric is the dielectric Fresnel with a relative eta.
__device__ inline float FresnelMoment1(float eta) {
    const float eta2 = eta * eta, eta3 = eta2 * eta, eta4 = eta3 * eta, eta5 = eta4 * eta;
    if (eta < 1.0f) return 0.45966f - 1.73965f * eta + 3.37668f * eta2 - 3.904945f * eta3 + 2.49277f * eta4 -
                              0.68441f * eta5;
    return -4.61686f + 11.1136f * eta - 10.4646f * eta2 + 5.11455f * eta3 - 1.27198f * eta4 + 0.12746f * eta5;
}

__device__ inline float FrDielectric(float cos_i, float eta) {
    cos_i = Clampf(cos_i, -1.0f, 1.0f);
    if (cos_i < 0.0f) {
        eta = 1.0f / eta;
        cos_i = -cos_i;
    }
    const float sin2_i = 1.0f - cos_i * cos_i;
    const float sin2_t = sin2_i / (eta * eta);
    if (sin2_t >= 1.0f) return 1.0f;
    const float cos_t = sqrtf(fmaxf(0.0f, 1.0f - sin2_t));
    const float r_parl = (eta * cos_i - cos_t) / (eta * cos_i + cos_t);
    const float r_perp = (cos_i - eta * cos_t) / (cos_i + eta * cos_t);
    return (r_parl * r_parl + r_perp * r_perp) / 2.0f;
}

__device__ inline float SubsurfaceSw(float cos_t, float eta) {
    const float c = 1.0f - 2.0f * FresnelMoment1(1.0f / eta);
    return (1.0f - FrDielectric(cos_t, eta)) / (c * kPi);
}

__device__ __forceinline__ bool IsDelta(const Mat& m) {
    switch (m.kind) {
        case kConductor:
        case kCoatedConductor:
        case kDielectric:
        case kThinDielectric:
            return m.ur == 0.0f && m.vr == 0.0f;
        case kSubsurface:
            return true;
        default:
            return false;
    }
}

struct DielectricFrame {
    V3 n;
    float eta_i, eta_t, eta, cos_o;
};

__device__ inline DielectricFrame MakeDielectricFrame(V3 wo, V3 n, float ior) {
    const bool entering = Dot(n, wo) >= 0.0f;
    const V3 on = entering ? n : -n;
    const float ei = entering ? 1.0f : fmaxf(1.0f, ior);
    const float et = entering ? fmaxf(1.0f, ior) : 1.0f;
    return DielectricFrame{on, ei, et, ei / et, fmaxf(0.0f, Dot(on, wo))};
}

// Non-layered BSDFs (the layered kinds evaluate through their base).
__device__ inline V3 EvalSimple(const Mat& m, V3 wo, V3 wi, V3 n) {
    switch (m.kind) {
        case kDiffuse:
        case kDiffuseTransmission:
        case kMix:
            if (!IsAbove(wo, n) || !IsAbove(wi, n)) return {0, 0, 0};
            return m.reflectance / kPi;
        case kMeasured:
            if (m.measured) return EvalMeasured(*m.measured, wo, wi, n);
            [[fallthrough]];
        case kConductor:
            if (m.ur <= kDeltaRoughness && m.vr <= kDeltaRoughness) return {0, 0, 0};
            return GgxSpecularBrdf(m.reflectance, m.ur, wo, wi, n);
        case kThinDielectric: {
            if (m.ur <= kDeltaRoughness) return {0, 0, 0};
            const V3 fwd = Normalize(-wo);
            if (fmaxf(0.0f, Dot(fwd, wi)) <= 0.0f) return {0, 0, 0};
            const float fr = FresnelDielectric(fabsf(Dot(n, wo)), 1.0f, fmaxf(1.0f, m.ior));
            return (m.reflectance / kPi) * (1.0f - fr);
        }
        case kDielectric:
            if (m.ur <= kDeltaRoughness) return {0, 0, 0};
            return SameHemisphere(wo, wi, n) ? GgxDielectricReflection(m.reflectance, m.ior, m.ur, wo, wi, n)
                                             : GgxDielectricTransmission(m.reflectance, m.ior, m.ur, wo, wi, n);
        case kSubsurfaceExit: {
            if (!IsAbove(wo, n) || !IsAbove(wi, n)) return {0, 0, 0};
            const float sw = SubsurfaceSw(fmaxf(0.0f, Dot(n, wi)), m.ior);
            return V3{sw, sw, sw};
        }
        default:
            return {0, 0, 0};
    }
}

__device__ inline float PdfSimple(const Mat& m, V3 wo, V3 wi, V3 n) {
    switch (m.kind) {
        case kDiffuse:
        case kDiffuseTransmission:
        case kMix:
        case kSubsurfaceExit:
            if (!IsAbove(wo, n) || !IsAbove(wi, n)) return 0.0f;
            return fmaxf(0.0f, Dot(n, wi)) / kPi;
        case kMeasured:
            if (m.measured) return PdfMeasuredBrdf(*m.measured, wo, wi, n);
            [[fallthrough]];
        case kConductor:
            if (m.ur <= kDeltaRoughness && m.vr <= kDeltaRoughness) return 0.0f;
            return GgxReflectionPdf(m.ur, wo, wi, n);
        case kThinDielectric: {
            if (m.ur <= kDeltaRoughness) return 0.0f;
            return fmaxf(0.0f, Dot(Normalize(-wo), wi)) / kPi;
        }
        case kDielectric:
            if (m.ur <= kDeltaRoughness) return 0.0f;
            return SameHemisphere(wo, wi, n) ? GgxDielectricReflectionPdf(m.ior, m.ur, wo, wi, n)
                                             : GgxDielectricTransmissionPdf(m.ior, m.ur, wo, wi, n);
        default:
            return 0.0f;
    }
}

__device__ inline BsdfSample SampleSimple(const Mat& m, V3 wo, V3 n, float sx, float sy) {
    switch (m.kind) {
        case kDiffuse:
        case kDiffuseTransmission:
        case kMix: {
            if (!IsAbove(wo, n) || IsBlack(m.reflectance)) return NoSample();
            const V3 wi = SampleCosineHemisphere(n, sx, sy);
            return BsdfSample{wi, m.reflectance, PdfSimple(m, wo, wi, n), true, false};
        }
        case kMeasured:
            if (m.measured) return SampleMeasuredBrdf(*m.measured, wo, n, sx, sy);
            [[fallthrough]];
        case kConductor:
            if (m.ur <= kDeltaRoughness && m.vr <= kDeltaRoughness) {
                if (!IsAbove(wo, n) || IsBlack(m.reflectance)) return NoSample();
                return BsdfSample{Reflect(-wo, n), m.reflectance, 1.0f, true, true};
            }
            return SampleGgxReflection(wo, n, sx, sy, m.reflectance, m.ur);
        case kThinDielectric: {
            if (IsBlack(m.reflectance)) return NoSample();
            const V3 on = Dot(n, wo) >= 0.0f ? n : -n;
            const float fr = FresnelDielectric(fabsf(Dot(on, wo)), 1.0f, fmaxf(1.0f, m.ior));
            if (m.ur <= kDeltaRoughness) {
                if (sx < fr) return BsdfSample{Reflect(-wo, on), m.reflectance, 1.0f, true, true};
                return BsdfSample{Normalize(-wo), m.reflectance, 1.0f, true, true};
            }
            if (sx < fr) {
                const float rx = fr > 0.0f ? sx / fr : sx;
                BsdfSample r = SampleGgxReflection(wo, on, rx, sy, m.reflectance * fr, m.ur);
                if (r.valid) r.specular = false;
                return r;
            }
            const float rx = (1.0f - fr) > 0.0f ? (sx - fr) / (1.0f - fr) : sx;
            const V3 fwd = Normalize(-wo);
            const V3 wi = SampleCosineHemisphere(fwd, rx, sy);
            const float pdf = fmaxf(0.0f, Dot(fwd, wi)) / kPi;
            if (pdf <= 0.0f) return NoSample();
            return BsdfSample{wi, m.reflectance * (1.0f - fr), pdf, true, false};
        }
        case kDielectric: {
            if (IsBlack(m.reflectance)) return NoSample();
            const DielectricFrame fr = MakeDielectricFrame(wo, n, m.ior);
            if (m.ur <= kDeltaRoughness) {
                V3 refr;
                const bool can = Refract(wo, fr.n, fr.eta, refr);
                const float f = can ? FresnelDielectric(fr.cos_o, fr.eta_i, fr.eta_t) : 1.0f;
                if (!can || sx < f) return BsdfSample{Reflect(-wo, fr.n), m.reflectance, 1.0f, true, true};
                return BsdfSample{refr, m.reflectance, 1.0f, true, true};
            }
            V3 h = SampleGgxHalf(fr.n, m.ur, sx, sy);
            if (Dot(h, wo) < 0.0f) h = -h;
            const float f = FresnelDielectric(fabsf(Dot(wo, h)), fr.eta_i, fr.eta_t);
            if (sx < f) {
                const float rx = f > 0.0f ? sx / f : sx;
                h = SampleGgxHalf(fr.n, m.ur, rx, sy);
                if (Dot(h, wo) < 0.0f) h = -h;
                const V3 wi = Reflect(-wo, h);
                const float pdf = PdfSimple(m, wo, wi, n);
                if (pdf <= 0.0f) return NoSample();
                const V3 fv = EvalSimple(m, wo, wi, n);
                return BsdfSample{wi, fv * (AbsDot(n, wi) / pdf), pdf, true, false};
            }
            const float rx = (1.0f - f) > 0.0f ? (sx - f) / (1.0f - f) : sx;
            h = SampleGgxHalf(fr.n, m.ur, rx, sy);
            if (Dot(h, wo) < 0.0f) h = -h;
            V3 wi;
            if (!Refract(wo, h, fr.eta, wi)) return BsdfSample{Reflect(-wo, h), m.reflectance, 1.0f, true, true};
            const float pdf = PdfSimple(m, wo, wi, n);
            if (pdf <= 0.0f) return NoSample();
            const V3 fv = EvalSimple(m, wo, wi, n);
            return BsdfSample{wi, fv * (AbsDot(n, wi) / pdf), pdf, true, false};
        }
        case kSubsurfaceExit: {
            if (!IsAbove(wo, n)) return NoSample();
            const V3 wi = SampleCosineHemisphere(n, sx, sy);
            const float pdf = fmaxf(0.0f, Dot(n, wi)) / kPi;
            if (pdf <= 0.0f) return NoSample();
            const float w = SubsurfaceSw(fmaxf(0.0f, Dot(n, wi)), m.ior) * kPi;
            return BsdfSample{wi, V3{w, w, w}, pdf, true, false};
        }
        default:
            return NoSample();
    }
}

// ------------------------------------------------------------- layered walk

__device__ inline V3 BeerLambertLayer(V3 tp, V3 absorption, float thickness, V3 w, V3 n) {
    const float c = fmaxf(1.0e-4f, fabsf(Dot(w, n)));
    const float dist = thickness / c;
    return V3{tp.x * expf(-absorption.x * dist), tp.y * expf(-absorption.y * dist), tp.z * expf(-absorption.z * dist)};
}

__device__ inline Mat LayeredBase(const Mat& m) {
    Mat b = m;
    b.kind = m.kind == kCoatedConductor ? kConductor : kDiffuse;
    if (b.kind == kDiffuse) b.ur = b.vr = 0.0f;
    return b;
}

__device__ inline float PdfLayered(const Mat& m, V3 wo, V3 wi, V3 n, Pcg32& rng) {
    if (!IsAbove(wo, n) || !IsAbove(wi, n)) return 0.0f;
    const float ce = fmaxf(1.0f, m.coating_ior);
    const Mat base = LayeredBase(m);
    V3 wo_t, wi_down;
    if (!Refract(wo, n, 1.0f / ce, wo_t)) return 0.0f;
    if (!Refract(wi, n, 1.0f / ce, wi_down)) return 0.0f;
    const V3 wi_int = -wi_down;
    if (!IsAbove(wi_int, n)) return 0.0f;
    const float t_enter = 1.0f - FresnelDielectric(fmaxf(0.0f, Dot(wo, n)), 1.0f, ce);
    const float t_exit = 1.0f - FresnelDielectric(fmaxf(0.0f, Dot(wi, n)), 1.0f, ce);
    if (t_enter <= 0.0f || t_exit <= 0.0f) return 0.0f;
    const float cos_wi = fmaxf(0.0f, Dot(wi, n));
    const float cos_int = fmaxf(1.0e-4f, Dot(wi_int, n));
    const float coupling = t_exit * cos_wi / (ce * ce * cos_int);
    const int ns = max(1, m.coat_nsamples);
    double sum = 0.0;
    for (int s = 0; s < ns; ++s) {
        float reach = t_enter;
        V3 w = wo_t;
        for (int depth = 0; depth < m.coat_maxdepth; ++depth) {
            const float bp = PdfSimple(base, -w, wi_int, n);
            sum += static_cast<double>(reach) * bp * coupling;
            const float r0 = rng.NextFloat();
            const float r1 = rng.NextFloat();
            const BsdfSample bs = SampleSimple(base, -w, n, r0, r1);
            if (!bs.valid || !IsAbove(bs.wi, n)) break;
            reach *= FresnelDielectric(fmaxf(0.0f, Dot(bs.wi, n)), ce, 1.0f);
            if (reach <= 0.0f) break;
            w = Reflect(bs.wi, n);
            if (IsAbove(w, n)) break;
        }
    }
    const float estimate = static_cast<float>(sum / ns);
    return 0.9f * estimate + 0.1f * (1.0f / (4.0f * kPi));
}

__device__ inline V3 EvalLayered(const Mat& m, V3 wo, V3 wi, V3 n, Pcg32& rng) {
    if (!IsAbove(wo, n) || !IsAbove(wi, n)) return {0, 0, 0};
    const float ce = fmaxf(1.0f, m.coating_ior);
    const Mat base = LayeredBase(m);
    V3 wo_t, wi_down;
    if (!Refract(wo, n, 1.0f / ce, wo_t)) return {0, 0, 0};
    if (!Refract(wi, n, 1.0f / ce, wi_down)) return {0, 0, 0};
    const V3 wi_int = -wi_down;
    if (!IsAbove(wi_int, n)) return {0, 0, 0};
    const float t_enter = 1.0f - FresnelDielectric(fmaxf(0.0f, Dot(wo, n)), 1.0f, ce);
    const float t_exit = 1.0f - FresnelDielectric(fmaxf(0.0f, Dot(wi, n)), 1.0f, ce);
    if (t_enter <= 0.0f || t_exit <= 0.0f) return {0, 0, 0};
    const int ns = max(1, m.coat_nsamples);
    V3 sum{0, 0, 0};
    for (int s = 0; s < ns; ++s) {
        V3 beta{t_enter, t_enter, t_enter};
        V3 w = wo_t;
        for (int depth = 0; depth < m.coat_maxdepth; ++depth) {
            beta = BeerLambertLayer(beta, m.coat_absorption, m.coat_thickness, w, n);
            const V3 bf = EvalSimple(base, -w, wi_int, n);
            if (!IsBlack(bf)) {
                const V3 tr = BeerLambertLayer(V3{1, 1, 1}, m.coat_absorption, m.coat_thickness, wi_int, n);
                const float ec = t_exit / (ce * ce);
                sum = sum + V3{beta.x * bf.x * tr.x * ec, beta.y * bf.y * tr.y * ec, beta.z * bf.z * tr.z * ec};
            }
            const float r0 = rng.NextFloat();
            const float r1 = rng.NextFloat();
            const BsdfSample bs = SampleSimple(base, -w, n, r0, r1);
            if (!bs.valid || IsBlack(bs.weight) || !IsAbove(bs.wi, n)) break;
            beta = Mul(beta, bs.weight);
            beta = BeerLambertLayer(beta, m.coat_absorption, m.coat_thickness, bs.wi, n);
            const float fb = FresnelDielectric(fmaxf(0.0f, Dot(bs.wi, n)), ce, 1.0f);
            if (rng.NextFloat() < fb) {
                w = Reflect(bs.wi, n);
                if (IsAbove(w, n)) break;
                continue;
            }
            break;
        }
    }
    return sum / static_cast<float>(ns);
}

__device__ inline BsdfSample SampleLayered(const Mat& m, V3 wo, V3 n, Pcg32& rng) {
    if (!IsAbove(wo, n)) return NoSample();
    const float ce = fmaxf(1.0f, m.coating_ior);
    const Mat base = LayeredBase(m);
    const float cos_o = fmaxf(0.0f, Dot(wo, n));
    const float f_enter = FresnelDielectric(cos_o, 1.0f, ce);
    if (rng.NextFloat() < f_enter) {
        const V3 wr = Reflect(-wo, n);
        if (!IsAbove(wr, n)) return NoSample();
        return BsdfSample{wr, V3{1, 1, 1}, 1.0f, true, true};
    }
    V3 w;
    if (!Refract(wo, n, 1.0f / ce, w)) {
        const V3 wr = Reflect(-wo, n);
        return IsAbove(wr, n) ? BsdfSample{wr, V3{1, 1, 1}, 1.0f, true, true} : NoSample();
    }
    V3 tp{1, 1, 1};
    for (int depth = 0; depth < m.coat_maxdepth; ++depth) {
        tp = BeerLambertLayer(tp, m.coat_absorption, m.coat_thickness, w, n);
        const float r0 = rng.NextFloat();
        const float r1 = rng.NextFloat();
        const BsdfSample bs = SampleSimple(base, -w, n, r0, r1);
        if (!bs.valid || IsBlack(bs.weight)) return NoSample();
        tp = Mul(tp, bs.weight);
        w = bs.wi;
        if (!IsAbove(w, n)) return NoSample();
        tp = BeerLambertLayer(tp, m.coat_absorption, m.coat_thickness, w, n);
        const float cos_t = fmaxf(0.0f, Dot(w, n));
        const float f_back = FresnelDielectric(cos_t, ce, 1.0f);
        if (rng.NextFloat() < f_back) {
            w = Reflect(w, n);
            if (IsAbove(w, n)) return NoSample();
            continue;
        }
        V3 wexit;
        if (!Refract(w, n, ce, wexit)) {
            w = Reflect(w, n);
            continue;
        }
        wexit = -wexit;
        if (!IsAbove(wexit, n)) return NoSample();
        const float pdf = PdfLayered(m, wo, wexit, n, rng);
        return BsdfSample{wexit, tp, fmaxf(pdf, 1.0e-4f), true, false};
    }
    return NoSample();
}

// ------------------------------------------------------------ dispatch

__device__ __forceinline__ bool IsLayered(int32_t kind) { return kind == kCoatedDiffuse || kind == kCoatedConductor; }

__device__ inline V3 EvalBsdf(const Mat& m, V3 wo, V3 wi, V3 n, Pcg32& rng) {
    return IsLayered(m.kind) ? EvalLayered(m, wo, wi, n, rng) : EvalSimple(m, wo, wi, n);
}

__device__ inline float PdfBsdf(const Mat& m, V3 wo, V3 wi, V3 n, Pcg32& rng) {
    return IsLayered(m.kind) ? PdfLayered(m, wo, wi, n, rng) : PdfSimple(m, wo, wi, n);
}

__device__ inline BsdfSample SampleBsdf(const Mat& m, V3 wo, V3 n, float sx, float sy, Pcg32& rng) {
    return IsLayered(m.kind) ? SampleLayered(m, wo, n, rng) : SampleSimple(m, wo, n, sx, sy);
}

}  // namespace yrc
