// Host builder of the tabulated photon-beam-diffusion BSSRDF profile used by
// subsurface materials: ComputeBeamDiffusionBSSRDF and its helpers
// (src/shading/bssrdf.cpp:19-151, src/shading/catmull_rom.cpp:66-88 in the
// reference), a restatement of pbrt-v4's published method. Compiled without
// FMA contraction, with the same libm calls, so the tables match the
// reference's bit for bit.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "yrc_internal.hpp"

namespace yrc {
namespace {

constexpr float kPiF = 3.14159265358979323846f;
constexpr float kInv4Pi = 0.07957747154594767f;

float SafeSqrt(float x) { return std::sqrt(std::max(0.0f, x)); }

float FrDielectricHost(float cos_i, float eta) {
    cos_i = std::clamp(cos_i, -1.0f, 1.0f);
    if (cos_i < 0) {
        eta = 1.0f / eta;
        cos_i = -cos_i;
    }
    const float sin2_i = 1.0f - cos_i * cos_i;
    const float sin2_t = sin2_i / (eta * eta);
    if (sin2_t >= 1.0f) return 1.0f;
    const float cos_t = SafeSqrt(1.0f - sin2_t);
    const float r_parl = (eta * cos_i - cos_t) / (eta * cos_i + cos_t);
    const float r_perp = (cos_i - eta * cos_t) / (cos_i + eta * cos_t);
    return 0.5f * (r_parl * r_parl + r_perp * r_perp);
}

float HenyeyGreensteinHost(float cos_theta, float g) {
    const float denom = 1.0f + g * g + 2.0f * g * cos_theta;
    return kInv4Pi * (1.0f - g * g) / (denom * SafeSqrt(denom));
}

float FresnelMoment1Host(float eta) {
    const float e2 = eta * eta, e3 = e2 * eta, e4 = e3 * eta, e5 = e4 * eta;
    if (eta < 1) return 0.45966f - 1.73965f * eta + 3.37668f * e2 - 3.904945f * e3 + 2.49277f * e4 - 0.68441f * e5;
    return -4.61686f + 11.1136f * eta - 10.4646f * e2 + 5.11455f * e3 - 1.27198f * e4 + 0.12746f * e5;
}

float FresnelMoment2Host(float eta) {
    const float e2 = eta * eta, e3 = e2 * eta, e4 = e3 * eta, e5 = e4 * eta;
    if (eta < 1) return 0.27614f - 0.87350f * eta + 1.12077f * e2 - 0.65095f * e3 + 0.07883f * e4 + 0.04860f * e5;
    return -547.033f + 45.3087f / e3 - 218.725f / e2 + 458.843f / eta + 404.557f * eta - 189.519f * e2 +
           54.9327f * e3 - 9.00603f * e4 + 0.63942f * e5;
}

// Multiple-scattering fluence of the photon beam diffusion dipole at radius r.
float BeamMultiple(float sigma_s, float sigma_a, float g, float eta, float r) {
    const int samples = 100;
    float ed = 0;
    const float sps = sigma_s * (1 - g);
    const float spt = sigma_a + sps;
    const float rhop = sps / spt;
    const float d_g = (2 * sigma_a + sps) / (3 * spt * spt);
    const float sigma_tr = std::sqrt(sigma_a / d_g);
    const float fm1 = FresnelMoment1Host(eta), fm2 = FresnelMoment2Host(eta);
    const float ze = -2 * d_g * (1 + 3 * fm2) / (1 - 2 * fm1);
    const float c_phi = 0.25f * (1 - 2 * fm1), c_e = 0.5f * (1 - 3 * fm2);
    for (int i = 0; i < samples; ++i) {
        const float zr = -std::log(1 - (i + 0.5f) / samples) / spt;
        const float zv = -zr + 2 * ze;
        const float dr = std::sqrt(r * r + zr * zr);
        const float dv = std::sqrt(r * r + zv * zv);
        const float phi_d = kInv4Pi / d_g * (std::exp(-sigma_tr * dr) / dr - std::exp(-sigma_tr * dv) / dv);
        const float ed_n = kInv4Pi * (zr * (1 + sigma_tr * dr) * std::exp(-sigma_tr * dr) / (dr * dr * dr) -
                                      zv * (1 + sigma_tr * dv) * std::exp(-sigma_tr * dv) / (dv * dv * dv));
        const float e = phi_d * c_phi + ed_n * c_e;
        const float kappa = 1 - std::exp(-2 * spt * (dr + zr));
        ed += rhop * rhop * std::exp(-spt * zr) * kappa * e / samples;
    }
    return ed;
}

// Single-scattering term at radius r.
float BeamSingle(float sigma_s, float sigma_a, float g, float eta, float r) {
    const float sigma_t = sigma_a + sigma_s;
    const float rho = sigma_s / sigma_t;
    const float t_crit = r * SafeSqrt(1 - 1 / (eta * eta));
    float ess = 0;
    const int samples = 100;
    for (int i = 0; i < samples; ++i) {
        const float ti = t_crit - std::log(1 - (i + 0.5f) / samples) / sigma_t;
        const float d = std::sqrt(r * r + ti * ti);
        const float cos_o = ti / d;
        ess += rho * std::exp(-sigma_t * (d + ti)) / (d * d) * HenyeyGreensteinHost(cos_o, g) *
               (1 - FrDielectricHost(-cos_o, eta)) * std::abs(cos_o);
    }
    return ess / samples;
}

// Integral of the Catmull-Rom interpolant of `values` over the nodes `x`,
// with its running CDF.
float IntegrateSpline(int n, const float* x, const float* values, float* cdf) {
    float sum = 0;
    cdf[0] = 0;
    for (int i = 0; i < n - 1; ++i) {
        const float x0 = x[i], x1 = x[i + 1];
        const float f0 = values[i], f1 = values[i + 1];
        const float width = x1 - x0;
        const float d0 = i > 0 ? width * (f1 - values[i - 1]) / (x1 - x[i - 1]) : f1 - f0;
        const float d1 = i + 2 < n ? width * (values[i + 2] - f0) / (x[i + 2] - x0) : f1 - f0;
        sum += ((d0 - d1) * (1.0f / 12.0f) + (f0 + f1) * 0.5f) * width;
        cdf[i + 1] = sum;
    }
    return sum;
}

}  // namespace
}  // namespace yrc

extern "C" yrc_status yrc_bssrdf_table_build(float g, float eta, int32_t rho_count, int32_t radius_count,
                                             float* rho_samples, float* radius_samples, float* profile,
                                             float* rho_eff, float* profile_cdf) {
    using namespace yrc;
    if (rho_count < 4 || radius_count < 4 || !rho_samples || !radius_samples || !profile || !rho_eff || !profile_cdf ||
        !(eta > 0.0f)) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_bssrdf_table_build: bad argument");
    }
    radius_samples[0] = 0.0f;
    radius_samples[1] = 2.5e-3f;
    for (int i = 2; i < radius_count; ++i) radius_samples[i] = radius_samples[i - 1] * 1.2f;
    for (int i = 0; i < rho_count; ++i) {
        rho_samples[i] = (1 - std::exp(-8.0f * i / static_cast<float>(rho_count - 1))) / (1 - std::exp(-8.0f));
    }
    for (int i = 0; i < rho_count; ++i) {
        for (int j = 0; j < radius_count; ++j) {
            const float rho = rho_samples[i];
            const float r = radius_samples[j];
            profile[static_cast<size_t>(i) * radius_count + j] =
                2 * kPiF * r * (BeamMultiple(rho, 1 - rho, g, eta, r) + BeamSingle(rho, 1 - rho, g, eta, r));
        }
        rho_eff[i] = IntegrateSpline(radius_count, radius_samples, profile + static_cast<size_t>(i) * radius_count,
                                     profile_cdf + static_cast<size_t>(i) * radius_count);
    }
    return Ok();
}
