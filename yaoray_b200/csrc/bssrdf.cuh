// Tabulated separable BSSRDF on the device: Catmull-Rom interpolation of the
// photon-beam-diffusion profile table (rho x optical radius), radius
// sampling by inverting the interpolated radial CDF, and the spatial pdf over
// the three projection axes and three colour channels.
//
// Follows the reference's TabulatedBSSRDF (src/shading/bssrdf.cpp:153-266)
// and its Catmull-Rom helpers (src/shading/catmull_rom.cpp:30-197), which
// restate pbrt-v4's published formulation; the render translation unit is
// compiled without FMA contraction so the arithmetic rounds as the
// reference's.
#pragma once

#include "render_types.hpp"
#include "shading.cuh"

namespace yrc {

// Index of the last interval [nodes[i], nodes[i+1]) whose left end satisfies
// `pred`, clamped to [0, n - 2] (binary search).
template <typename Pred>
__device__ __forceinline__ int FindSplineInterval(int n, Pred pred) {
    int size = n - 2;
    int first = 1;
    while (size > 0) {
        const int half = size >> 1;
        const int middle = first + half;
        if (pred(middle)) {
            first = middle + 1;
            size -= half + 1;
        } else {
            size = half;
        }
    }
    return min(max(first - 1, 0), n - 2);
}

// Catmull-Rom spline weights of the 4 nodes around x (offset = first node);
// false when x lies outside [nodes[0], nodes[n-1]].
__device__ inline bool SplineWeights(int n, const float* nodes, float x, int& offset, float w[4]) {
    if (!(x >= nodes[0] && x <= nodes[n - 1])) return false;
    const int idx = FindSplineInterval(n, [&](int i) { return nodes[i] <= x; });
    offset = idx - 1;
    const float x0 = nodes[idx], x1 = nodes[idx + 1];
    const float t = (x - x0) / (x1 - x0);
    const float t2 = t * t, t3 = t2 * t;
    w[1] = 2.0f * t3 - 3.0f * t2 + 1.0f;
    w[2] = -2.0f * t3 + 3.0f * t2;
    if (idx > 0) {
        const float w0 = (t3 - 2.0f * t2 + t) * (x1 - x0) / (x1 - nodes[idx - 1]);
        w[0] = -w0;
        w[2] += w0;
    } else {
        const float w0 = t3 - 2.0f * t2 + t;
        w[0] = 0.0f;
        w[1] -= w0;
        w[2] += w0;
    }
    if (idx + 2 < n) {
        const float w3 = (t3 - t2) * (x1 - x0) / (nodes[idx + 2] - x0);
        w[1] -= w3;
        w[3] = w3;
    } else {
        const float w3 = t3 - t2;
        w[1] -= w3;
        w[2] += w3;
        w[3] = 0.0f;
    }
    return true;
}

// Samples the second dimension of a 2-D Catmull-Rom tabulated function at
// first-dimension parameter `alpha`, by inverting the interpolated CDF with
// Newton-bisection; returns the sampled node-space value (0 when alpha is
// out of range).
__device__ inline float SampleSpline2D(int size1, int size2, const float* nodes1, const float* nodes2,
                                       const float* values, const float* cdf, float alpha, float u) {
    int offset;
    float w[4];
    if (!SplineWeights(size1, nodes1, alpha, offset, w)) return 0.0f;
    auto interp = [&](const float* arr, int idx) {
        float v = 0.0f;
        for (int i = 0; i < 4; ++i)
            if (w[i] != 0.0f) v += arr[(offset + i) * size2 + idx] * w[i];
        return v;
    };
    const float maximum = interp(cdf, size2 - 1);
    u *= maximum;
    const int idx = FindSplineInterval(size2, [&](int i) { return interp(cdf, i) <= u; });
    const float f0 = interp(values, idx), f1 = interp(values, idx + 1);
    const float x0 = nodes2[idx], x1 = nodes2[idx + 1];
    const float width = x1 - x0;
    u = (u - interp(cdf, idx)) / width;
    float d0, d1;
    if (idx > 0) {
        d0 = width * (f1 - interp(values, idx - 1)) / (x1 - nodes2[idx - 1]);
    } else {
        d0 = f1 - f0;
    }
    if (idx + 2 < size2) {
        d1 = width * (interp(values, idx + 2) - f0) / (nodes2[idx + 2] - x0);
    } else {
        d1 = f1 - f0;
    }
    float t = (f0 != f1) ? (f0 - sqrtf(fmaxf(0.0f, f0 * f0 + 2.0f * u * (f1 - f0)))) / (f0 - f1)
                         : (f0 != 0.0f ? u / f0 : 0.0f);
    float a = 0.0f, b = 1.0f;
    // The reference iterates until convergence; 64 Newton-bisection steps
    // bound the loop on the device (each halves [a, b] at worst).
    for (int iter = 0; iter < 64; ++iter) {
        if (!(t >= a && t <= b)) t = 0.5f * (a + b);
        const float Fhat =
            t * (f0 + t * (0.5f * d0 + t * ((1.0f / 3.0f) * (-2.0f * d0 - d1) + f1 - f0 +
                                            t * (0.25f * (d0 + d1) + 0.5f * (f0 - f1)))));
        const float fhat = f0 + t * (d0 + t * (-2.0f * d0 - d1 + 3.0f * (f1 - f0) + t * (d0 + d1 + 2.0f * (f0 - f1))));
        if (fabsf(Fhat - u) < 1.0e-6f || b - a < 1.0e-6f) break;
        if (Fhat - u < 0.0f) {
            a = t;
        } else {
            b = t;
        }
        t -= (Fhat - u) / fhat;
    }
    return x0 + width * t;
}

// One shading point's TabulatedBSSRDF: per-channel extinction and albedo.
struct TabBssrdf {
    float st[3];
    float rho[3];
    float eta;
    DevBssrdf table;
};

__device__ inline TabBssrdf MakeTabBssrdf(const DevMaterial& m, const DevBssrdf& table) {
    TabBssrdf b;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        b.st[k] = m.sigma_a[k] + m.sigma_s[k];
        b.rho[k] = b.st[k] != 0.0f ? m.sigma_s[k] / b.st[k] : 0.0f;
    }
    b.eta = m.bssrdf_eta;
    b.table = table;
    return b;
}

// Radial profile Sr(r) per channel.
__device__ inline V3 BssrdfSr(const TabBssrdf& b, float r) {
    float out[3] = {0.0f, 0.0f, 0.0f};
    const DevBssrdf& t = b.table;
    for (int ch = 0; ch < 3; ++ch) {
        const float ro = r * b.st[ch];
        int rho_off, rad_off;
        float rho_w[4], rad_w[4];
        if (!SplineWeights(t.rho_count, t.rho, b.rho[ch], rho_off, rho_w) ||
            !SplineWeights(t.radius_count, t.radius, ro, rad_off, rad_w)) {
            continue;
        }
        float sr = 0.0f;
        for (int i = 0; i < 4; ++i) {
            for (int j = 0; j < 4; ++j) {
                const float w = rho_w[i] * rad_w[j];
                if (w != 0.0f) sr += w * t.profile[(rho_off + i) * t.radius_count + rad_off + j];
            }
        }
        if (ro != 0.0f) sr /= 2.0f * kPi * ro;
        out[ch] = sr;
    }
    return V3{fmaxf(0.0f, out[0] * b.st[0] * b.st[0]), fmaxf(0.0f, out[1] * b.st[1] * b.st[1]),
              fmaxf(0.0f, out[2] * b.st[2] * b.st[2])};
}

// Sampled radius for channel ch (-1 when the channel does not scatter).
__device__ inline float BssrdfSampleSr(const TabBssrdf& b, int ch, float u) {
    if (b.st[ch] == 0.0f) return -1.0f;
    const DevBssrdf& t = b.table;
    return SampleSpline2D(t.rho_count, t.radius_count, t.rho, t.radius, t.profile, t.profile_cdf, b.rho[ch], u) /
           b.st[ch];
}

__device__ inline float BssrdfPdfSr(const TabBssrdf& b, int ch, float r) {
    const DevBssrdf& t = b.table;
    const float ro = r * b.st[ch];
    int rho_off, rad_off;
    float rho_w[4], rad_w[4];
    if (!SplineWeights(t.rho_count, t.rho, b.rho[ch], rho_off, rho_w) ||
        !SplineWeights(t.radius_count, t.radius, ro, rad_off, rad_w)) {
        return 0.0f;
    }
    float sr = 0.0f, rho_eff = 0.0f;
    for (int i = 0; i < 4; ++i) {
        if (rho_w[i] == 0.0f) continue;
        rho_eff += t.rho_eff[rho_off + i] * rho_w[i];
        for (int j = 0; j < 4; ++j) {
            if (rad_w[j] == 0.0f) continue;
            sr += t.profile[(rho_off + i) * t.radius_count + rad_off + j] * rho_w[i] * rad_w[j];
        }
    }
    if (ro != 0.0f) sr /= 2.0f * kPi * ro;
    if (rho_eff <= 0.0f) return 0.0f;
    return fmaxf(0.0f, sr * b.st[ch] * b.st[ch] / rho_eff);
}

// Area-measure pdf of the exit point pi (normal ni) from the entry po with
// frame (ss, ts, ns): MIS over the projection axes (0.25, 0.25, 0.5) and the
// three channels (1/3 each).
__device__ inline float BssrdfPdfSp(const TabBssrdf& b, V3 po, V3 ss, V3 ts, V3 ns, V3 pi, V3 ni) {
    const V3 d = po - pi;
    const float dl[3] = {Dot(ss, d), Dot(ts, d), Dot(ns, d)};
    const float nl[3] = {Dot(ss, ni), Dot(ts, ni), Dot(ns, ni)};
    const float rproj[3] = {sqrtf(dl[1] * dl[1] + dl[2] * dl[2]), sqrtf(dl[2] * dl[2] + dl[0] * dl[0]),
                            sqrtf(dl[0] * dl[0] + dl[1] * dl[1])};
    const float axis_prob[3] = {0.25f, 0.25f, 0.5f};
    const float ch_prob = 1.0f / 3.0f;
    float pdf = 0.0f;
    for (int axis = 0; axis < 3; ++axis)
        for (int ch = 0; ch < 3; ++ch) pdf += BssrdfPdfSr(b, ch, rproj[axis]) * fabsf(nl[axis]) * ch_prob * axis_prob[axis];
    return pdf;
}

// Orthonormal frame about ns (path_integrator.cpp:106-110).
__device__ inline void BssrdfFrame(V3 ns, V3& ss, V3& ts) {
    ss = fabsf(ns.x) > 0.9f ? Normalize(Cross(ns, V3{0.0f, 1.0f, 0.0f})) : Normalize(Cross(ns, V3{1.0f, 0.0f, 0.0f}));
    ts = Cross(ns, ss);
}

}  // namespace yrc
