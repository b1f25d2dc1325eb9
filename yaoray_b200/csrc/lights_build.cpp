// Host-side light preparation with the reference's exact tables:
//   BuildAliasTable (src/lighting/light_sampling.cpp:148-183): Vose's alias
//     method with LIFO small/large work lists, so equal inputs give the same
//     probability / alias columns as the reference's PrepareLightSampling;
//   BuildEnvironmentDistribution (src/lighting/environment.cpp:73-123):
//     luminance * sin(theta) texel weights, per-row running sums and a row CDF.
#include <algorithm>
#include <cmath>
#include <vector>

#include "yrc_internal.hpp"

extern "C" {

yrc_status yrc_alias_table_build(const float* weights, int32_t count, float* probability, int32_t* alias,
                                 float* pmf) {
    if (count < 0 || (count > 0 && (!weights || !probability || !alias || !pmf))) {
        return yrc::Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_alias_table_build: bad argument");
    }
    if (count == 0) return yrc::Ok();
    float total = 0.0f;
    for (int32_t i = 0; i < count; ++i) {
        if (std::isfinite(weights[i]) && weights[i] > 0.0f) total += weights[i];
    }
    std::vector<float> scaled(static_cast<size_t>(count));
    std::vector<int32_t> small, large;
    small.reserve(static_cast<size_t>(count));
    large.reserve(static_cast<size_t>(count));
    for (int32_t i = 0; i < count; ++i) {
        const float w = std::isfinite(weights[i]) && weights[i] > 0.0f ? weights[i] : 0.0f;
        pmf[i] = total > 0.0f ? w / total : 1.0f / static_cast<float>(count);
        probability[i] = 1.0f;
        scaled[static_cast<size_t>(i)] = pmf[i] * static_cast<float>(count);
        alias[i] = i;
        (scaled[static_cast<size_t>(i)] < 1.0f ? small : large).push_back(i);
    }
    while (!small.empty() && !large.empty()) {
        const int32_t lo = small.back();
        small.pop_back();
        const int32_t hi = large.back();
        large.pop_back();
        probability[lo] = scaled[static_cast<size_t>(lo)];
        alias[lo] = hi;
        scaled[static_cast<size_t>(hi)] = scaled[static_cast<size_t>(hi)] + scaled[static_cast<size_t>(lo)] - 1.0f;
        (scaled[static_cast<size_t>(hi)] < 1.0f ? small : large).push_back(hi);
    }
    return yrc::Ok();
}

yrc_status yrc_environment_distribution_build(const float* texels, int32_t width, int32_t height,
                                              float* texel_weights, float* row_weights, float* row_cdf,
                                              float* conditional_cdfs, float* total_weight) {
    if (width <= 0 || height <= 0 || !texel_weights || !row_weights || !row_cdf || !conditional_cdfs ||
        !total_weight) {
        return yrc::Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_environment_distribution_build: bad argument");
    }
    const float pi = 3.14159265358979323846f;
    float total = 0.0f;
    for (int32_t y = 0; y < height; ++y) {
        const float theta = (static_cast<float>(y) + 0.5f) * pi / static_cast<float>(height);
        const float sin_theta = std::max(1.0e-6f, std::sin(theta));
        float row = 0.0f;
        for (int32_t x = 0; x < width; ++x) {
            const size_t i = static_cast<size_t>(y) * static_cast<size_t>(width) + static_cast<size_t>(x);
            const float* c = texels ? texels + 4 * i : nullptr;
            const float lum = c ? std::max(0.0f, 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2]) : 0.0f;
            const float w = lum * sin_theta;
            texel_weights[i] = w;
            row += w;
            conditional_cdfs[i] = row;
        }
        row_weights[y] = row;
        total += row;
        row_cdf[y] = total;
    }
    if (total <= 0.0f || !std::isfinite(total)) {
        total = static_cast<float>(width * height);
        for (int32_t y = 0; y < height; ++y) {
            float row = 0.0f;
            for (int32_t x = 0; x < width; ++x) {
                const size_t i = static_cast<size_t>(y) * static_cast<size_t>(width) + static_cast<size_t>(x);
                texel_weights[i] = 1.0f;
                row += 1.0f;
                conditional_cdfs[i] = row;
            }
            row_weights[y] = row;
            row_cdf[y] = static_cast<float>((y + 1) * width);
        }
    }
    *total_weight = total;
    return yrc::Ok();
}

}  // extern "C"
