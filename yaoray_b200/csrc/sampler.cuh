// Device sampler: the reference's Sampler (src/sampling/sampler.cpp) with
// its semantic sample dimensions (include/yaoray/sampling/sampler.hpp:12-23),
// the PCG32 Rng (include/yaoray/core/rng.hpp:15-48) and SeedForPixelSample.
// Everything here is integer arithmetic plus an exact int->float scale, so the
// device values are bit-identical to the CPU reference.
#pragma once

#include <cstdint>

#include "yrc_math_host.hpp"

namespace yrc {

// SampleDimension values.
enum SampleDim : uint32_t {
    kDimPixel = 0,
    kDimDirectLightSelect = 2,
    kDimDirectLightSurface = 3,
    kDimBsdf = 5,
    kDimRussianRoulette = 7,
    kDimBssrdfReflect = 8,
    kDimBssrdfAxis = 9,
    kDimBssrdfDisk = 10,
    kDimBssrdfExitBsdf = 12,
    kDimAnalyticLightSelect = 14,
};
constexpr uint32_t kBounceDimStride = 16;

// RenderSamplerKind values.
enum SamplerKind : int32_t { kIndependent = 0, kStratified = 1, kOwenSobol = 2, kZSobol = 3 };

constexpr uint64_t kDefaultSeed = 0x9E3779B97F4A7C15ull;

// SplitMix64 finaliser (sampler.cpp Mix64).
YRC_HD uint64_t Mix64(uint64_t v) {
    v += 0x9E3779B97F4A7C15ull;
    v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ull;
    v = (v ^ (v >> 27)) * 0x94D049BB133111EBull;
    return v ^ (v >> 31);
}

YRC_HD uint32_t Mix32(uint32_t v) {
    v ^= v >> 16;
    v *= 0x7FEB352Du;
    v ^= v >> 15;
    v *= 0x846CA68Bu;
    return v ^ (v >> 16);
}

YRC_HD uint32_t Hash32(uint64_t seed, uint32_t dim, int lane) {
    const uint64_t m = Mix64(seed ^ (static_cast<uint64_t>(dim) * 0xD1B54A32D192ED03ull) ^
                             (static_cast<uint64_t>(static_cast<uint32_t>(lane)) * 0x94D049BB133111EBull));
    return Mix32(static_cast<uint32_t>(m) ^ static_cast<uint32_t>(m >> 32));
}

YRC_HD float UnitFloat(uint32_t v) { return static_cast<float>(v >> 8) * (1.0f / 16777216.0f); }

YRC_HD uint32_t ReverseBits32(uint32_t v) {
#if defined(__CUDA_ARCH__)
    return __brev(v);
#else
    v = ((v & 0x55555555u) << 1) | ((v >> 1) & 0x55555555u);
    v = ((v & 0x33333333u) << 2) | ((v >> 2) & 0x33333333u);
    v = ((v & 0x0F0F0F0Fu) << 4) | ((v >> 4) & 0x0F0F0F0Fu);
    v = ((v & 0x00FF00FFu) << 8) | ((v >> 8) & 0x00FF00FFu);
    return (v << 16) | (v >> 16);
#endif
}

// Sobol axis 0 is the bit reversal of the index; axis 1 XORs the direction
// numbers v_0 = 2^31, v_k = v_{k-1} ^ (v_{k-1} >> 1) for each set index bit.
YRC_HD uint32_t SobolAxis(uint32_t index, int axis) {
    if (axis == 0) return ReverseBits32(index);
    uint32_t value = 0, dir = 0x80000000u;
    while (index) {
        if (index & 1u) value ^= dir;
        index >>= 1;
        dir ^= dir >> 1;
    }
    return value;
}

// Laine-Karras nested-uniform scrambling on the bit-reversed value.
YRC_HD uint32_t OwenScramble(uint32_t v, uint32_t seed) {
    v = ReverseBits32(v);
    v += seed;
    v ^= v * 0x6C50B47Cu;
    v ^= v * 0xB82F1E52u;
    v ^= v * 0xC7AFE638u;
    v ^= v * 0x8D22F6E6u;
    return ReverseBits32(v);
}

YRC_HD uint32_t SpreadBits16(uint32_t v) {
    v &= 0x0000FFFFu;
    v = (v | (v << 8)) & 0x00FF00FFu;
    v = (v | (v << 4)) & 0x0F0F0F0Fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

// Per (pixel, sample) sampler state (Sampler's pixel constructor,
// sampler.cpp:138-166).
struct PixelSampler {
    uint64_t scene_seed;
    uint64_t pixel_seed;
    uint32_t sobol_index;
    int32_t sample_index;
    int32_t spp;
    int32_t kind;

    YRC_HD void Init(int32_t k, uint64_t seed, int x, int y, int sample, int samples_per_pixel) {
        kind = k;
        scene_seed = seed;
        pixel_seed = Mix64(seed ^ (static_cast<uint64_t>(static_cast<uint32_t>(x)) << 32) ^
                           static_cast<uint64_t>(static_cast<uint32_t>(y)));
        sample_index = sample;
        spp = samples_per_pixel < 1 ? 1 : samples_per_pixel;
        if (kind == kZSobol) {
            uint32_t c = 1, bits = 0;
            while (c < static_cast<uint32_t>(spp)) {
                c <<= 1;
                ++bits;
            }
            sobol_index = ((SpreadBits16(static_cast<uint32_t>(x)) | (SpreadBits16(static_cast<uint32_t>(y)) << 1))
                           << bits) |
                          static_cast<uint32_t>(sample);
        } else {
            sobol_index = static_cast<uint32_t>(sample);
        }
    }

    // AbsoluteDimension: every dimension but Pixel advances 16 per bounce.
    YRC_HD static uint32_t Abs(uint32_t dim, int bounce) {
        return dim == kDimPixel ? dim : dim + static_cast<uint32_t>(bounce < 0 ? 0 : bounce) * kBounceDimStride;
    }

    YRC_HD float At1D(uint32_t dim, int lane) const {
        if (kind == kOwenSobol) return UnitFloat(OwenScramble(SobolAxis(sobol_index, 0), Hash32(pixel_seed ^ kDefaultSeed, dim, lane)));
        if (kind == kZSobol) return UnitFloat(OwenScramble(SobolAxis(sobol_index, 0), Hash32(scene_seed, dim, lane)));
        return UnitFloat(Hash32(pixel_seed ^ static_cast<uint64_t>(static_cast<int64_t>(sample_index)), dim, lane));
    }

    YRC_HD void At2D(uint32_t dim, int lane, float& ox, float& oy) const {
        if (dim == kDimPixel && spp == 1) {
            ox = 0.5f;
            oy = 0.5f;
            return;
        }
        if (kind == kStratified) {
            const int count = dim == kDimPixel ? spp : 1;
            const int index = dim == kDimPixel ? sample_index : lane;
            const int columns = static_cast<int>(ceilf(sqrtf(static_cast<float>(count))));
            const int rows = (count + columns - 1) / columns;
            const int ci = index < 0 ? 0 : (index > count - 1 ? count - 1 : index);
            const float hi = 0.99999994f;  // nextafter(1, 0)
            float fx = YRC_DIV(YRC_ADD(static_cast<float>(ci % columns), At1D(dim, lane)), static_cast<float>(columns));
            float fy = YRC_DIV(YRC_ADD(static_cast<float>(ci / columns), At1D(dim + 1, lane)), static_cast<float>(rows));
            ox = fx < 0.0f ? 0.0f : (hi < fx ? hi : fx);
            oy = fy < 0.0f ? 0.0f : (hi < fy ? hi : fy);
            return;
        }
        if (kind == kOwenSobol || kind == kZSobol) {
            const uint64_t seed = kind == kOwenSobol ? pixel_seed : scene_seed;
            ox = UnitFloat(OwenScramble(SobolAxis(sobol_index, 0), Hash32(seed, dim, lane)));
            oy = UnitFloat(OwenScramble(SobolAxis(sobol_index, 1), Hash32(seed, dim + 1, lane)));
            return;
        }
        ox = At1D(dim, lane);
        oy = At1D(dim + 1, lane);
    }

    YRC_HD float Sample1D(uint32_t dim, int bounce, int lane = 0) const { return At1D(Abs(dim, bounce), lane); }
    YRC_HD void Sample2D(uint32_t dim, int bounce, float& x, float& y, int lane = 0) const {
        At2D(Abs(dim, bounce), lane, x, y);
    }
};

// SeedForPixelSample (sampler.cpp:304-310).
YRC_HD uint64_t SeedForPixelSample(uint64_t seed, int x, int y, int sample) {
    uint64_t v = Mix64(seed);
    v ^= Mix64(static_cast<uint64_t>(static_cast<int64_t>(x)) + 0xA24BAED4963EE407ull);
    v ^= Mix64(static_cast<uint64_t>(static_cast<int64_t>(y)) + 0x9FB21C651E98DF25ull);
    v ^= Mix64(static_cast<uint64_t>(static_cast<int64_t>(sample)) + 0xC2B2AE3D27D4EB4Full);
    return Mix64(v);
}

// PCG32 with the XSH-RR output (O'Neill 2014) as seeded by Rng(seed).
struct Pcg32 {
    uint64_t state;
    uint64_t inc;

    YRC_HD uint32_t Next() {
        const uint64_t old = state;
        state = old * 6364136223846793005ull + inc;
        const uint32_t xs = static_cast<uint32_t>(((old >> 18u) ^ old) >> 27u);
        const uint32_t rot = static_cast<uint32_t>(old >> 59u);
        return (xs >> rot) | (xs << ((0u - rot) & 31u));
    }
    YRC_HD void Seed(uint64_t seed) {
        state = 0u;
        inc = (seed << 1u) | 1u;
        Next();
        state += seed;
        Next();
    }
    YRC_HD float NextFloat() { return static_cast<float>(Next() >> 8) * (1.0f / 16777216.0f); }
};

}  // namespace yrc
