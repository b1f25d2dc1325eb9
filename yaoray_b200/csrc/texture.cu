// Scene textures on the device: upload with de-duplication, mip chains built
// by a box-filter kernel per level, the EWA weight table, and C-ABI entry
// points that evaluate lookups for callers that compare them with the
// reference's (SampleTexture4, BuildTextureMipChain).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "texture.hpp"
#include "yrc_internal.hpp"

namespace yrc {
namespace {

// BuildTextureMipChain's inner loop (src/shading/texture.cpp:253-260): each
// texel is ((a + b) + c) + d over the 2x2 block of the finer level, addressed
// with the texture's wrap modes, times 0.25.
__global__ void MipLevelKernel(DevTexLevel src, float4* dst, int32_t dw, int32_t dh, int32_t ws, int32_t wt) {
    const int64_t n = static_cast<int64_t>(dw) * dh;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(i % dw), y = static_cast<int>(i / dw);
        float4 f = Add4(TexelAt(src, x * 2, y * 2, ws, wt), TexelAt(src, x * 2 + 1, y * 2, ws, wt));
        f = Add4(f, TexelAt(src, x * 2, y * 2 + 1, ws, wt));
        f = Add4(f, TexelAt(src, x * 2 + 1, y * 2 + 1, ws, wt));
        dst[i] = Scale4(f, 0.25f);
    }
}

__global__ void SampleEvalKernel(const DevTexture* tex, const float2* uvs, const float4* footprints, int64_t n,
                                 const float* weights, float4* out) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const float2 uv = uvs[i];
    TexFootprint f{0.0f, 0.0f, 0.0f, 0.0f};
    if (footprints) {
        const float4 q = footprints[i];
        f = TexFootprint{q.x, q.y, q.z, q.w};
    }
    out[i] = SampleTexture4(*tex, uv.x, uv.y, f, weights);
}

// EwaWeights (texture.cpp:140-152), evaluated with the host C library's expf
// exactly as the reference evaluates it.
std::vector<float> EwaWeightsHost() {
    std::vector<float> w(kEwaWeightCount);
    const float alpha = 2.0f;
    const float edge = std::exp(-alpha);
    for (int i = 0; i < kEwaWeightCount; ++i) {
        const float r2 = static_cast<float>(i) / static_cast<float>(kEwaWeightCount - 1);
        w[static_cast<size_t>(i)] = std::exp(-alpha * r2) - edge;
    }
    return w;
}

// Mip chain sizes (BuildTextureMipChain, texture.cpp:242-251): halve with
// round-up until 1x1.
std::vector<int2> ChainDims(int32_t w, int32_t h) {
    std::vector<int2> dims{make_int2(w, h)};
    while (w > 1 || h > 1) {
        w = std::max(1, (w + 1) / 2);
        h = std::max(1, (h + 1) / 2);
        dims.push_back(make_int2(w, h));
    }
    return dims;
}

bool HasData(const yrc_texture& t) { return t.width > 0 && t.height > 0 && t.texels; }

// TextureStorageHash (texture.cpp:64-88): FNV-1a over size, wrap modes and
// texel bits; equal hashes are confirmed byte for byte before sharing.
uint64_t StorageHash(const yrc_texture& t) {
    uint64_t hash = 14695981039346656037ull;
    auto mix = [&](uint32_t v) {
        for (int b = 0; b < 4; ++b) {
            hash ^= static_cast<uint8_t>(v >> (b * 8));
            hash *= 1099511628211ull;
        }
    };
    mix(static_cast<uint32_t>(t.width));
    mix(static_cast<uint32_t>(t.height));
    mix(static_cast<uint32_t>(t.wrap_s));
    mix(static_cast<uint32_t>(t.wrap_t));
    const size_t words = static_cast<size_t>(t.width) * static_cast<size_t>(t.height) * 4;
    const uint32_t* p = reinterpret_cast<const uint32_t*>(t.texels);
    for (size_t i = 0; i < words; ++i) mix(p[i]);
    return hash;
}

bool SameStorage(const yrc_texture& a, const yrc_texture& b) {
    return a.width == b.width && a.height == b.height && a.wrap_s == b.wrap_s && a.wrap_t == b.wrap_t &&
           std::memcmp(a.texels, b.texels, sizeof(float) * 4 * static_cast<size_t>(a.width) * a.height) == 0;
}

template <typename T>
T* DevAlloc(TextureSet& s, size_t count, cudaError_t& err) {
    if (err != cudaSuccess) return nullptr;
    void* p = nullptr;
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    err = cudaMalloc(&p, bytes);
    if (err != cudaSuccess) return nullptr;
    s.blocks.push_back(p);
    s.bytes += static_cast<int64_t>(bytes);
    return static_cast<T*>(p);
}

}  // namespace

void TextureSet::Release() {
    for (void* p : blocks) cudaFree(p);
    blocks.clear();
    textures = nullptr;
    ewa_weights = nullptr;
    count = 0;
    bytes = 0;
}

yrc_status UploadTextures(const yrc_texture* textures, int32_t count, cudaStream_t stream, TextureSet& out) {
    out.Release();
    if (count < 0 || (count > 0 && !textures)) return Fail(YRC_ERR_INVALID_ARGUMENT, "invalid texture array");
    for (int32_t i = 0; i < count; ++i) {
        const yrc_texture& t = textures[i];
        if (t.filter < kTexNearest || t.filter > kTexEwa || t.wrap_s < kWrapRepeat || t.wrap_s > kWrapMirror ||
            t.wrap_t < kWrapRepeat || t.wrap_t > kWrapMirror) {
            return Fail(YRC_ERR_INVALID_ARGUMENT, "texture " + std::to_string(i) + ": unknown filter or wrap mode");
        }
        if (HasData(t) && static_cast<int64_t>(t.width) * t.height > (int64_t{1} << 31)) {
            return Fail(YRC_ERR_INVALID_ARGUMENT, "texture " + std::to_string(i) + ": more than 2^31 texels");
        }
    }
    // Distinct pyramids: source texture index per pyramid, pyramid per texture.
    std::vector<int32_t> owner, pyramid_of(static_cast<size_t>(count), -1);
    std::unordered_map<uint64_t, std::vector<int32_t>> by_hash;
    for (int32_t i = 0; i < count; ++i) {
        if (!HasData(textures[i])) continue;
        auto& bucket = by_hash[StorageHash(textures[i])];
        for (int32_t p : bucket) {
            if (SameStorage(textures[owner[static_cast<size_t>(p)]], textures[i])) {
                pyramid_of[static_cast<size_t>(i)] = p;
                break;
            }
        }
        if (pyramid_of[static_cast<size_t>(i)] < 0) {
            pyramid_of[static_cast<size_t>(i)] = static_cast<int32_t>(owner.size());
            bucket.push_back(static_cast<int32_t>(owner.size()));
            owner.push_back(i);
        }
    }
    // Level table and texel offsets of every pyramid.
    std::vector<std::vector<int2>> dims(owner.size());
    std::vector<int32_t> level_base(owner.size());
    std::vector<int64_t> level_offset;
    int64_t texels = 0;
    for (size_t p = 0; p < owner.size(); ++p) {
        const yrc_texture& t = textures[owner[p]];
        dims[p] = ChainDims(t.width, t.height);
        level_base[p] = static_cast<int32_t>(level_offset.size());
        for (const int2& d : dims[p]) {
            level_offset.push_back(texels);
            texels += static_cast<int64_t>(d.x) * d.y;
        }
    }
    cudaError_t err = cudaSuccess;
    float4* store = DevAlloc<float4>(out, static_cast<size_t>(texels), err);
    DevTexLevel* levels = DevAlloc<DevTexLevel>(out, level_offset.size(), err);
    DevTexture* dev_textures = DevAlloc<DevTexture>(out, static_cast<size_t>(count), err);
    float* weights = DevAlloc<float>(out, kEwaWeightCount, err);
    if (err != cudaSuccess) {
        out.Release();
        return Fail(YRC_ERR_OUT_OF_MEMORY, std::string("texture upload: ") + cudaGetErrorString(err));
    }
    std::vector<DevTexLevel> host_levels(level_offset.size());
    for (size_t p = 0; p < owner.size(); ++p) {
        for (size_t l = 0; l < dims[p].size(); ++l) {
            const size_t k = static_cast<size_t>(level_base[p]) + l;
            host_levels[k] = DevTexLevel{store + level_offset[k], dims[p][l].x, dims[p][l].y};
        }
    }
    std::vector<DevTexture> host_textures(static_cast<size_t>(count));
    for (int32_t i = 0; i < count; ++i) {
        const yrc_texture& t = textures[i];
        DevTexture& d = host_textures[static_cast<size_t>(i)];
        d = DevTexture{nullptr, t.width, t.height, 0, t.filter, t.wrap_s, t.wrap_t};
        const int32_t p = pyramid_of[static_cast<size_t>(i)];
        if (p >= 0) {
            d.levels = levels + level_base[static_cast<size_t>(p)];
            d.level_count = static_cast<int32_t>(dims[static_cast<size_t>(p)].size());
        }
    }
    const std::vector<float> w = EwaWeightsHost();
    err = cudaMemcpyAsync(weights, w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice, stream);
    if (err == cudaSuccess && !host_levels.empty()) {
        err = cudaMemcpyAsync(levels, host_levels.data(), sizeof(DevTexLevel) * host_levels.size(),
                              cudaMemcpyHostToDevice, stream);
    }
    if (err == cudaSuccess && count > 0) {
        err = cudaMemcpyAsync(dev_textures, host_textures.data(), sizeof(DevTexture) * host_textures.size(),
                              cudaMemcpyHostToDevice, stream);
    }
    for (size_t p = 0; p < owner.size() && err == cudaSuccess; ++p) {
        const yrc_texture& t = textures[owner[p]];
        const size_t base = static_cast<size_t>(level_base[p]);
        err = cudaMemcpyAsync(store + level_offset[base], t.texels,
                              sizeof(float4) * static_cast<size_t>(t.width) * t.height, cudaMemcpyHostToDevice,
                              stream);
        for (size_t l = 1; l < dims[p].size() && err == cudaSuccess; ++l) {
            const DevTexLevel& src = host_levels[base + l - 1];
            const int64_t n = static_cast<int64_t>(dims[p][l].x) * dims[p][l].y;
            const unsigned blocks = static_cast<unsigned>(std::min<int64_t>((n + 255) / 256, 4096));
            MipLevelKernel<<<blocks, 256, 0, stream>>>(src, store + level_offset[base + l], dims[p][l].x,
                                                       dims[p][l].y, t.wrap_s, t.wrap_t);
            err = cudaGetLastError();
        }
    }
    if (err == cudaSuccess) err = cudaStreamSynchronize(stream);
    if (err != cudaSuccess) {
        out.Release();
        return Fail(YRC_ERR_CUDA, std::string("texture upload: ") + cudaGetErrorString(err));
    }
    out.textures = dev_textures;
    out.ewa_weights = weights;
    out.count = count;
    return Ok();
}

}  // namespace yrc

extern "C" {

yrc_status yrc_texture_sample_eval(const yrc_texture* texture, const float* uvs, const float* footprints, int64_t n,
                                   float* out) {
    using namespace yrc;
    if (!texture || n < 0 || (n > 0 && (!uvs || !out))) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_texture_sample_eval: bad argument");
    }
    if (n == 0) return Ok();
    TextureSet set;
    yrc_status st = UploadTextures(texture, 1, nullptr, set);
    if (st != YRC_OK) return st;
    cudaError_t err = cudaSuccess;
    float2* d_uv = DevAlloc<float2>(set, static_cast<size_t>(n), err);
    float4* d_fp = footprints ? DevAlloc<float4>(set, static_cast<size_t>(n), err) : nullptr;
    float4* d_out = DevAlloc<float4>(set, static_cast<size_t>(n), err);
    if (err == cudaSuccess) err = cudaMemcpy(d_uv, uvs, sizeof(float2) * static_cast<size_t>(n), cudaMemcpyHostToDevice);
    if (err == cudaSuccess && d_fp) {
        err = cudaMemcpy(d_fp, footprints, sizeof(float4) * static_cast<size_t>(n), cudaMemcpyHostToDevice);
    }
    if (err == cudaSuccess) {
        SampleEvalKernel<<<static_cast<unsigned>((n + 255) / 256), 256>>>(set.textures, d_uv, d_fp, n,
                                                                          set.ewa_weights, d_out);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemcpy(out, d_out, sizeof(float4) * static_cast<size_t>(n), cudaMemcpyDeviceToHost);
    set.Release();
    if (err != cudaSuccess) return Fail(YRC_ERR_CUDA, std::string("yrc_texture_sample_eval: ") + cudaGetErrorString(err));
    return Ok();
}

yrc_status yrc_texture_mip_chain_eval(const yrc_texture* texture, float* texels, int64_t capacity, int32_t* level_dims,
                                      int32_t* level_count) {
    using namespace yrc;
    if (!texture || !level_count || capacity < 0 || (capacity > 0 && !texels)) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_texture_mip_chain_eval: bad argument");
    }
    *level_count = 0;
    if (!HasData(*texture)) return Ok();
    const std::vector<int2> dims = ChainDims(texture->width, texture->height);
    int64_t total = 0;
    for (const int2& d : dims) total += static_cast<int64_t>(d.x) * d.y;
    if (total > capacity || !level_dims) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_texture_mip_chain_eval: output holds " + std::to_string(capacity) +
                                                  " texels, the chain has " + std::to_string(total));
    }
    TextureSet set;
    yrc_status st = UploadTextures(texture, 1, nullptr, set);
    if (st != YRC_OK) return st;
    DevTexture host_tex;
    cudaError_t err = cudaMemcpy(&host_tex, set.textures, sizeof(DevTexture), cudaMemcpyDeviceToHost);
    std::vector<DevTexLevel> lv(dims.size());
    if (err == cudaSuccess) {
        err = cudaMemcpy(lv.data(), host_tex.levels, sizeof(DevTexLevel) * lv.size(), cudaMemcpyDeviceToHost);
    }
    int64_t at = 0;
    for (size_t l = 0; l < lv.size() && err == cudaSuccess; ++l) {
        const int64_t n = static_cast<int64_t>(lv[l].width) * lv[l].height;
        err = cudaMemcpy(texels + 4 * at, lv[l].texels, sizeof(float4) * static_cast<size_t>(n), cudaMemcpyDeviceToHost);
        level_dims[2 * l] = lv[l].width;
        level_dims[2 * l + 1] = lv[l].height;
        at += n;
    }
    set.Release();
    if (err != cudaSuccess) return Fail(YRC_ERR_CUDA, std::string("yrc_texture_mip_chain_eval: ") + cudaGetErrorString(err));
    *level_count = static_cast<int32_t>(dims.size());
    return Ok();
}

}  // extern "C"
