// Device-resident scene textures (texture.cu): RenderTexture images with
// their mip chains, built on the device, and the EWA tap weights.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "texture.cuh"
#include "yrcuda.h"

namespace yrc {

struct TextureSet {
    DevTexture* textures = nullptr;  // device array, one per scene texture
    const float* ewa_weights = nullptr;
    int32_t count = 0;
    int64_t bytes = 0;
    std::vector<void*> blocks;  // device allocations owned by the set
    void Release();
};

// BuildTextureSamplingCaches (src/shading/texture.cpp:266-295) on the
// device: identical images (same size, wrap modes and texels) share one
// pyramid; each mip level is the box average of the level above it
// (BuildTextureMipChain, texture.cpp:242-264). Synchronous on `stream`.
yrc_status UploadTextures(const yrc_texture* textures, int32_t count, cudaStream_t stream, TextureSet& out);

}  // namespace yrc
