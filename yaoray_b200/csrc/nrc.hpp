// Internal interface of the neural radiance cache (nrc.cu) for the render
// stages; the public C ABI is declared in yrcuda.h.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "yrcuda.h"

namespace yrc {
namespace nrc {

// rgb[i] (float4, w unused) = cache(queries[i]) for n queries of 16 floats.
yrc_status Infer(yrc_nrc* cache, const float* queries, int64_t n, float* rgb, cudaStream_t stream);
// One optimiser step on n (query, target float4) pairs.
yrc_status TrainStep(yrc_nrc* cache, const float* queries, const float* targets, int64_t n, cudaStream_t stream);

}  // namespace nrc
}  // namespace yrc
