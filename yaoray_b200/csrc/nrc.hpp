// Internal interface of the neural radiance cache (nrc.cu) for the render
// stages; the public C ABI is declared in yrcuda.h.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "yrcuda.h"

namespace yrc {
namespace nrc {

// rgb[i] (float4, w unused) = cache(queries[i]) for n queries of 16 floats;
// with n_ptr, the count is min(*n_ptr, n) read on the device (graph-safe).
// `averaged` queries the moving average of the parameters.
yrc_status Infer(yrc_nrc* cache, const float* queries, int64_t n, const unsigned long long* n_ptr, float* rgb,
                 cudaStream_t stream, bool averaged);
// One optimiser step on n (query, target float4) pairs (n_ptr as above).
yrc_status TrainStep(yrc_nrc* cache, const float* queries, const float* targets, int64_t n,
                     const unsigned long long* n_ptr, cudaStream_t stream);

}  // namespace nrc
}  // namespace yrc
