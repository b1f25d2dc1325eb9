// Device-resident measured BRDFs (measured.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "measured.cuh"
#include "yrcuda.h"

namespace yrc {

struct MeasuredSet {
    DevMeasuredBrdf* brdfs = nullptr;  // device array, one per measured BRDF
    int32_t count = 0;
    int64_t bytes = 0;
    std::vector<void*> blocks;
    void Release();
};

// Checks the tensors (isotropic only, as the reference's loader), builds the
// five warps on the host and uploads them. Synchronous.
yrc_status UploadMeasured(const yrc_measured_brdf* brdfs, int32_t count, MeasuredSet& out);

}  // namespace yrc
