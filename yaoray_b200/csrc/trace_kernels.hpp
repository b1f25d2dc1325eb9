// Launch interface of the traversal kernels (trace_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "device_layout.cuh"
#include "yrcuda.h"

namespace yrc {

constexpr int kTraceBlock = 128;    // threads per block
constexpr int kShortStack = 12;     // stack entries per thread kept in shared memory
constexpr int kTraceShapes = 7;     // launch shapes the autotuner may choose from
constexpr int kMaxTraceStack = 256; // deepest traversal stack any kernel supports

// Status bits a kernel may set in the accelerator's device error word.
constexpr int kTraceErrorStackOverflow = 1;

struct TraceArgs {
    AccelParams accel;
    const float4* rays;  // 2 x float4 per ray (yrc_ray)
    int64_t count;
    yrc_hit* hits;            // closest-hit output
    int32_t* instances;       // optional per-ray instance output
    uint8_t* occluded;        // any-hit output
    uint32_t* node_tests;     // optional stats outputs
    uint32_t* triangle_tests;
    uint32_t* sphere_tests;
    unsigned long long* counter;  // ray work counter, zeroed before the launch
    int* error;                   // device error word
};

constexpr int kProbeMaxHits = YRC_PROBE_MAX_HITS;  // BvhProbeHits::MaxHits
constexpr int kProbeMaxIterations = 4096;           // IntersectBvhProbe's iteration cap

struct ProbeArgs {
    AccelParams accel;
    const float4* rays;
    const yrc_probe_target* targets;
    int64_t count;
    yrc_hit* hits;       // kProbeMaxHits per ray
    int32_t* instances;  // optional, kProbeMaxHits per ray
    int32_t* counts;
    uint8_t* exhausted;
    int* error;
};

// shape: index of the launch shape (block size / refill interval / register
// budget) for the flat closest- and any-hit kernels, 0 = default.
cudaError_t LaunchTrace(const TraceArgs& args, bool any_hit, bool stats, int shape, cudaStream_t stream,
                        int sm_count);
cudaError_t LaunchProbe(const ProbeArgs& args, cudaStream_t stream, int sm_count);

}  // namespace yrc
