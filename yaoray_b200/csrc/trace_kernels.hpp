// Launch interface of the traversal kernels (trace_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "device_layout.cuh"
#include "yrcuda.h"

namespace yrc {

constexpr int kTraceBlock = 128;    // threads per block
constexpr int kShortStack = 12;     // stack entries per thread kept in shared memory
constexpr int kTraceShapes = 17;     // launch shapes the autotuner may choose from
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
    const unsigned long long* count_ptr;  // optional: ray count read on the device (count = capacity)
    const int32_t* out_index;             // optional: any-hit output slot per ray
    unsigned long long* occluded_count;   // optional: any-hit rays that hit something (RenderStats)
    const uint32_t* order;                // optional: ray index per traversal slot (OrderRays)
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
struct DevMaterial;

struct ShadowArgs {
    AccelParams accel;
    const float4* rays;                   // shadow queue (2 x float4 per ray)
    const unsigned long long* count_ptr;  // entries in the queue (device)
    int64_t capacity;                     // grid sizing bound
    const int32_t* out_index;             // slot per ray
    float4* transmittance;                // per slot
    const int32_t* tri_prim;
    const int32_t* prim_material;
    const int32_t* sphere_material;
    const DevMaterial* materials;
    const uint8_t* tri_clear;             // per flat triangle: passes light (1) or occludes (0)
    const uint8_t* sphere_clear;          // per sphere
    unsigned long long* counter;          // ray work counter, zeroed before the launch
    unsigned long long* occluded_count;   // shadow rays found not visible (RenderStats::occluded_shadow_rays)
    int32_t* overflow;                    // queue indices left to the exact loop (more than 16 clear surfaces)
    unsigned long long* overflow_count;   // entries in `overflow`, zeroed before the launch
    int* error;
    int32_t leaf_batch;                   // > 0: leaf tests batched across the warp (TraceKernel's kLeafBatch)
};

// The leaf batch of a launch shape (TraceKernel's kLeafBatch; shapes 7-16).
constexpr int LeafBatchOfShape(int shape) {
    return shape == 7 ? 4 : (shape == 9 || shape == 12) ? 16 : (shape == 8 || shape == 10 || shape == 11 || shape >= 13) ? 8 : 0;
}

// Subsurface probes of the render path: rays in the yrc_ray layout (t_min,
// t_max = probe length), targets (mesh primitive, instance, sphere, path),
// per probe a selection sample in selection[2 * k].w; outputs the selected
// target hit and the number of target hits (<= kProbeMaxHits).
struct RenderProbeArgs {
    AccelParams accel;
    const float4* rays;
    const int4* targets;
    const float4* selection;
    const unsigned long long* count_ptr;
    int64_t capacity;
    float4* hit;
    int32_t* hits;
    int* error;
};

cudaError_t LaunchRenderProbe(const RenderProbeArgs& args, cudaStream_t stream, int sm_count);

// Pooled traversal: one persistent launch over the ray queues of several
// render jobs. Each job's rays keep their own queue, accelerator and
// outputs (its TraceArgs / ShadowArgs entry in a device-resident table,
// with the ray count read from count_ptr on the device); the launch's lanes
// take rays from one work counter over the jobs' queues laid end to end, so
// that no job's tail leaves the GPU idle while another's rays wait.
constexpr int kMaxPoolJobs = 128;

struct TracePool {
    const TraceArgs* jobs;          // njobs entries (count_ptr required; counter unused)
    int32_t njobs;
    int64_t capacity;               // bound on the total rays, for grid sizing
    unsigned long long* counter;    // work counter, zeroed before the launch
};

struct ShadowPool {
    const ShadowArgs* jobs;         // njobs entries (counter unused)
    int32_t njobs;
    int64_t capacity;
    unsigned long long* counter;
};

// Every job of a pool must share the BVH kind (flat or two-level) and
// depth class (stack limit <= 64 or not) given here.
cudaError_t LaunchPooledTrace(const TracePool& pool, bool any_hit, bool two_level, bool deep, cudaStream_t stream,
                              int sm_count);
cudaError_t LaunchPooledShadowTransmittance(const ShadowPool& pool, bool two_level, bool deep, cudaStream_t stream,
                                            int sm_count);

// Accessors of accelerator internals used by the render stages (accel.cu).
AccelParams AccelParamsOf(const yrc_accel* a);
int TraceShapeOf(const yrc_accel* a, int any_hit);
int* AccelErrorWord(yrc_accel* a);
yrc_status CheckDeviceError(yrc_accel* a);

cudaError_t LaunchShadowTransmittance(const ShadowArgs& args, cudaStream_t stream, int sm_count);

cudaError_t LaunchTrace(const TraceArgs& args, bool any_hit, bool stats, int shape, cudaStream_t stream,
                        int sm_count);
cudaError_t LaunchProbe(const ProbeArgs& args, cudaStream_t stream, int sm_count);

// Ray reordering ahead of a traversal launch (ray_order.cu).
constexpr int kRayOrderOff = 0;
constexpr int kRayOrderDirection = 1;  // key: origin and direction
constexpr int kRayOrderTwoPoint = 2;   // key: origin and a point along the ray
constexpr int kRayOrderMinBits = 8;
constexpr int kRayOrderMaxBits = 24;

struct RayOrderScratch {
    uint32_t* keys;       // one per ray
    uint32_t* order;      // one per ray: the permutation
    uint32_t* hist;       // 2^bits bin counters
    uint32_t* tile_sums;  // RayOrderTiles(bits)
};

// Key bits for `count` rays (`requested` > 0 is clamped to the supported range).
int RayOrderBits(int64_t count, int requested);
int64_t RayOrderTiles(int bits);
// Writes scratch.order[0..count) = ray indices sorted by their key bin.
// `length` is the two-point key's distance as a fraction of the root box
// diagonal. count must be below 2^32.
cudaError_t OrderRays(const float4* rays, int64_t count, const AccelParams& accel, int mode, int bits, float length,
                      const RayOrderScratch& scratch, cudaStream_t stream, int sm_count);
// Loads the code of the two statistics traversal kernels (closest and any
// hit) that a BVH of this kind and stack limit uses, so that their first
// launch under lazy module loading does not take device memory.
cudaError_t PreloadStatsKernels(bool two_level, int stack_limit);

}  // namespace yrc
