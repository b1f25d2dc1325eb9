// Launch interface of the wavefront render kernels (render_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "render_types.hpp"
#include "yrcuda.h"

namespace yrc {

// Per-batch device state shared by generate / film / active-list kernels.
struct BatchArgs {
    int32_t* active;                         // active pixel indices
    const unsigned long long* active_count;  // entries in `active`
    unsigned long long* active_count_next;   // rebuilt list size
    const int32_t* batch;                    // sample attempts per active pixel in this batch
    yrc_film_pixel* film;                    // device film
};

struct FilmArgs {
    int32_t* attempts_left;   // per pixel: passes this pixel may still take
    unsigned long long* bad_samples;
    unsigned long long* converged;
    int32_t adaptive;
    int32_t min_spp;
    float relative_error;
    float absolute_error;
    float confidence;
};

// Host launchers (grid sizes are multiples of the SM count; every kernel
// reads its work count from device memory, so the sequence is graph-safe).
void LaunchGenerate(const DevScene& sc, const PathState& ps, const Queues& q, const BatchArgs& b,
                    const CacheArgs& cache, int64_t capacity, int sm_count, cudaStream_t st);
void LaunchResetCounters(const Queues& q, cudaStream_t st);
void LaunchAdvanceQueue(const Queues& q, cudaStream_t st);
void LaunchShade(const DevScene& sc, const PathState& ps, const Queues& q, const CacheArgs& cache, int depth,
                 int64_t capacity, int sm_count, cudaStream_t st);
// LaunchShade in two parts: the texture stage and the sort of the extend
// queue by shading class, then the shade kernel of every class.
void LaunchShadeSort(const DevScene& sc, const PathState& ps, const Queues& q, int depth, int64_t capacity,
                     int sm_count, cudaStream_t st);
void LaunchShadeClasses(const DevScene& sc, const PathState& ps, const Queues& q, const CacheArgs& cache, int depth,
                        int64_t capacity, int sm_count, cudaStream_t st);
// One job of a pooled shade launch: its scene, path state, queues at this
// bounce (sorted by LaunchShadeSort), cache arguments and bounce.
struct ShadeJob {
    DevScene sc;
    PathState ps;
    Queues q;
    CacheArgs cache;
    int32_t depth;
};
// The shade kernel of every class, each launch over the class's entries of
// all `njobs` jobs (a device array); `capacity` bounds their sum.
void LaunchPooledShade(const ShadeJob* jobs, int njobs, int64_t capacity, int sm_count, cudaStream_t st);
// Subsurface: close the probes traced by LaunchRenderProbe (exit point,
// Sp / pdf, NEE at the exit, continuation).
// Scenes with cut-out (alpha) materials: the extend stage's skip loop over
// cut-out hits, and the exact per-thread shadow-visibility loop, over the
// whole shadow queue or (`list`) over the entries the single-pass shadow
// kernel left to it (q.shadow_overflow, counted in kCtrShadowOverflow).
void LaunchAlphaExtend(const DevScene& sc, const PathState& ps, const Queues& q, int depth, int64_t capacity,
                       int sm_count, int* error, cudaStream_t st);
void LaunchShadowExact(const DevScene& sc, const Queues& q, float4* transmittance, unsigned long long* occluded_count,
                       int64_t capacity, int sm_count, int* error, cudaStream_t st, const int32_t* list = nullptr);
void LaunchSubsurfaceExit(const DevScene& sc, const PathState& ps, const Queues& q, int depth, int64_t capacity,
                          int sm_count, cudaStream_t st);
// Radiance cache: add cached radiance to the paths that ended at the cache;
// build the training records of the training paths.
void LaunchCacheResolve(const PathState& ps, const CacheArgs& cache, int64_t capacity, int sm_count,
                        cudaStream_t st);
void LaunchCacheTargets(const PathState& ps, const CacheArgs& cache, int sm_count, cudaStream_t st);
// Coated (layered) vertices deferred by the shade stage: their emissive next
// events and the analytic / environment samples after the first shadow stage
// (LaunchLayeredNee, which also empties the shadow queue for the second
// stage), their analytic / environment results and continuation after the
// second (LaunchLayeredContinue). `transmittance` is null in scenes whose
// shadow stage is the any-hit kernel.
void LaunchLayeredNee(const DevScene& sc, const PathState& ps, const Queues& q, const float4* transmittance,
                      int depth, int64_t capacity, int sm_count, cudaStream_t st);
void LaunchLayeredContinue(const DevScene& sc, const PathState& ps, const Queues& q, const float4* transmittance,
                           int depth, int64_t capacity, int sm_count, cudaStream_t st);
void LaunchNeeResolve(const PathState& ps, const Queues& q, const float4* transmittance, int64_t capacity,
                      int sm_count, cudaStream_t st);
void LaunchFilm(const DevScene& sc, const PathState& ps, const BatchArgs& b, const FilmArgs& f, int64_t pixels,
                int sm_count, cudaStream_t st);
void LaunchActivePixels(const DevScene& sc, const BatchArgs& b, const FilmArgs& f, int64_t pixels, int sm_count,
                        cudaStream_t st);
// dst[0..n) = value.
void LaunchFillInt32(int32_t* dst, int64_t n, int32_t value, int sm_count, cudaStream_t st);
// Sums the film's per-pixel sample counts into *out (zeroed by the caller).
void LaunchSumSamples(const yrc_film_pixel* film, int64_t pixels, unsigned long long* out, int sm_count,
                      cudaStream_t st);
void LaunchFinishActive(unsigned long long* active_count, unsigned long long* active_count_next, int32_t* batch,
                        int32_t max_batch, int64_t capacity, cudaStream_t st);

}  // namespace yrc
