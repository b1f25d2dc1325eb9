// Closest-hit / any-hit / probe traversal kernels for the flat and two-level
// BVH.
//
// Semantics are those of IntersectBvh (src/accel/bvh_traversal.cpp:253-345),
// IntersectTwoLevelBvh (src/accel/two_level_bvh.cpp:365-481) and
// IntersectAccelerationProbe (src/accel/acceleration.cpp:63-108), including
// the exact visiting order: depth-first, both children box-tested against the
// current nearest t, the nearer child (left on a tie) taken next and the other
// pushed, popped entries culled when their entry t exceeds the nearest t.
// Following the same order with the same IEEE operations makes the hit IDs and
// t values bit-identical to the CPU reference, not merely close.
//
// Execution model (sm_100a):
//  * persistent grid sized from the occupancy calculator (a multiple of the SM
//    count); each lane owns one ray and fetches a new one as soon as its ray
//    finishes (warp-aggregated atomicAdd on a global ray counter), checked
//    every kSteps node visits so lanes with short rays do not idle;
//  * traversal stack: the first kShortStack entries of each thread live in
//    shared memory laid out [depth][thread] (bank-conflict free), deeper
//    entries in a per-thread local array; the host picks a kernel whose
//    total depth covers the BVH's longest root-to-leaf path;
//  * nodes and leaf records are read with 128-bit read-only loads.
#include "device_layout.cuh"
#include "render_types.hpp"
#include "trace_kernels.hpp"
#include "traversal.cuh"

#include <cuda_runtime.h>

namespace yrc {
namespace {

template <bool kAny, bool kStats>
__device__ __forceinline__ void WriteResult(const TraceArgs& args, int64_t ray, const Traversal& s) {
    if (kAny) {
        args.occluded[args.out_index ? args.out_index[ray] : ray] = s.best.hit ? 1 : 0;
        if (args.occluded_count && s.best.hit) CountLanes(args.occluded_count);
    } else {
        reinterpret_cast<float4*>(args.hits)[ray] =
            make_float4(s.best.t, __int_as_float(s.best.hit ? s.best.id : -1), s.best.u, s.best.v);
        if (args.instances) args.instances[ray] = s.best.hit ? s.best_inst : -1;
    }
    if (kStats) {
        if (args.node_tests) args.node_tests[ray] = s.nodes;
        if (args.triangle_tests) args.triangle_tests[ray] = s.tris;
        if (args.sphere_tests) args.sphere_tests[ray] = s.spheres;
    }
}

// kLeafBatch > 0: a lane that reaches a leaf waits (its ray keeps its place
// in its own visiting order) until at least kLeafBatch lanes of the warp
// are at leaves or no lane is at an interior node, so that the leaf tests,
// the longest branch of a step, run for many lanes at once instead of for
// the one or two lanes that reached a leaf at each step. Interior steps go
// on meanwhile; every ray's visiting order, and so every hit and count,
// is unchanged.
template <bool kAny, bool kStats, bool kTwo, int kTotal, int kBlock, int kStepsPerRefill, int kMinBlocks,
          bool kWide = false, int kLeafBatch = 0>
__global__ void __launch_bounds__(kBlock, kMinBlocks) TraceKernel(TraceArgs args) {
    __shared__ int2 s_stack[kShortStack * kBlock];
    int2* col = s_stack + threadIdx.x;
    StackStore<kTotal, kBlock> st;
    Traversal s;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt_mask = (1u << lane) - 1u;
    int64_t ray = -1;
    bool alive = false;
    bool exhausted = false;
    const unsigned long long count =
        args.count_ptr ? *args.count_ptr : static_cast<unsigned long long>(args.count);

    for (;;) {
        const unsigned need = __ballot_sync(kFull, !alive && !exhausted);
        if (need) {
            unsigned long long base = 0;
            const int leader = __ffs(need) - 1;
            if (static_cast<int>(lane) == leader) {
                base = atomicAdd(args.counter, static_cast<unsigned long long>(__popc(need)));
            }
            base = __shfl_sync(kFull, base, leader);
            if (!alive && !exhausted) {
                const unsigned long long idx = base + __popc(need & lt_mask);
                if (idx >= count) {
                    exhausted = true;
                } else {
                    ray = args.order ? static_cast<int64_t>(__ldg(args.order + idx)) : static_cast<int64_t>(idx);
                    const float4 b = Ld(args.rays + 2 * ray + 1);
                    const float tmin = Ld(args.rays + 2 * ray).w;
                    alive = Begin(args.accel, args.rays, ray, tmin, b.w, s);
                    if (kWide && alive) s.cur = args.accel.wide_root;
                    if (!alive) WriteResult<kAny, kStats>(args, ray, s);
                }
            }
        }
        if (!__any_sync(kFull, alive)) {
            if (__all_sync(kFull, exhausted)) break;
            continue;
        }
        if constexpr (kLeafBatch > 0) {
            // Uniform loop: every lane runs every iteration, so the votes
            // see the whole warp.
#pragma unroll 1
            for (int k = 0; k < kStepsPerRefill; ++k) {
                const unsigned at_leaf = __ballot_sync(kFull, alive && s.cur < 0);
                const unsigned at_node = __ballot_sync(kFull, alive && s.cur >= 0);
                if (!(at_leaf | at_node)) break;
                const bool leaves = at_node == 0u || __popc(at_leaf) >= kLeafBatch;
                if (alive && (s.cur >= 0 || leaves)) {
                    alive = Step<kAny, kStats, kTwo, StackStore<kTotal, kBlock>, false, kWide>(args.accel, args.rays,
                                                                                               ray, s, st, col,
                                                                                               args.error);
                    if (!alive) WriteResult<kAny, kStats>(args, ray, s);
                }
            }
        } else {
#pragma unroll 1
            for (int k = 0; k < kStepsPerRefill && alive; ++k) {
                alive = Step<kAny, kStats, kTwo, StackStore<kTotal, kBlock>, false, kWide>(args.accel, args.rays, ray,
                                                                                           s, st, col, args.error);
                if (!alive) WriteResult<kAny, kStats>(args, ray, s);
            }
        }
    }
}

// TraceKernel over the ray queues of several jobs at once (TracePool): the
// same traversal and refill, with the accelerator, rays and outputs of the
// job each lane's ray came from.
template <bool kAny, bool kTwo, int kTotal, int kBlock, int kStepsPerRefill, int kMinBlocks, int kLeafBatch>
__global__ void __launch_bounds__(kBlock, kMinBlocks) PooledTraceKernel(TracePool pool) {
    __shared__ int2 s_stack[kShortStack * kBlock];
    __shared__ unsigned long long s_ends[kMaxPoolJobs];
    const unsigned long long count = LoadPoolEnds(pool.jobs, pool.njobs, s_ends);
    int2* col = s_stack + threadIdx.x;
    StackStore<kTotal, kBlock> st;
    Traversal s;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt_mask = (1u << lane) - 1u;
    const TraceArgs* job = pool.jobs;
    AccelParams acc = job->accel;
    const float4* rays = job->rays;
    int64_t ray = -1;
    bool alive = false;
    bool exhausted = false;

    for (;;) {
        const unsigned need = __ballot_sync(kFull, !alive && !exhausted);
        if (need) {
            unsigned long long base = 0;
            const int leader = __ffs(need) - 1;
            if (static_cast<int>(lane) == leader) {
                base = atomicAdd(pool.counter, static_cast<unsigned long long>(__popc(need)));
            }
            base = __shfl_sync(kFull, base, leader);
            if (!alive && !exhausted) {
                const unsigned long long idx = base + __popc(need & lt_mask);
                if (idx >= count) {
                    exhausted = true;
                } else {
                    const int j = PoolJobOf(s_ends, pool.njobs, idx);
                    job = pool.jobs + j;
                    acc = job->accel;
                    rays = job->rays;
                    ray = static_cast<int64_t>(idx - (j ? s_ends[j - 1] : 0ull));
                    const float4 b = Ld(rays + 2 * ray + 1);
                    const float tmin = Ld(rays + 2 * ray).w;
                    alive = Begin(acc, rays, ray, tmin, b.w, s);
                    if (!alive) WriteResult<kAny, false>(*job, ray, s);
                }
            }
        }
        if (!__any_sync(kFull, alive)) {
            if (__all_sync(kFull, exhausted)) break;
            continue;
        }
#pragma unroll 1
        for (int k = 0; k < kStepsPerRefill; ++k) {
            const unsigned at_leaf = __ballot_sync(kFull, alive && s.cur < 0);
            const unsigned at_node = __ballot_sync(kFull, alive && s.cur >= 0);
            if (!(at_leaf | at_node)) break;
            const bool leaves = at_node == 0u || __popc(at_leaf) >= kLeafBatch;
            if (alive && (s.cur >= 0 || leaves)) {
                alive = Step<kAny, false, kTwo, StackStore<kTotal, kBlock>>(acc, rays, ray, s, st, col, job->error);
                if (!alive) WriteResult<kAny, false>(*job, ray, s);
            }
        }
    }
}

// IntersectAccelerationProbe: one thread per probe ray iterating closest-hit
// queries with an advancing cursor; target hits are appended in t order.
template <bool kTwo, int kTotal>
__global__ void __launch_bounds__(kTraceBlock) ProbeKernel(ProbeArgs args) {
    __shared__ int2 s_stack[kShortStack * kTraceBlock];
    int2* col = s_stack + threadIdx.x;
    StackStore<kTotal> st;
    Traversal s;
    for (int64_t ray = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; ray < args.count;
         ray += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int4 target = __ldg(reinterpret_cast<const int4*>(args.targets) + ray);
        const float t_min = Ld(args.rays + 2 * ray).w;
        const float t_max = Ld(args.rays + 2 * ray + 1).w;
        int32_t count = 0;
        uint8_t exhausted = 0;
        float cursor = t_min;
        for (int iter = 0; iter < kProbeMaxIterations; ++iter) {
            bool alive = Begin(args.accel, args.rays, ray, cursor, t_max, s);
            while (alive) alive = Step<false, false, kTwo>(args.accel, args.rays, ray, s, st, col, args.error);
            if (!s.best.hit) break;
            const bool inst_ok = !kTwo || target.y < 0 || s.best_inst == target.y;
            const bool is_target = (target.x >= 0 && s.best.id >= 0 && s.best.prim == target.x && inst_ok) ||
                                   (target.z >= 0 && s.best.id == -2 - target.z);
            if (is_target) {
                if (count < kProbeMaxHits) {
                    const int64_t o = ray * kProbeMaxHits + count;
                    reinterpret_cast<float4*>(args.hits)[o] =
                        make_float4(s.best.t, __int_as_float(s.best.id), s.best.u, s.best.v);
                    if (args.instances) args.instances[o] = s.best_inst;
                    ++count;
                } else {
                    exhausted = 1;
                    break;
                }
            }
            float next = __fadd_rn(s.best.t, __fmul_rn(1.0e-4f, __fadd_rn(1.0f, fabsf(s.best.t))));
            if (!(next > cursor)) next = __fadd_rn(cursor, 1.0e-4f);
            cursor = next;
            if (cursor >= t_max) break;
        }
        args.counts[ray] = count;
        args.exhausted[ray] = exhausted;
    }
}

// SampleBssrdfProbe's probe (src/integrators/bssrdf_probe.cpp:51-66) for the
// render path: IntersectAccelerationProbe's loop (closest-hit queries with an
// advancing cursor, target hits kept in t order, at most kProbeMaxHits)
// run twice per probe, first to count the target hits, then to return the
// one the selection sample picks (floor(u * count), clamped), so no per-probe
// hit list is stored.
template <bool kTwo, int kTotal>
__global__ void __launch_bounds__(kTraceBlock) RenderProbeKernel(RenderProbeArgs args) {
    __shared__ int2 s_stack[kShortStack * kTraceBlock];
    int2* col = s_stack + threadIdx.x;
    StackStore<kTotal> st;
    Traversal s;
    const int64_t n = static_cast<int64_t>(*args.count_ptr);
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int4 target = args.targets[k];
        const float t_min = Ld(args.rays + 2 * k).w;
        const float t_max = Ld(args.rays + 2 * k + 1).w;
        // pass == 0 counts; pass == 1 stops at the selected target hit
        int32_t count = 0;
        int32_t selected = -1;
        float4 chosen = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        for (int pass = 0; pass < 2; ++pass) {
            if (pass == 1) {
                if (count == 0) break;
                const float u = args.selection[2 * k].w;
                selected = min(max(static_cast<int32_t>(u * static_cast<float>(count)), 0), count - 1);
            }
            int32_t seen = 0;
            float cursor = t_min;
            for (int iter = 0; iter < kProbeMaxIterations; ++iter) {
                bool alive = Begin(args.accel, args.rays, k, cursor, t_max, s);
                while (alive) alive = Step<false, false, kTwo>(args.accel, args.rays, k, s, st, col, args.error);
                if (!s.best.hit) break;
                const bool inst_ok = !kTwo || target.y < 0 || s.best_inst == target.y;
                const bool is_target = (target.x >= 0 && s.best.id >= 0 && s.best.prim == target.x && inst_ok) ||
                                       (target.z >= 0 && s.best.id == -2 - target.z);
                if (is_target) {
                    if (seen >= kProbeMaxHits) break;
                    if (pass == 1 && seen == selected) {
                        chosen = make_float4(s.best.t, __int_as_float(s.best.id), s.best.u, s.best.v);
                        break;
                    }
                    ++seen;
                }
                float next = __fadd_rn(s.best.t, __fmul_rn(1.0e-4f, __fadd_rn(1.0f, fabsf(s.best.t))));
                if (!(next > cursor)) next = __fadd_rn(cursor, 1.0e-4f);
                cursor = next;
                if (cursor >= t_max) break;
            }
            if (pass == 0) count = seen;
        }
        args.hits[k] = count;
        args.hit[k] = chosen;
    }
}

// TraceShadowVisibility (src/integrators/path_direct_lighting.cpp:23-113)
// for every shadow ray in one traversal. The reference runs up to 16
// closest-hit queries along the segment, each from just past the previous
// hit: an opaque surface occludes, a Dielectric toggles a Beer-Lambert
// medium, a ThinDielectric multiplies by its clamped reflectance. Here one
// any-hit traversal over the whole segment skips the surfaces that pass light
// and keeps the nearest 16 of them (ClearHits); it stops at the first opaque
// surface, which gives 0 whatever lies before it (the loop reaches it or
// turns black, or gives up at 16 queries — all occluded). With no surface at
// all the ray is fully visible. Otherwise the reference's loop is replayed
// over the kept list in t order: each query returns the first kept surface
// beyond the query's origin plus t_min (1e-5), t measured from that origin,
// with the same bias, remaining-distance and 16-query rules. When more than
// 16 clear surfaces were seen and a query would need one beyond the kept
// list, the ray's queue index goes to an overflow list that the exact loop
// (ShadowExactKernel, re-spawning each query) traces afterwards, and this
// kernel writes nothing for it. What differs from re-tracing is rounding: t
// is the traversal's t from the ray origin less the distance already
// advanced, not a new intersection from the re-spawned origin. Persistent
// warps with per-lane refill, like TraceKernel.
//
// kPooled: the launch serves the shadow queues of several jobs (ShadowPool);
// each lane works with the job of the ray it holds.
// kLeafBatch: leaf tests batched across the warp, as in TraceKernel.
template <bool kTwo, int kTotal, bool kPooled = false, int kLeafBatch = 0>
__global__ void __launch_bounds__(kTraceBlock, kShadowBlocksPerSm)
    ShadowTransmittanceKernel(const __grid_constant__ ShadowArgs args, const __grid_constant__ ShadowPool pool) {
    __shared__ int2 s_stack[kShadowShortStack * kTraceBlock];
    __shared__ float s_clear_t[kClearHits * kTraceBlock];
    __shared__ int32_t s_clear_id[kClearHits * kTraceBlock];
    __shared__ unsigned long long s_ends[kPooled ? kMaxPoolJobs : 1];
    const ShadowArgs* A = kPooled ? pool.jobs : &args;
    AccelParams acc = A->accel;
    const unsigned long long count = kPooled ? LoadPoolEnds(pool.jobs, pool.njobs, s_ends) : *args.count_ptr;
    unsigned long long* const counter = kPooled ? pool.counter : args.counter;
    int2* col = s_stack + threadIdx.x;
    StackStore<kTotal, kTraceBlock, kShadowShortStack> st;
    Traversal s;
    s.best.hit = false;  // defined before the first Begin, for the compiler's flow analysis
    s.saw = false;
    ClearHits clear{s_clear_t + threadIdx.x, s_clear_id + threadIdx.x, 0, false};
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt_mask = (1u << lane) - 1u;
    int64_t ray = -1;
    bool alive = false;
    bool exhausted = false;

    // The reference loop over the kept clear surfaces; returns the RGB
    // transmittance, w = 1 when visible, all 0 when occluded.
    auto replay = [&]() -> float4 {
        const float4 ra = Ld(A->rays + 2 * ray);
        const float4 rb = Ld(A->rays + 2 * ray + 1);
        float o[3] = {ra.x, ra.y, ra.z};
        const float d[3] = {rb.x, rb.y, rb.z};
        float remaining = rb.w;
        float T[3] = {1.0f, 1.0f, 1.0f}, mc[3] = {1.0f, 1.0f, 1.0f}, md = 1.0f;
        bool medium = false;
        float qmin = ra.w;   // t_min of the current query
        float off = 0.0f;    // distance from the ray origin to the current query's origin
        const float4 occluded = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        auto black = [&]() { return fmaxf(T[0], fmaxf(T[1], T[2])) <= 1.0e-6f; };
        auto beer = [&](float dist) {
            if (dist <= 0.0f || md <= 0.0f) return;
            const float inv = 1.0f / md;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float c = fminf(fmaxf(mc[k], 1.0e-6f), 1.0f);
                T[k] = T[k] * expf(logf(c) * dist * inv);
            }
        };
        int k = 0;
        for (int query = 0; query < kClearHits; ++query) {
            const bool finite = isfinite(remaining);
            float t = 0.0f;
            int32_t id = 0;
            bool found = false;
            for (; k < clear.n; ++k) {
                t = __fsub_rn(clear.t[k * kTraceBlock], off);
                if (t > qmin && t <= remaining) {
                    id = clear.id[k * kTraceBlock];
                    found = true;
                    ++k;
                    break;
                }
            }
            if (!found) {
                // A surface beyond the kept ones would be this query's
                // answer: the exact loop traces this ray instead.
                if (clear.dropped) return make_float4(0.0f, 0.0f, 0.0f, -1.0f);
                if (medium) {
                    if (!finite) return occluded;
                    beer(remaining);
                }
                return black() ? occluded : make_float4(T[0], T[1], T[2], 1.0f);
            }
            if (medium) {
                beer(t);
                if (black()) return occluded;
            }
            const int32_t material = id >= 0 ? A->prim_material[A->tri_prim[id]] : A->sphere_material[-2 - id];
            if (material < 0 || (A->materials[material].kind != 2 && A->materials[material].kind != 3)) {
                return occluded;
            }
            const DevMaterial& m = A->materials[material];
            float hp[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) hp[c] = __fadd_rn(o[c], __fmul_rn(d[c], t));
            if (m.kind == 3) {
#pragma unroll
                for (int c = 0; c < 3; ++c) T[c] = T[c] * fminf(fmaxf(m.reflectance[c], 0.0f), 1.0f);
                if (black()) return occluded;
            } else if (medium) {
                medium = false;
                mc[0] = mc[1] = mc[2] = 1.0f;
                md = 1.0f;
            } else {
                medium = true;
                mc[0] = m.absorption_color[0];
                mc[1] = m.absorption_color[1];
                mc[2] = m.absorption_color[2];
                md = m.absorption_distance;
            }
            const float bias = fmaxf(1.0e-4f, fmaxf(fabsf(hp[0]), fmaxf(fabsf(hp[1]), fabsf(hp[2]))) * 1.0e-5f);
            if (finite) {
                remaining = __fsub_rn(remaining, __fadd_rn(t, bias));
                if (remaining <= 0.0f) return black() ? occluded : make_float4(T[0], T[1], T[2], 1.0f);
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) o[c] = __fadd_rn(hp[c], __fmul_rn(d[c], bias));
            off = __fadd_rn(off, __fadd_rn(t, bias));
            qmin = 1.0e-5f;
        }
        return occluded;  // the reference gives up after 16 queries
    };
    auto finish = [&]() {
        const int32_t slot = A->out_index[ray];
        float4 tr;
        if (s.best.hit) {
            tr = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        } else if (!s.saw) {
            tr = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
        } else {
            tr = replay();
            if (tr.w < 0.0f) {
                const unsigned long long o = atomicAdd(A->overflow_count, 1ull);
                A->overflow[o] = static_cast<int32_t>(ray);
                return;
            }
        }
        A->transmittance[slot] = tr;
        if (tr.w == 0.0f) CountLanes(A->occluded_count);
    };
    for (;;) {
        const unsigned need = __ballot_sync(kFull, !alive && !exhausted);
        if (need) {
            unsigned long long base = 0;
            const int leader = __ffs(need) - 1;
            if (static_cast<int>(lane) == leader) {
                base = atomicAdd(counter, static_cast<unsigned long long>(__popc(need)));
            }
            base = __shfl_sync(kFull, base, leader);
            if (!alive && !exhausted) {
                const unsigned long long idx = base + __popc(need & lt_mask);
                if (idx >= count) {
                    exhausted = true;
                } else {
                    ray = static_cast<int64_t>(idx);
                    if (kPooled) {
                        const int j = PoolJobOf(s_ends, pool.njobs, idx);
                        A = pool.jobs + j;
                        acc = A->accel;
                        ray -= static_cast<int64_t>(j ? s_ends[j - 1] : 0ull);
                    }
                    const float4 b = Ld(A->rays + 2 * ray + 1);
                    const float tmin = Ld(A->rays + 2 * ray).w;
                    clear.n = 0;
                    clear.dropped = false;
                    alive = Begin(acc, A->rays, ray, tmin, b.w, s);
                    if (!alive) finish();
                }
            }
        }
        if (!__any_sync(kFull, alive)) {
            if (__all_sync(kFull, exhausted)) break;
            continue;
        }
        if constexpr (kLeafBatch > 0) {
#pragma unroll 1
            for (int k = 0; k < 8; ++k) {
                const unsigned at_leaf = __ballot_sync(kFull, alive && s.cur < 0);
                const unsigned at_node = __ballot_sync(kFull, alive && s.cur >= 0);
                if (!(at_leaf | at_node)) break;
                const bool leaves = at_node == 0u || __popc(at_leaf) >= kLeafBatch;
                if (alive && (s.cur >= 0 || leaves)) {
                    alive = Step<true, false, kTwo, StackStore<kTotal, kTraceBlock, kShadowShortStack>, true>(
                        acc, A->rays, ray, s, st, col, A->error, A->tri_clear, A->sphere_clear, &clear);
                    if (!alive) finish();
                }
            }
        } else {
#pragma unroll 1
            for (int k = 0; k < 8 && alive; ++k) {
                alive = Step<true, false, kTwo, StackStore<kTotal, kTraceBlock, kShadowShortStack>, true>(
                    acc, A->rays, ray, s, st, col, A->error, A->tri_clear, A->sphere_clear, &clear);
                if (!alive) finish();
            }
        }
    }
}

template <typename Kernel>
cudaError_t PersistentGrid(Kernel kernel, int block, int64_t count, int sm_count, int64_t& blocks) {
    int per_sm = 0;
    const cudaError_t err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0);
    if (err != cudaSuccess) return err;
    if (per_sm < 1) per_sm = 1;
    blocks = static_cast<int64_t>(per_sm) * sm_count;
    const int64_t needed = (count + block - 1) / block;
    if (blocks > needed) blocks = needed < 1 ? 1 : needed;
    return cudaSuccess;
}

template <bool kAny, bool kStats, bool kTwo, int kTotal, int kBlock, int kStepsPerRefill, int kMinBlocks,
          bool kWide = false, int kLeafBatch = 0>
cudaError_t LaunchOne(const TraceArgs& args, cudaStream_t stream, int sm_count) {
    auto kernel = TraceKernel<kAny, kStats, kTwo, kTotal, kBlock, kStepsPerRefill, kMinBlocks, kWide, kLeafBatch>;
    int64_t blocks = 0;
    const cudaError_t err = PersistentGrid(kernel, kBlock, args.count, sm_count, blocks);
    if (err != cudaSuccess) return err;
    kernel<<<static_cast<unsigned>(blocks), kBlock, 0, stream>>>(args);
    return cudaGetLastError();
}

// The tunable launch shapes (block size, node visits between ray refills,
// minimum resident blocks for the register budget). Index 0 is the default;
// the autotuner times the rest on the actual accelerator.
template <bool kAny, bool kStats, bool kTwo, int kTotal, bool kWide = false>
cudaError_t LaunchShape(const TraceArgs& args, int shape, cudaStream_t stream, int sm_count) {
    switch (kStats ? 0 : shape) {
        case 1: return LaunchOne<kAny, kStats, kTwo, kTotal, 128, 4, 1, kWide>(args, stream, sm_count);
        case 2: return LaunchOne<kAny, kStats, kTwo, kTotal, 128, 16, 1, kWide>(args, stream, sm_count);
        case 3: return LaunchOne<kAny, kStats, kTwo, kTotal, 128, 8, 12, kWide>(args, stream, sm_count);
        case 4: return LaunchOne<kAny, kStats, kTwo, kTotal, 64, 8, 1, kWide>(args, stream, sm_count);
        case 5: return LaunchOne<kAny, kStats, kTwo, kTotal, 256, 8, 1, kWide>(args, stream, sm_count);
        case 6: return LaunchOne<kAny, kStats, kTwo, kTotal, 64, 8, 24, kWide>(args, stream, sm_count);
        case 7: return LaunchOne<kAny, kStats, kTwo, kTotal, 128, 8, 1, kWide, 4>(args, stream, sm_count);
        case 8: return LaunchOne<kAny, kStats, kTwo, kTotal, 128, 8, 1, kWide, 8>(args, stream, sm_count);
        case 9: return LaunchOne<kAny, kStats, kTwo, kTotal, 128, 8, 1, kWide, 16>(args, stream, sm_count);
        case 10: return LaunchOne<kAny, kStats, kTwo, kTotal, 128, 8, 12, kWide, 8>(args, stream, sm_count);
        case 11: return LaunchOne<kAny, kStats, kTwo, kTotal, 256, 8, 1, kWide, 8>(args, stream, sm_count);
        case 12: return LaunchOne<kAny, kStats, kTwo, kTotal, 128, 8, 8, kWide, 16>(args, stream, sm_count);
        case 13: return LaunchOne<kAny, kStats, kTwo, kTotal, 128, 16, 1, kWide, 8>(args, stream, sm_count);
        case 14: return LaunchOne<kAny, kStats, kTwo, kTotal, 128, 32, 1, kWide, 8>(args, stream, sm_count);
        case 15: return LaunchOne<kAny, kStats, kTwo, kTotal, 128, 8, 9, kWide, 8>(args, stream, sm_count);
        case 16: return LaunchOne<kAny, kStats, kTwo, kTotal, 128, 8, 10, kWide, 8>(args, stream, sm_count);
        default: return LaunchOne<kAny, kStats, kTwo, kTotal, 128, 8, 1, kWide>(args, stream, sm_count);
    }
}

template <bool kAny, bool kStats, bool kTwo>
cudaError_t LaunchDepth(const TraceArgs& args, int shape, cudaStream_t stream, int sm_count) {
    if (args.accel.stack_limit <= 64) return LaunchShape<kAny, kStats, kTwo, 64>(args, shape, stream, sm_count);
    return LaunchShape<kAny, kStats, kTwo, kMaxTraceStack>(args, 0, stream, sm_count);
}

// The four-wide traversal (flat, triangle-only, no statistics).
template <bool kAny>
cudaError_t LaunchWide(const TraceArgs& args, int shape, cudaStream_t stream, int sm_count) {
    if (args.accel.wide_stack_limit <= 64) {
        return LaunchShape<kAny, false, false, 64, true>(args, shape, stream, sm_count);
    }
    return LaunchOne<kAny, false, false, kMaxTraceStack, 128, 8, 1, true>(args, stream, sm_count);
}

template <bool kTwo, int kTotal>
cudaError_t LaunchProbeOne(const ProbeArgs& args, cudaStream_t stream, int sm_count) {
    auto kernel = ProbeKernel<kTwo, kTotal>;
    int64_t blocks = 0;
    const cudaError_t err = PersistentGrid(kernel, kTraceBlock, args.count, sm_count, blocks);
    if (err != cudaSuccess) return err;
    kernel<<<static_cast<unsigned>(blocks), kTraceBlock, 0, stream>>>(args);
    return cudaGetLastError();
}

template <bool kTwo, int kTotal, bool kPooled = false>
cudaError_t LaunchShadowOne(const ShadowArgs& args, const ShadowPool& pool, cudaStream_t stream, int sm_count) {
    // A pooled launch batches leaf tests by 8; a single one as its shape asks
    // (leaf batch 4 runs as 8).
    auto kernel = kPooled                  ? ShadowTransmittanceKernel<kTwo, kTotal, kPooled, 8>
                  : args.leaf_batch >= 16 ? ShadowTransmittanceKernel<kTwo, kTotal, kPooled, 16>
                  : args.leaf_batch > 0   ? ShadowTransmittanceKernel<kTwo, kTotal, kPooled, 8>
                                          : ShadowTransmittanceKernel<kTwo, kTotal, kPooled, 0>;
    int64_t blocks = 0;
    const cudaError_t err =
        PersistentGrid(kernel, kTraceBlock, kPooled ? pool.capacity : args.capacity, sm_count, blocks);
    if (err != cudaSuccess) return err;
    kernel<<<static_cast<unsigned>(blocks), kTraceBlock, 0, stream>>>(args, pool);
    return cudaGetLastError();
}

template <bool kAny, bool kTwo, int kTotal>
cudaError_t LaunchPooledOne(const TracePool& pool, cudaStream_t stream, int sm_count) {
    constexpr int kBlock = 128;
    auto kernel = PooledTraceKernel<kAny, kTwo, kTotal, kBlock, 8, 1, 8>;
    int64_t blocks = 0;
    const cudaError_t err = PersistentGrid(kernel, kBlock, pool.capacity, sm_count, blocks);
    if (err != cudaSuccess) return err;
    kernel<<<static_cast<unsigned>(blocks), kBlock, 0, stream>>>(pool);
    return cudaGetLastError();
}

}  // namespace

template <bool kTwo, int kTotal>
cudaError_t LaunchRenderProbeOne(const RenderProbeArgs& args, cudaStream_t stream, int sm_count) {
    auto kernel = RenderProbeKernel<kTwo, kTotal>;
    int64_t blocks = 0;
    const cudaError_t err = PersistentGrid(kernel, kTraceBlock, args.capacity, sm_count, blocks);
    if (err != cudaSuccess) return err;
    kernel<<<static_cast<unsigned>(blocks), kTraceBlock, 0, stream>>>(args);
    return cudaGetLastError();
}

cudaError_t LaunchRenderProbe(const RenderProbeArgs& args, cudaStream_t stream, int sm_count) {
    const bool two = args.accel.two_level != 0;
    const bool deep = args.accel.stack_limit > 64;
    if (two) return deep ? LaunchRenderProbeOne<true, kMaxTraceStack>(args, stream, sm_count)
                         : LaunchRenderProbeOne<true, 64>(args, stream, sm_count);
    return deep ? LaunchRenderProbeOne<false, kMaxTraceStack>(args, stream, sm_count)
                : LaunchRenderProbeOne<false, 64>(args, stream, sm_count);
}

cudaError_t LaunchShadowTransmittance(const ShadowArgs& args, cudaStream_t stream, int sm_count) {
    const bool two = args.accel.two_level != 0;
    const bool deep = args.accel.stack_limit > 64;
    const ShadowPool none{};
    if (two) return deep ? LaunchShadowOne<true, kMaxTraceStack>(args, none, stream, sm_count)
                         : LaunchShadowOne<true, 64>(args, none, stream, sm_count);
    return deep ? LaunchShadowOne<false, kMaxTraceStack>(args, none, stream, sm_count)
                : LaunchShadowOne<false, 64>(args, none, stream, sm_count);
}

cudaError_t LaunchPooledShadowTransmittance(const ShadowPool& pool, bool two, bool deep, cudaStream_t stream,
                                            int sm_count) {
    if (pool.njobs <= 0) return cudaSuccess;
    if (pool.njobs > kMaxPoolJobs) return cudaErrorInvalidValue;
    const ShadowArgs none{};
    if (two) return deep ? LaunchShadowOne<true, kMaxTraceStack, true>(none, pool, stream, sm_count)
                         : LaunchShadowOne<true, 64, true>(none, pool, stream, sm_count);
    return deep ? LaunchShadowOne<false, kMaxTraceStack, true>(none, pool, stream, sm_count)
                : LaunchShadowOne<false, 64, true>(none, pool, stream, sm_count);
}

cudaError_t LaunchPooledTrace(const TracePool& pool, bool any, bool two, bool deep, cudaStream_t stream,
                              int sm_count) {
    if (pool.njobs <= 0) return cudaSuccess;
    if (pool.njobs > kMaxPoolJobs) return cudaErrorInvalidValue;
    if (any) {
        if (two) return deep ? LaunchPooledOne<true, true, kMaxTraceStack>(pool, stream, sm_count)
                             : LaunchPooledOne<true, true, 64>(pool, stream, sm_count);
        return deep ? LaunchPooledOne<true, false, kMaxTraceStack>(pool, stream, sm_count)
                    : LaunchPooledOne<true, false, 64>(pool, stream, sm_count);
    }
    if (two) return deep ? LaunchPooledOne<false, true, kMaxTraceStack>(pool, stream, sm_count)
                         : LaunchPooledOne<false, true, 64>(pool, stream, sm_count);
    return deep ? LaunchPooledOne<false, false, kMaxTraceStack>(pool, stream, sm_count)
                : LaunchPooledOne<false, false, 64>(pool, stream, sm_count);
}

cudaError_t LaunchTrace(const TraceArgs& args, bool any_hit, bool stats, int shape, cudaStream_t stream,
                        int sm_count) {
    const bool two = args.accel.two_level != 0;
    if (!two && !stats && args.accel.wide) {
        return any_hit ? LaunchWide<true>(args, shape, stream, sm_count) : LaunchWide<false>(args, shape, stream, sm_count);
    }
    if (any_hit) {
        if (two) return stats ? LaunchDepth<true, true, true>(args, shape, stream, sm_count)
                              : LaunchDepth<true, false, true>(args, shape, stream, sm_count);
        return stats ? LaunchDepth<true, true, false>(args, shape, stream, sm_count)
                     : LaunchDepth<true, false, false>(args, shape, stream, sm_count);
    }
    if (two) return stats ? LaunchDepth<false, true, true>(args, shape, stream, sm_count)
                          : LaunchDepth<false, false, true>(args, shape, stream, sm_count);
    return stats ? LaunchDepth<false, true, false>(args, shape, stream, sm_count)
                 : LaunchDepth<false, false, false>(args, shape, stream, sm_count);
}

template <bool kTwo, int kTotal>
cudaError_t PreloadStatsPair() {
    cudaFuncAttributes attr;
    cudaError_t err = cudaFuncGetAttributes(&attr, TraceKernel<false, true, kTwo, kTotal, 128, 8, 1>);
    if (err == cudaSuccess) err = cudaFuncGetAttributes(&attr, TraceKernel<true, true, kTwo, kTotal, 128, 8, 1>);
    return err;
}

cudaError_t PreloadStatsKernels(bool two_level, int stack_limit) {
    // The kernels LaunchDepth picks for statistics (shape 0 whatever the
    // tuned shape, the depth class of the BVH).
    const bool deep = stack_limit > 64;
    if (two_level) return deep ? PreloadStatsPair<true, kMaxTraceStack>() : PreloadStatsPair<true, 64>();
    return deep ? PreloadStatsPair<false, kMaxTraceStack>() : PreloadStatsPair<false, 64>();
}

cudaError_t LaunchProbe(const ProbeArgs& args, cudaStream_t stream, int sm_count) {
    const bool two = args.accel.two_level != 0;
    const bool deep = args.accel.stack_limit > 64;
    if (two) return deep ? LaunchProbeOne<true, kMaxTraceStack>(args, stream, sm_count)
                         : LaunchProbeOne<true, 64>(args, stream, sm_count);
    return deep ? LaunchProbeOne<false, kMaxTraceStack>(args, stream, sm_count)
                : LaunchProbeOne<false, 64>(args, stream, sm_count);
}

}  // namespace yrc
