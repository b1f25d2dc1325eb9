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

#include <cuda_runtime.h>

namespace yrc {
namespace {

constexpr unsigned kFull = 0xffffffffu;

struct Traversal {
    RayPre r;        // current ray (world, or object space inside a BLAS)
    float tmin;
    Nearest best;    // world (flat) nearest
    Nearest local;   // BLAS-local nearest while inside an instance
    int32_t best_inst;
    int32_t cur;        // node pair (>= 0) or leaf (~first record)
    int32_t sp;
    int32_t level;      // 0: root level (flat BVH or TLAS), 1: inside a BLAS
    int32_t blas_base;  // stack pointer when the BLAS was entered
    int32_t tl_resume;  // TLAS record to resume after the BLAS, -1 = none
    int32_t cur_inst;   // instance being traversed
    uint32_t nodes, tris, spheres;  // BvhTraceStats
    float wo[3], wd[3];  // world-space ray, restored after a BLAS
    bool saw;            // filtered any-hit: a surface that passes light was skipped
};

__device__ __forceinline__ float4 Ld(const float4* p) { return __ldg(p); }

// Interior-node loads carry an L2 evict-last policy: the node pairs are read
// about twenty times per ray and the leaf records and ray streams a few
// times, so the tree should be what L2 keeps.
__device__ __forceinline__ unsigned long long NodePolicy() {
    unsigned long long pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ float4 LdNode(const float4* p, unsigned long long pol) {
    float4 v;
    asm volatile("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p), "l"(pol));
    return v;
}

// Warp-aggregated increment of a statistics counter by the calling lanes.
__device__ __forceinline__ void CountLanes(unsigned long long* counter) {
    const unsigned mask = __activemask();
    if ((threadIdx.x & 31u) == static_cast<unsigned>(__ffs(mask) - 1)) {
        atomicAdd(counter, static_cast<unsigned long long>(__popc(mask)));
    }
}

// Traversal stack of kTotal entries per thread: the first kShortStack in the
// block's shared memory (column `col`, stride kBlock), the rest local.
template <int kTotal, int kBlock = kTraceBlock, int kShort = kShortStack>
struct StackStore {
    static constexpr int kTotalEntries = kTotal;
    static constexpr int kLocal = kTotal > kShort ? kTotal - kShort : 1;
    int2 local[kLocal];

    __device__ __forceinline__ void Put(int2* col, int sp, int2 e) {
        if (sp < kShort) {
            col[sp * kBlock] = e;
        } else {
            local[sp - kShort] = e;
        }
    }
    __device__ __forceinline__ int2 Get(const int2* col, int sp) const {
        return sp < kShort ? col[sp * kBlock] : local[sp - kShort];
    }
};

__device__ __forceinline__ void RestoreWorldRay(Traversal& s) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        s.r.o[k] = s.wo[k];
        s.r.d[k] = s.wd[k];
    }
    Precompute(s.r);
}

// Begins a traversal of the ray (o, d) over [tmin, tmax]; returns false when
// the ray already finished at the root (empty BVH or root box missed).
__device__ __forceinline__ bool BeginRay(const AccelParams& a, const float o[3], const float d[3], float tmin,
                                         float tmax, Traversal& s) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        s.wo[k] = o[k];
        s.wd[k] = d[k];
    }
    RestoreWorldRay(s);
    s.tmin = tmin;
    s.best.t = tmax;
    s.best.id = -1;
    s.best.prim = -1;
    s.best.u = 0.0f;
    s.best.v = 0.0f;
    s.best.hit = false;
    s.best_inst = -1;
    s.sp = 0;
    s.level = 0;
    s.tl_resume = -1;
    s.nodes = s.tris = s.spheres = 0;
    s.saw = false;
    if (a.root_ref == kAbsentRef) return false;
    s.nodes = 1;
    float entry;
    if (!SlabTest(s.r, a.root_lo[0], a.root_lo[1], a.root_lo[2], a.root_hi[0], a.root_hi[1], a.root_hi[2], s.tmin,
                  s.best.t, entry)) {
        return false;
    }
    s.cur = a.root_ref;
    return true;
}

// Begin for ray i of a yrc_ray array.
__device__ __forceinline__ bool Begin(const AccelParams& a, const float4* rays, int64_t i, float tmin, float tmax,
                                      Traversal& s) {
    const float4 ra = Ld(rays + 2 * i);
    const float4 rb = Ld(rays + 2 * i + 1);
    const float o[3] = {ra.x, ra.y, ra.z};
    const float d[3] = {rb.x, rb.y, rb.z};
    return BeginRay(a, o, d, tmin, tmax, s);
}

// Pops the next live stack entry into s.cur (culled against the nearest t of
// the current level) and closes finished BLAS traversals. Returns false when
// the ray's traversal is complete.
template <bool kAny, bool kTwo, typename Stack>
__device__ __forceinline__ bool Pop(const float4* rays, int64_t ray, Traversal& s, Stack& st, const int2* col) {
    for (;;) {
        if (kTwo && s.level == 1 && s.sp == s.blas_base) {
            // IntersectTwoLevelBvh accepts the BLAS hit only if strictly nearer.
            if (s.local.hit && s.local.t < s.best.t) {
                s.best = s.local;
                s.best_inst = s.cur_inst;
            }
            s.level = 0;
            RestoreWorldRay(s);
            if (kAny && s.best.hit) return false;
            if (s.tl_resume >= 0) {
                s.cur = ~s.tl_resume;
                return true;
            }
            continue;
        }
        if (s.sp == 0) return false;
        --s.sp;
        const int2 e = st.Get(col, s.sp);
        const float limit = (kTwo && s.level == 1) ? s.local.t : s.best.t;
        if (__int_as_float(e.y) > limit) continue;
        s.cur = e.x;
        return true;
    }
}

// The clear surfaces (those that pass light) a filtered any-hit traversal
// skipped: the lane's kClearHits nearest as (t, surface id) pairs, ordered by
// t then id, in the block's shared memory laid out [entry][thread]. More than
// kClearHits of them never matter: the reference's shadow loop gives up after
// that many queries.
constexpr int kClearHits = 16;  // MaxTransparentShadowHits
// The shadow kernel keeps 11 stack entries in shared memory (the clear list
// takes the rest) so that 8 blocks of 128 threads fit an SM.
constexpr int kShadowShortStack = 11;
constexpr int kShadowBlocksPerSm = 8;

struct ClearHits {
    float* t;     // the lane's column, stride kTraceBlock
    int32_t* id;
    int n;        // entries held (<= kClearHits)
    bool dropped; // a farther clear surface did not fit

    __device__ __forceinline__ void Add(float tv, int32_t idv) {
        int j = n;  // slot the new entry would take; kClearHits = past the end
        while (j > 0) {
            const float tp = t[(j - 1) * kTraceBlock];
            const int32_t ip = id[(j - 1) * kTraceBlock];
            if (tp < tv || (tp == tv && ip < idv)) break;
            if (j < kClearHits) {
                t[j * kTraceBlock] = tp;
                id[j * kTraceBlock] = ip;
            } else {
                dropped = true;
            }
            --j;
        }
        if (j < kClearHits) {
            t[j * kTraceBlock] = tv;
            id[j * kTraceBlock] = idv;
        } else {
            dropped = true;
        }
        if (n < kClearHits) ++n;
    }
};

// One traversal step: an interior node (test both children) or a leaf (test
// its records). Returns false when the ray's traversal is complete.
//
// kFilter (any-hit only): candidates on surfaces flagged in `tri_clear` /
// `sphere_clear` are not accepted; the traversal records that it skipped one
// (s.saw), adds it to `clear` and goes on, so it ends at the first hit on any
// other surface.
// Compare-exchange of two (miss, entry, ref) candidates of a four-wide node:
// hits before misses, then nearer entry first.
__device__ __forceinline__ void OrderPair(bool& ma, float& ea, int32_t& ra, bool& mb, float& eb, int32_t& rb) {
    const bool swap = (mb < ma) || (mb == ma && eb < ea);
    if (swap) {
        const bool m = ma;
        const float e = ea;
        const int32_t r = ra;
        ma = mb, ea = eb, ra = rb;
        mb = m, eb = e, rb = r;
    }
}

// One step at a four-wide node: the four child boxes are slab-tested with
// the binary traversal's test; the nearest hit child is taken next and the
// others are pushed farthest first. Returns 1 when s.cur holds the next
// node, 0 when no child was hit, -1 on a stack overflow (traversal ends).
template <typename Stack>
__device__ __forceinline__ int WideStep(const AccelParams& a, Traversal& s, Stack& st, int2* col, int* error) {
    const float4* p = reinterpret_cast<const float4*>(a.wide + s.cur);
    const float4 lx = Ld(p), hx = Ld(p + 1), ly = Ld(p + 2), hy = Ld(p + 3), lz = Ld(p + 4), hz = Ld(p + 5);
    const int4 rf = __ldg(reinterpret_cast<const int4*>(p + 6));
    const float limit = s.best.t;
    bool m0 = true, m1 = true, m2 = true, m3 = true;
    float e0 = 0.0f, e1 = 0.0f, e2 = 0.0f, e3 = 0.0f;
    int32_t r0 = rf.x, r1 = rf.y, r2 = rf.z, r3 = rf.w;
    if (r0 != kAbsentRef) m0 = !SlabTest(s.r, lx.x, ly.x, lz.x, hx.x, hy.x, hz.x, s.tmin, limit, e0);
    if (r1 != kAbsentRef) m1 = !SlabTest(s.r, lx.y, ly.y, lz.y, hx.y, hy.y, hz.y, s.tmin, limit, e1);
    if (r2 != kAbsentRef) m2 = !SlabTest(s.r, lx.z, ly.z, lz.z, hx.z, hy.z, hz.z, s.tmin, limit, e2);
    if (r3 != kAbsentRef) m3 = !SlabTest(s.r, lx.w, ly.w, lz.w, hx.w, hy.w, hz.w, s.tmin, limit, e3);
    // Sorting network on four.
    OrderPair(m0, e0, r0, m1, e1, r1);
    OrderPair(m2, e2, r2, m3, e3, r3);
    OrderPair(m0, e0, r0, m2, e2, r2);
    OrderPair(m1, e1, r1, m3, e3, r3);
    OrderPair(m1, e1, r1, m2, e2, r2);
    if (m0) return 0;  // no child hit
    const int pushes = (m1 ? 0 : 1) + (m2 ? 0 : 1) + (m3 ? 0 : 1);
    if (s.sp + pushes > Stack::kTotalEntries) {  // unreachable when the host's depth bound holds
        atomicOr(error, kTraceErrorStackOverflow);
        s.best.hit = false;
        return -1;
    }
    if (!m3) st.Put(col, s.sp++, make_int2(r3, __float_as_int(e3)));
    if (!m2) st.Put(col, s.sp++, make_int2(r2, __float_as_int(e2)));
    if (!m1) st.Put(col, s.sp++, make_int2(r1, __float_as_int(e1)));
    s.cur = r0;
    return 1;
}

template <bool kAny, bool kStats, bool kTwo, typename Stack, bool kFilter = false, bool kWide = false>
__device__ __forceinline__ bool Step(const AccelParams& a, const float4* rays, int64_t ray, Traversal& s, Stack& st,
                                     int2* col, int* error, const uint8_t* tri_clear = nullptr,
                                     const uint8_t* sphere_clear = nullptr, ClearHits* clear = nullptr) {
    const bool in_blas = kTwo && s.level == 1;
    if (kWide && s.cur >= 0) {
        const int r = WideStep(a, s, st, col, error);
        if (r != 0) return r > 0;
        return Pop<kAny, kTwo>(rays, ray, s, st, col);
    }
    if (s.cur >= 0) {
        const float4* p = reinterpret_cast<const float4*>(a.pairs + s.cur);
        const unsigned long long pol = NodePolicy();
        const float4 pa = LdNode(p, pol), pb = LdNode(p + 1, pol), pc = LdNode(p + 2, pol);
        const float4 pdf = LdNode(p + 3, pol);
        const int4 pd = make_int4(__float_as_int(pdf.x), __float_as_int(pdf.y), __float_as_int(pdf.z),
                                  __float_as_int(pdf.w));
        const float limit = in_blas ? s.local.t : s.best.t;
        float le = 0.0f, re = 0.0f;
        bool hl = false, hr = false;
        if (pd.x != kAbsentRef) {
            if (kStats) ++s.nodes;
            hl = SlabTest(s.r, pa.x, pa.y, pa.z, pa.w, pb.x, pb.y, s.tmin, limit, le);
        }
        if (pd.y != kAbsentRef) {
            if (kStats) ++s.nodes;
            hr = SlabTest(s.r, pb.z, pb.w, pc.x, pc.y, pc.z, pc.w, s.tmin, limit, re);
        }
        if (hl && hr) {
            const bool left_first = le <= re;
            if (s.sp >= Stack::kTotalEntries) {  // unreachable when the host's depth bound holds
                atomicOr(error, kTraceErrorStackOverflow);
                s.best.hit = false;
                return false;
            }
            st.Put(col, s.sp, left_first ? make_int2(pd.y, __float_as_int(re)) : make_int2(pd.x, __float_as_int(le)));
            ++s.sp;
            s.cur = left_first ? pd.x : pd.y;
            return true;
        }
        if (hl) {
            s.cur = pd.x;
            return true;
        }
        if (hr) {
            s.cur = pd.y;
            return true;
        }
        return Pop<kAny, kTwo>(rays, ray, s, st, col);
    }

    // Leaf: a run of records ending at the one flagged kRecLast.
    int32_t rec = ~s.cur;
    for (;;) {
        const float4* q = reinterpret_cast<const float4*>(a.records + rec);
        const float4 v0 = Ld(q), v1 = Ld(q + 1);
        const int32_t flags = __float_as_int(v1.w);
        const int32_t kind = (flags >> 1) & 7;
        if (kind == kRecTriangle) {
            const float4 v2 = Ld(q + 2);
            if (kStats) ++s.tris;
            if (in_blas) {
                const Nearest keep = s.local;
                const bool acc = TriangleTest(s.r, v0, v1, v2, s.tmin, s.local);
                if (kAny && acc && s.local.t < s.best.t) {
                    if (kFilter && tri_clear[s.local.id]) {
                        s.saw = true;
                        clear->Add(s.local.t, s.local.id);
                        s.local = keep;
                    } else {
                        s.best = s.local;
                        s.best_inst = s.cur_inst;
                        return false;
                    }
                }
            } else {
                const Nearest keep = s.best;
                const bool acc = TriangleTest(s.r, v0, v1, v2, s.tmin, s.best);
                if (kAny && acc) {
                    if (kFilter && tri_clear[s.best.id]) {
                        s.saw = true;
                        clear->Add(s.best.t, s.best.id);
                        s.best = keep;
                    } else {
                        return false;
                    }
                }
            }
        } else if (kind == kRecSphere) {
            if (kStats) ++s.spheres;
            if (in_blas) {
                const Nearest keep = s.local;
                const bool acc = SphereTest(s.r, v0, v1, s.tmin, s.local);
                if (kAny && acc && s.local.t < s.best.t) {
                    if (kFilter && sphere_clear[-2 - s.local.id]) {
                        s.saw = true;
                        clear->Add(s.local.t, s.local.id);
                        s.local = keep;
                    } else {
                        s.best = s.local;
                        s.best_inst = s.cur_inst;
                        return false;
                    }
                }
            } else {
                const Nearest keep = s.best;
                const bool acc = SphereTest(s.r, v0, v1, s.tmin, s.best);
                if (acc) s.best_inst = -1;
                if (kAny && acc) {
                    if (kFilter && sphere_clear[-2 - s.best.id]) {
                        s.saw = true;
                        clear->Add(s.best.t, s.best.id);
                        s.best = keep;
                    } else {
                        return false;
                    }
                }
            }
        } else if (kTwo && kind == kRecInstance) {
            // Descend into the instance's BLAS with the ray in object space
            // (TransformPoint / TransformVector by world_to_object; the
            // direction is not normalised, so t stays in world units).
            const int32_t inst = __float_as_int(v0.w);
            const float4* ip = reinterpret_cast<const float4*>(a.instances + inst);
            const float4 m0 = Ld(ip), m1 = Ld(ip + 1), m2 = Ld(ip + 2), ba = Ld(ip + 3), bb = Ld(ip + 4);
            const float4 rows[3] = {m0, m1, m2};
            RayPre obj;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float4 m = rows[k];
                obj.o[k] = __fadd_rn(
                    __fadd_rn(__fadd_rn(__fmul_rn(m.x, s.r.o[0]), __fmul_rn(m.y, s.r.o[1])), __fmul_rn(m.z, s.r.o[2])),
                    m.w);
                obj.d[k] =
                    __fadd_rn(__fadd_rn(__fmul_rn(m.x, s.r.d[0]), __fmul_rn(m.y, s.r.d[1])), __fmul_rn(m.z, s.r.d[2]));
            }
            Precompute(obj);
            const int32_t root = __float_as_int(bb.z);
            if (root != kAbsentRef) {
                if (kStats) ++s.nodes;
                float entry;
                if (SlabTest(obj, ba.x, ba.y, ba.z, ba.w, bb.x, bb.y, s.tmin, s.best.t, entry)) {
                    s.local.t = s.best.t;
                    s.local.id = -1;
                    s.local.prim = -1;
                    s.local.u = 0.0f;
                    s.local.v = 0.0f;
                    s.local.hit = false;
                    s.level = 1;
                    s.blas_base = s.sp;
                    s.cur_inst = inst;
                    s.tl_resume = (flags & kRecLast) ? -1 : rec + 1;
                    s.r = obj;
                    s.cur = root;
                    return true;
                }
            }
        } else if (kStats) {
            if (kind == kRecSkipCountTriangle) ++s.tris;
            if (kind == kRecSkipCountSphere) ++s.spheres;
        }
        if (flags & kRecLast) break;
        ++rec;
    }
    return Pop<kAny, kTwo>(rays, ray, s, st, col);
}

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

template <bool kAny, bool kStats, bool kTwo, int kTotal, int kBlock, int kStepsPerRefill, int kMinBlocks,
          bool kWide = false>
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
                    ray = static_cast<int64_t>(idx);
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
#pragma unroll 1
        for (int k = 0; k < kStepsPerRefill && alive; ++k) {
            alive = Step<kAny, kStats, kTwo, StackStore<kTotal, kBlock>, false, kWide>(args.accel, args.rays, ray, s, st,
                                                                                       col, args.error);
            if (!alive) WriteResult<kAny, kStats>(args, ray, s);
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
// with the same bias, remaining-distance and 16-query rules. What differs
// from re-tracing is rounding: t is the traversal's t from the ray origin
// less the distance already advanced, not a new intersection from the
// re-spawned origin. Persistent warps with per-lane refill, like TraceKernel.
template <bool kTwo, int kTotal>
__global__ void __launch_bounds__(kTraceBlock, kShadowBlocksPerSm) ShadowTransmittanceKernel(ShadowArgs args) {
    __shared__ int2 s_stack[kShadowShortStack * kTraceBlock];
    __shared__ float s_clear_t[kClearHits * kTraceBlock];
    __shared__ int32_t s_clear_id[kClearHits * kTraceBlock];
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
    const unsigned long long count = *args.count_ptr;

    // The reference loop over the kept clear surfaces; returns the RGB
    // transmittance, w = 1 when visible, all 0 when occluded.
    auto replay = [&]() -> float4 {
        const float4 ra = Ld(args.rays + 2 * ray);
        const float4 rb = Ld(args.rays + 2 * ray + 1);
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
                // A surface beyond the kept ones would be this query's answer.
                if (clear.dropped) return occluded;
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
            const int32_t material = id >= 0 ? args.prim_material[args.tri_prim[id]] : args.sphere_material[-2 - id];
            if (material < 0 || (args.materials[material].kind != 2 && args.materials[material].kind != 3)) {
                return occluded;
            }
            const DevMaterial& m = args.materials[material];
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
        const int32_t slot = args.out_index[ray];
        float4 tr;
        if (s.best.hit) {
            tr = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        } else if (!s.saw) {
            tr = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
        } else {
            tr = replay();
        }
        args.transmittance[slot] = tr;
        if (tr.w == 0.0f) CountLanes(args.occluded_count);
    };
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
                    ray = static_cast<int64_t>(idx);
                    const float4 b = Ld(args.rays + 2 * ray + 1);
                    const float tmin = Ld(args.rays + 2 * ray).w;
                    clear.n = 0;
                    clear.dropped = false;
                    alive = Begin(args.accel, args.rays, ray, tmin, b.w, s);
                    if (!alive) finish();
                }
            }
        }
        if (!__any_sync(kFull, alive)) {
            if (__all_sync(kFull, exhausted)) break;
            continue;
        }
#pragma unroll 1
        for (int k = 0; k < 8 && alive; ++k) {
            alive = Step<true, false, kTwo, StackStore<kTotal, kTraceBlock, kShadowShortStack>, true>(
                args.accel, args.rays, ray, s, st, col, args.error, args.tri_clear, args.sphere_clear, &clear);
            if (!alive) finish();
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
          bool kWide = false>
cudaError_t LaunchOne(const TraceArgs& args, cudaStream_t stream, int sm_count) {
    auto kernel = TraceKernel<kAny, kStats, kTwo, kTotal, kBlock, kStepsPerRefill, kMinBlocks, kWide>;
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

template <bool kTwo, int kTotal>
cudaError_t LaunchShadowOne(const ShadowArgs& args, cudaStream_t stream, int sm_count) {
    auto kernel = ShadowTransmittanceKernel<kTwo, kTotal>;
    int64_t blocks = 0;
    const cudaError_t err = PersistentGrid(kernel, kTraceBlock, args.capacity, sm_count, blocks);
    if (err != cudaSuccess) return err;
    kernel<<<static_cast<unsigned>(blocks), kTraceBlock, 0, stream>>>(args);
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
    if (two) return deep ? LaunchShadowOne<true, kMaxTraceStack>(args, stream, sm_count)
                         : LaunchShadowOne<true, 64>(args, stream, sm_count);
    return deep ? LaunchShadowOne<false, kMaxTraceStack>(args, stream, sm_count)
                : LaunchShadowOne<false, 64>(args, stream, sm_count);
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

cudaError_t LaunchProbe(const ProbeArgs& args, cudaStream_t stream, int sm_count) {
    const bool two = args.accel.two_level != 0;
    const bool deep = args.accel.stack_limit > 64;
    if (two) return deep ? LaunchProbeOne<true, kMaxTraceStack>(args, stream, sm_count)
                         : LaunchProbeOne<true, 64>(args, stream, sm_count);
    return deep ? LaunchProbeOne<false, kMaxTraceStack>(args, stream, sm_count)
                : LaunchProbeOne<false, 64>(args, stream, sm_count);
}

}  // namespace yrc
