// Per-ray BVH traversal core shared by the traversal kernels
// (trace_kernels.cu) and the render stages that trace rays one per thread
// (render_kernels.cu): the traversal state, the split shared/local stack,
// ray set-up, the stack pop with culling and one traversal step.
//
// Semantics are those of IntersectBvh (src/accel/bvh_traversal.cpp:253-345)
// and IntersectTwoLevelBvh (src/accel/two_level_bvh.cpp:365-481) with the
// reference's visiting order; every float operation goes through an
// explicitly rounded intrinsic, so results do not depend on the including
// translation unit's contraction setting.
#pragma once

#include <cuda_runtime.h>

#include "device_layout.cuh"
#include "trace_kernels.hpp"

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

// Warp-aggregated increment of a statistics counter by the calling lanes;
// lanes that hold different counters (a pooled launch's lanes may serve
// different jobs) count into their own.
__device__ __forceinline__ void CountLanes(unsigned long long* counter) {
    const unsigned mask = __activemask();
    const unsigned peers = __match_any_sync(mask, reinterpret_cast<unsigned long long>(counter));
    if ((threadIdx.x & 31u) == static_cast<unsigned>(__ffs(peers) - 1)) {
        atomicAdd(counter, static_cast<unsigned long long>(__popc(peers)));
    }
}

// Loads the pooled jobs' work counts (written on the device by the stage
// that filled their queues) into `ends` as an inclusive prefix sum;
// returns the total. Called by the whole block.
template <typename Job>
__device__ __forceinline__ unsigned long long LoadPoolEnds(const Job* jobs, int njobs, unsigned long long* ends) {
    for (int j = threadIdx.x; j < njobs; j += blockDim.x) ends[j] = *jobs[j].count_ptr;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int j = 1; j < njobs; ++j) ends[j] += ends[j - 1];
    }
    __syncthreads();
    return njobs > 0 ? ends[njobs - 1] : 0ull;
}

// The job that pooled work item idx (< the total) belongs to: the first
// whose queue ends past it.
__device__ __forceinline__ int PoolJobOf(const unsigned long long* ends, int njobs, unsigned long long idx) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (ends[mid] > idx) {
            hi = mid;
        } else {
            lo = mid + 1;
        }
    }
    return lo;
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
// The shadow kernel keeps 6 stack entries in shared memory (with the clear
// list, 22 KB per block of 128 threads, 8 blocks per SM); the rest of the
// shared-memory carve-out stays L1 cache for the tree (11 entries, 27.6 KB
// per block, measured 1.5-2 % slower on the instanced render).
constexpr int kShadowShortStack = 6;
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
    if (r0 != kAbsentRef) m0 = !SlabTestInterval(s.r, lx.x, ly.x, lz.x, hx.x, hy.x, hz.x, s.tmin, limit, e0);
    if (r1 != kAbsentRef) m1 = !SlabTestInterval(s.r, lx.y, ly.y, lz.y, hx.y, hy.y, hz.y, s.tmin, limit, e1);
    if (r2 != kAbsentRef) m2 = !SlabTestInterval(s.r, lx.z, ly.z, lz.z, hx.z, hy.z, hz.z, s.tmin, limit, e2);
    if (r3 != kAbsentRef) m3 = !SlabTestInterval(s.r, lx.w, ly.w, lz.w, hx.w, hy.w, hz.w, s.tmin, limit, e3);
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
            hl = SlabTestInterval(s.r, pa.x, pa.y, pa.z, pa.w, pb.x, pb.y, s.tmin, limit, le);
        }
        if (pd.y != kAbsentRef) {
            if (kStats) ++s.nodes;
            hr = SlabTestInterval(s.r, pb.z, pb.w, pc.x, pc.y, pc.z, pc.w, s.tmin, limit, re);
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
                if (SlabTestInterval(obj, ba.x, ba.y, ba.z, ba.w, bb.x, bb.y, s.tmin, s.best.t, entry)) {
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

}  // namespace
}  // namespace yrc
