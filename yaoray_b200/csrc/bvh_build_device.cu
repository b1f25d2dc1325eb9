// Device builder of the reference's binned-SAH BVH (BuildBvh,
// src/accel/bvh_builder.cpp:269-286, split policy
// src/accel/bvh_split_policy.cpp:38-182, serial recursion
// src/accel/bvh_serial_builder.cpp:8-57): the same nodes and primitive
// slots, byte for byte, as the host builder in bvh_build.cpp.
//
// Why the parallel build can be exact:
//  * range bounds, centroid bounds and the SAH buckets are min / max / count
//    reductions, independent of order except for the sign of zero: the
//    reference keeps the earlier operand on ties (std::min(acc, x)), so a
//    reduction that orders by (value with -0 == +0, position) and then reads
//    the winning element's own float picks the same bits;
//  * the SAH sweep and the cost comparisons are a dozen sequential float
//    operations per range, done by one thread in the reference's order with
//    round-to-nearest intrinsics (no contraction);
//  * std::partition on random-access iterators is the two-pointer partition:
//    with T elements satisfying the predicate, the i-th element that fails it
//    inside [begin, begin + T) (counted from the left) is swapped with the
//    i-th element that satisfies it inside [begin + T, end) (counted from the
//    right) and nothing else moves, which is a pair of prefix counts.
// The median split (std::nth_element) has no order-free description; it only
// occurs for degenerate ranges (every centroid extent below 1e-8 or a
// zero-area box). Its permutation is by definition the standard library's,
// so the host computes it with its own std::nth_element: between levels for
// large ranges (the device lists them, the host permutes them before their
// children are read), and by the host's serial builder for a small subtree
// that meets one. Everything else stays on the device.
//
// Execution: ranges larger than kSmall are processed level by level, one
// 512-thread block per range (bounds, buckets with per-warp bins, decision,
// partition, child ranges), the rest as whole subtrees by one thread each;
// then subtree sizes bottom-up and pre-order indices top-down give every
// node its slot in the reference's depth-first layout.
#include "yrc_internal.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

namespace yrc {
namespace {

constexpr int kBuckets = 12;            // SahBucketCount
constexpr float kTraversalCost = 0.5f;  // SahTraversalCost
constexpr float kDegenerateExtent = 1.0e-8f;
constexpr int kSmall = 64;   // ranges of at most this many refs: one thread builds the subtree
constexpr int kBlock = 512;  // threads per large range
constexpr int kWarps = kBlock / 32;
constexpr int kMaxSmallDepth = 64;  // explicit stack of the one-thread subtree build (depth <= kSmall)

enum BuildFlag : int { kFlagNonFinite = 2, kFlagEmpty = 4, kFlagHostSubtree = 8 };

// One ref in the device layout: lo.w carries the flat index.
struct DevRef {
    float4 lo, hi, c;
};

struct Range {
    int32_t begin, end, depth, id;
};

// A range of the level-by-level phase.
struct BigNode {
    float lo[3], hi[3];
    int32_t begin, count, depth, leaf;
    int32_t left, right;  // >= 0: big node id; < 0: small subtree -1 - id
};

struct SmallTask {
    int32_t begin, count, depth, pad;
};

__device__ __forceinline__ float Comp(const float4& v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

// Order key of a float for min / max reductions: monotone in the value,
// -0 and +0 equal.
__device__ __forceinline__ uint32_t OrderKey(float f) {
    const uint32_t u = __float_as_uint(f == 0.0f ? 0.0f : f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ unsigned long long MinKey(float f, uint32_t pos) {
    return (static_cast<unsigned long long>(OrderKey(f)) << 32) | pos;
}
__device__ __forceinline__ unsigned long long MaxKey(float f, uint32_t pos) {
    return (static_cast<unsigned long long>(OrderKey(f)) << 32) | (0xffffffffu - pos);
}
__device__ __forceinline__ uint32_t MinPos(unsigned long long k) { return static_cast<uint32_t>(k); }
__device__ __forceinline__ uint32_t MaxPos(unsigned long long k) { return 0xffffffffu - static_cast<uint32_t>(k); }
constexpr unsigned long long kMinEmpty = ~0ull;
constexpr unsigned long long kMaxEmpty = 0ull;

// std::min / std::max with the accumulated operand first.
__device__ __forceinline__ float MinKeep(float acc, float x) { return x < acc ? x : acc; }
__device__ __forceinline__ float MaxKeep(float acc, float x) { return acc < x ? x : acc; }

struct FBox {
    float lo[3], hi[3];
};
__device__ __forceinline__ void Empty(FBox& b) {
    for (int a = 0; a < 3; ++a) {
        b.lo[a] = __int_as_float(0x7f800000);
        b.hi[a] = __int_as_float(0xff800000);
    }
}
__device__ __forceinline__ void MergeInto(FBox& acc, const FBox& b) {
    for (int a = 0; a < 3; ++a) {
        acc.lo[a] = MinKeep(acc.lo[a], b.lo[a]);
        acc.hi[a] = MaxKeep(acc.hi[a], b.hi[a]);
    }
}
__device__ __forceinline__ float HalfArea2(const FBox& b) {
    if (b.lo[0] > b.hi[0] || b.lo[1] > b.hi[1] || b.lo[2] > b.hi[2]) return 0.0f;
    const float ex = __fsub_rn(b.hi[0], b.lo[0]);
    const float ey = __fsub_rn(b.hi[1], b.lo[1]);
    const float ez = __fsub_rn(b.hi[2], b.lo[2]);
    const float s = __fadd_rn(__fadd_rn(__fmul_rn(ex, ey), __fmul_rn(ey, ez)), __fmul_rn(ez, ex));
    return __fmul_rn(2.0f, s);
}
__device__ __forceinline__ int BucketOf(float c, float lo, float extent) {
    const float offset = __fdiv_rn(__fsub_rn(c, lo), extent);
    const int b = __float2int_rz(__fmul_rn(offset, static_cast<float>(kBuckets)));
    return b < 0 ? 0 : (b > kBuckets - 1 ? kBuckets - 1 : b);
}

// SAH over the 3 x 12 buckets of one range: the reference's sweeps and cost
// comparisons in its order. counts / boxes are [axis][bucket]; axes whose
// centroid extent is below the threshold are skipped.
__device__ bool BestSplit(const int* counts, const FBox* boxes, const FBox& node, const float cext[3], int& best_axis,
                          int& best_split, float& best_cost) {
    best_axis = -1;
    best_split = -1;
    best_cost = __int_as_float(0x7f800000);
    const float parent_area = HalfArea2(node);
    if (!(parent_area > 0.0f)) return false;
    for (int axis = 0; axis < 3; ++axis) {
        if (cext[axis] < kDegenerateExtent) continue;
        const int* cnt = counts + axis * kBuckets;
        const FBox* box = boxes + axis * kBuckets;
        int lc[kBuckets], rc[kBuckets];
        FBox lb[kBuckets], rb[kBuckets];
        lc[0] = cnt[0];
        lb[0] = box[0];
        for (int i = 1; i < kBuckets; ++i) {
            lc[i] = lc[i - 1] + cnt[i];
            lb[i] = lb[i - 1];
            MergeInto(lb[i], box[i]);
        }
        rc[kBuckets - 1] = cnt[kBuckets - 1];
        rb[kBuckets - 1] = box[kBuckets - 1];
        for (int i = kBuckets - 2; i >= 0; --i) {
            rc[i] = rc[i + 1] + cnt[i];
            rb[i] = rb[i + 1];
            MergeInto(rb[i], box[i]);
        }
        for (int s = 0; s < kBuckets - 1; ++s) {
            const int nl = lc[s], nr = rc[s + 1];
            if (nl == 0 || nr == 0) continue;
            const float num = __fadd_rn(__fmul_rn(__int2float_rn(nl), HalfArea2(lb[s])),
                                        __fmul_rn(__int2float_rn(nr), HalfArea2(rb[s + 1])));
            const float cost = __fadd_rn(kTraversalCost, __fdiv_rn(num, parent_area));
            if (cost < best_cost) {
                best_cost = cost;
                best_axis = axis;
                best_split = s;
            }
        }
    }
    return best_axis >= 0;
}

// Bounds keys and buckets of a range reduced by many blocks (ranges larger
// than kWide): 12 bound keys (node lo/hi, centroid lo/hi, interleaved per
// axis) and per axis and bucket a count and 6 box keys.
constexpr int kWide = 1 << 15;
constexpr int kChunk = 1 << 13;
struct WideResult {
    unsigned long long keys[12];
    unsigned cnt[3][kBuckets];
    unsigned long long bins[3][kBuckets][6];
};
struct WideChunk {
    int32_t begin, end, slot, pad;
};

struct LevelArgs {
    DevRef* refs;
    int32_t* tmp;  // per position: scratch for the partition
    const Range* ranges;
    int32_t range_count;
    Range* next;
    unsigned* next_count;
    BigNode* big;
    unsigned* big_count;
    SmallTask* small;
    unsigned* small_count;
    int32_t max_leaf;
    int* flags;
    const int32_t* wide_of;  // per range of this level: its WideResult, -1 none (nullptr: none at all)
    const WideResult* wide;
    int2* median;            // ranges split at their median: (begin, end), permuted by the host
    unsigned* median_count;
};

// Warp-level min / max of 64-bit keys.
__device__ __forceinline__ unsigned long long WarpMin(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}
__device__ __forceinline__ unsigned long long WarpMax(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

// Creates the child range [b, e) of big node `parent` (side 0 left, 1 right).
__device__ void SpawnChild(const LevelArgs& a, int parent, int side, int b, int e, int depth) {
    int32_t ref;
    if (e - b > kSmall) {
        const unsigned id = atomicAdd(a.big_count, 1u);
        const unsigned slot = atomicAdd(a.next_count, 1u);
        a.next[slot] = Range{b, e, depth, static_cast<int32_t>(id)};
        ref = static_cast<int32_t>(id);
    } else {
        const unsigned id = atomicAdd(a.small_count, 1u);
        a.small[id] = SmallTask{b, e - b, depth, 0};
        ref = -1 - static_cast<int32_t>(id);
    }
    if (side == 0) a.big[parent].left = ref;
    else a.big[parent].right = ref;
}

// One block per range larger than kSmall.
__global__ void __launch_bounds__(kBlock) LevelKernel(LevelArgs a) {
    __shared__ unsigned long long s_red[12][kWarps];
    __shared__ unsigned s_cnt[kWarps][3][kBuckets];
    __shared__ unsigned long long s_key[kWarps][3][kBuckets][6];
    __shared__ float s_node[6], s_cen[6];
    __shared__ int s_decision[4];  // leaf, axis, split, left count
    __shared__ unsigned s_scan[2][kWarps];
    __shared__ unsigned s_base[2];

    const Range r = a.ranges[blockIdx.x];
    const int begin = r.begin, end = r.end, count = end - begin;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    DevRef* refs = a.refs;
    const int wslot = a.wide_of ? a.wide_of[blockIdx.x] : -1;
    const WideResult* wide = wslot >= 0 ? a.wide + wslot : nullptr;

    // --- range bounds and centroid bounds (first minimum / maximum wins)
    unsigned long long k[12];
    for (int j = 0; j < 6; ++j) k[j] = (j % 2 == 0) ? kMinEmpty : kMaxEmpty;  // node lo/hi interleaved
    for (int j = 6; j < 12; ++j) k[j] = (j % 2 == 0) ? kMinEmpty : kMaxEmpty;  // centroid lo/hi interleaved
    for (int i = begin + tid; !wide && i < end; i += kBlock) {
        const DevRef e = refs[i];
        const uint32_t p = static_cast<uint32_t>(i);
        for (int ax = 0; ax < 3; ++ax) {
            const unsigned long long lo = MinKey(Comp(e.lo, ax), p), hi = MaxKey(Comp(e.hi, ax), p);
            const unsigned long long clo = MinKey(Comp(e.c, ax), p), chi = MaxKey(Comp(e.c, ax), p);
            k[2 * ax] = lo < k[2 * ax] ? lo : k[2 * ax];
            k[2 * ax + 1] = hi > k[2 * ax + 1] ? hi : k[2 * ax + 1];
            k[6 + 2 * ax] = clo < k[6 + 2 * ax] ? clo : k[6 + 2 * ax];
            k[7 + 2 * ax] = chi > k[7 + 2 * ax] ? chi : k[7 + 2 * ax];
        }
    }
    for (int j = 0; j < 12; ++j) {
        const unsigned long long v = (j % 2 == 0) ? WarpMin(k[j]) : WarpMax(k[j]);
        if (lane == 0) s_red[j][warp] = v;
    }
    __syncthreads();
    if (tid < 12) {
        unsigned long long v = s_red[tid][0];
        for (int w = 1; w < kWarps; ++w) {
            const unsigned long long x = s_red[tid][w];
            v = (tid % 2 == 0) ? (x < v ? x : v) : (x > v ? x : v);
        }
        if (wide) v = wide->keys[tid];
        const int ax = (tid % 6) / 2;
        const bool is_min = tid % 2 == 0;
        const uint32_t p = is_min ? MinPos(v) : MaxPos(v);
        const DevRef e = refs[p];
        if (tid < 6) s_node[is_min ? ax : 3 + ax] = Comp(is_min ? e.lo : e.hi, ax);
        else s_cen[is_min ? ax : 3 + ax] = Comp(e.c, ax);
    }
    // --- buckets (per-warp bins)
    for (int j = tid; j < kWarps * 3 * kBuckets; j += kBlock) {
        (&s_cnt[0][0][0])[j] = 0u;
        for (int q = 0; q < 6; ++q) (&s_key[0][0][0][0])[j * 6 + q] = (q < 3) ? kMinEmpty : kMaxEmpty;
    }
    __syncthreads();
    FBox node;
    float cext[3], clo[3];
    for (int ax = 0; ax < 3; ++ax) {
        node.lo[ax] = s_node[ax];
        node.hi[ax] = s_node[3 + ax];
        clo[ax] = s_cen[ax];
        cext[ax] = __fsub_rn(s_cen[3 + ax], s_cen[ax]);
    }
    const bool leaf_by_size = count <= a.max_leaf;
    const float parent_area = HalfArea2(node);
    if (!wide && !leaf_by_size && parent_area > 0.0f) {
        for (int i = begin + tid; i < end; i += kBlock) {
            const DevRef e = refs[i];
            const uint32_t p = static_cast<uint32_t>(i);
            for (int ax = 0; ax < 3; ++ax) {
                if (cext[ax] < kDegenerateExtent) continue;
                const int b = BucketOf(Comp(e.c, ax), clo[ax], cext[ax]);
                atomicAdd(&s_cnt[warp][ax][b], 1u);
                unsigned long long* key = s_key[warp][ax][b];
                for (int q = 0; q < 3; ++q) {
                    atomicMin(key + q, MinKey(Comp(e.lo, q), p));
                    atomicMax(key + 3 + q, MaxKey(Comp(e.hi, q), p));
                }
            }
        }
    }
    __syncthreads();
    if (tid == 0) {
        int leaf = 1, axis = -1, split = -1, left_count = 0;
        if (!leaf_by_size) {
            int counts[3 * kBuckets];
            FBox boxes[3 * kBuckets];
            for (int j = 0; j < 3 * kBuckets; ++j) {
                unsigned c = 0;
                unsigned long long key[6];
                for (int q = 0; q < 6; ++q) key[q] = q < 3 ? kMinEmpty : kMaxEmpty;
                for (int w = 0; w < (wide ? 1 : kWarps); ++w) {
                    c += wide ? (&wide->cnt[0][0])[j] : (&s_cnt[w][0][0])[j];
                    const unsigned long long* kk = wide ? (&wide->bins[0][0][0]) + j * 6 : (&s_key[w][0][0][0]) + j * 6;
                    for (int q = 0; q < 3; ++q) {
                        key[q] = kk[q] < key[q] ? kk[q] : key[q];
                        key[3 + q] = kk[3 + q] > key[3 + q] ? kk[3 + q] : key[3 + q];
                    }
                }
                counts[j] = static_cast<int>(c);
                Empty(boxes[j]);
                if (c > 0) {
                    for (int q = 0; q < 3; ++q) {
                        boxes[j].lo[q] = Comp(refs[MinPos(key[q])].lo, q);
                        boxes[j].hi[q] = Comp(refs[MaxPos(key[3 + q])].hi, q);
                    }
                }
            }
            float best_cost;
            const bool found = BestSplit(counts, boxes, node, cext, axis, split, best_cost);
            if (found && best_cost >= __int2float_rn(count)) {
                leaf = 1;
            } else if (!found) {
                // The reference's median split (std::nth_element): an
                // interior node at begin + count / 2 whose range the host
                // permutes with its own std::nth_element before the next
                // level reads it.
                leaf = 0;
                axis = -1;
                left_count = count / 2;
                a.median[atomicAdd(a.median_count, 1u)] = make_int2(begin, end);
            } else {
                leaf = 0;
                for (int b = 0; b <= split; ++b) left_count += counts[axis * kBuckets + b];
            }
        }
        s_decision[0] = leaf;
        s_decision[1] = axis;
        s_decision[2] = split;
        s_decision[3] = left_count;
        BigNode& n = a.big[r.id];
        for (int ax = 0; ax < 3; ++ax) {
            n.lo[ax] = node.lo[ax];
            n.hi[ax] = node.hi[ax];
        }
        n.begin = begin;
        n.count = count;
        n.depth = r.depth;
        n.leaf = leaf;
        n.left = n.right = 0;
    }
    __syncthreads();
    if (s_decision[0]) return;
    const int axis = s_decision[1], split = s_decision[2];
    const int mid = begin + s_decision[3];
    if (axis < 0) {  // median split: no partition here
        if (tid == 0) {
            SpawnChild(a, r.id, 0, begin, mid, r.depth + 1);
            SpawnChild(a, r.id, 1, mid, end, r.depth + 1);
        }
        return;
    }
    const float lo = clo[axis], extent = cext[axis];

    // --- two-pointer partition: the i-th left-side failure (from the left)
    // swaps with the i-th right-side success (from the right).
    // Pass 1: positions of right-side successes in ascending order -> tmp.
    if (tid == 0) s_base[0] = s_base[1] = 0;
    __syncthreads();
    for (int base = begin; base < end; base += kBlock) {
        const int i = base + tid;
        bool mr = false, ml = false;
        if (i < end) {
            const bool pred = BucketOf(Comp(refs[i].c, axis), lo, extent) <= split;
            mr = i >= mid && pred;
            ml = i < mid && !pred;
        }
        const unsigned bm = __ballot_sync(0xffffffffu, mr), bl = __ballot_sync(0xffffffffu, ml);
        if (lane == 0) {
            s_scan[0][warp] = __popc(bm);
            s_scan[1][warp] = __popc(bl);
        }
        __syncthreads();
        unsigned off_r = s_base[0], off_l = s_base[1];
        for (int w = 0; w < warp; ++w) {
            off_r += s_scan[0][w];
            off_l += s_scan[1][w];
        }
        const unsigned lt = (1u << lane) - 1u;
        if (mr) a.tmp[begin + off_r + __popc(bm & lt)] = i;
        (void)off_l;
        __syncthreads();
        if (tid == 0) {
            for (int w = 0; w < kWarps; ++w) {
                s_base[0] += s_scan[0][w];
                s_base[1] += s_scan[1][w];
            }
        }
        __syncthreads();
    }
    const unsigned m = s_base[0];  // == s_base[1]
    __syncthreads();
    if (tid == 0) s_base[1] = 0;
    __syncthreads();
    // Pass 2: each left-side failure of ascending rank j swaps with the
    // right-side success of descending rank j.
    for (int base = begin; base < mid; base += kBlock) {
        const int i = base + tid;
        bool ml = false;
        if (i < mid) ml = !(BucketOf(Comp(refs[i].c, axis), lo, extent) <= split);
        const unsigned bl = __ballot_sync(0xffffffffu, ml);
        if (lane == 0) s_scan[1][warp] = __popc(bl);
        __syncthreads();
        unsigned off_l = s_base[1];
        for (int w = 0; w < warp; ++w) off_l += s_scan[1][w];
        const unsigned lt = (1u << lane) - 1u;
        if (ml) {
            const unsigned j = off_l + __popc(bl & lt);
            const int partner = a.tmp[begin + (m - 1u - j)];
            const DevRef x = refs[i];
            refs[i] = refs[partner];
            refs[partner] = x;
        }
        __syncthreads();
        if (tid == 0) {
            for (int w = 0; w < kWarps; ++w) s_base[1] += s_scan[1][w];
        }
        __syncthreads();
    }
    if (tid == 0) {
        SpawnChild(a, r.id, 0, begin, mid, r.depth + 1);
        SpawnChild(a, r.id, 1, mid, end, r.depth + 1);
    }
}

// Bounds keys of the chunks of wide ranges (one block per chunk).
__global__ void __launch_bounds__(kBlock) WideBoundsKernel(const DevRef* refs, const WideChunk* chunks,
                                                           WideResult* wide) {
    __shared__ unsigned long long s_red[12][kWarps];
    const WideChunk ch = chunks[blockIdx.x];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    unsigned long long k[12];
    for (int j = 0; j < 12; ++j) k[j] = (j % 2 == 0) ? kMinEmpty : kMaxEmpty;
    for (int i = ch.begin + tid; i < ch.end; i += kBlock) {
        const DevRef e = refs[i];
        const uint32_t p = static_cast<uint32_t>(i);
        for (int ax = 0; ax < 3; ++ax) {
            const unsigned long long lo = MinKey(Comp(e.lo, ax), p), hi = MaxKey(Comp(e.hi, ax), p);
            const unsigned long long clo = MinKey(Comp(e.c, ax), p), chi = MaxKey(Comp(e.c, ax), p);
            k[2 * ax] = lo < k[2 * ax] ? lo : k[2 * ax];
            k[2 * ax + 1] = hi > k[2 * ax + 1] ? hi : k[2 * ax + 1];
            k[6 + 2 * ax] = clo < k[6 + 2 * ax] ? clo : k[6 + 2 * ax];
            k[7 + 2 * ax] = chi > k[7 + 2 * ax] ? chi : k[7 + 2 * ax];
        }
    }
    for (int j = 0; j < 12; ++j) {
        const unsigned long long v = (j % 2 == 0) ? WarpMin(k[j]) : WarpMax(k[j]);
        if (lane == 0) s_red[j][warp] = v;
    }
    __syncthreads();
    if (tid < 12) {
        unsigned long long v = s_red[tid][0];
        for (int w = 1; w < kWarps; ++w) {
            const unsigned long long x = s_red[tid][w];
            v = (tid % 2 == 0) ? (x < v ? x : v) : (x > v ? x : v);
        }
        if (tid % 2 == 0) atomicMin(&wide[ch.slot].keys[tid], v);
        else atomicMax(&wide[ch.slot].keys[tid], v);
    }
}

// Buckets of the chunks of wide ranges (block bins, then one atomic per bin
// and key into the range's result).
__global__ void __launch_bounds__(kBlock) WideBinsKernel(const DevRef* refs, const WideChunk* chunks,
                                                         const int32_t* counts, WideResult* wide, int32_t max_leaf) {
    __shared__ unsigned s_cnt[3][kBuckets];
    __shared__ unsigned long long s_key[3][kBuckets][6];
    __shared__ float s_box[12];
    const WideChunk ch = chunks[blockIdx.x];
    const int tid = threadIdx.x;
    WideResult& w = wide[ch.slot];
    if (tid < 12) {
        const unsigned long long v = w.keys[tid];
        const int ax = (tid % 6) / 2;
        const bool is_min = tid % 2 == 0;
        const DevRef e = refs[is_min ? MinPos(v) : MaxPos(v)];
        s_box[tid] = tid < 6 ? Comp(is_min ? e.lo : e.hi, ax) : Comp(e.c, ax);
    }
    for (int j = tid; j < 3 * kBuckets; j += kBlock) {
        (&s_cnt[0][0])[j] = 0u;
        for (int q = 0; q < 6; ++q) (&s_key[0][0][0])[j * 6 + q] = q < 3 ? kMinEmpty : kMaxEmpty;
    }
    __syncthreads();
    FBox node;
    float clo[3], cext[3];
    for (int ax = 0; ax < 3; ++ax) {
        node.lo[ax] = s_box[2 * ax];
        node.hi[ax] = s_box[2 * ax + 1];
        clo[ax] = s_box[6 + 2 * ax];
        cext[ax] = __fsub_rn(s_box[7 + 2 * ax], s_box[6 + 2 * ax]);
    }
    if (counts[ch.slot] <= max_leaf || !(HalfArea2(node) > 0.0f)) return;  // uniform over the block
    for (int i = ch.begin + tid; i < ch.end; i += kBlock) {
        const DevRef e = refs[i];
        const uint32_t p = static_cast<uint32_t>(i);
        for (int ax = 0; ax < 3; ++ax) {
            if (cext[ax] < kDegenerateExtent) continue;
            const int b = BucketOf(Comp(e.c, ax), clo[ax], cext[ax]);
            atomicAdd(&s_cnt[ax][b], 1u);
            unsigned long long* key = s_key[ax][b];
            for (int q = 0; q < 3; ++q) {
                atomicMin(key + q, MinKey(Comp(e.lo, q), p));
                atomicMax(key + 3 + q, MaxKey(Comp(e.hi, q), p));
            }
        }
    }
    __syncthreads();
    for (int j = tid; j < 3 * kBuckets; j += kBlock) {
        const unsigned c = (&s_cnt[0][0])[j];
        if (c == 0) continue;
        atomicAdd(&w.cnt[0][0] + j, c);
        for (int q = 0; q < 6; ++q) {
            const unsigned long long v = (&s_key[0][0][0])[j * 6 + q];
            if (q < 3) atomicMin(&w.bins[0][0][0] + j * 6 + q, v);
            else atomicMax(&w.bins[0][0][0] + j * 6 + q, v);
        }
    }
}

// Triangle and sphere refs with the reference's float expressions
// (bvh_builder.cpp:144-238): box = Union(Union({p0, p0}, p1), p2), centroid
// ((p0 + p1) + p2) * (1 / 3), sphere box center -/+ radius. Invalid or
// non-finite input raises kFlagNonFinite (the host then reports the
// reference's error).
struct RefArgs {
    const char* positions;
    int64_t stride;
    int64_t vertex_count;
    const uint32_t* indices;
    const uint32_t* prim_first;  // per mesh primitive
    const int32_t* tri_base;     // per mesh primitive: its first flat triangle; [prims] = total
    int32_t prim_count;
    int64_t triangles;
    const yrc_sphere* spheres;
    int32_t sphere_count;
    DevRef* refs;
    yrc_bvh_primitive* prims;
    int* flags;
};

__device__ __forceinline__ float3 Vertex(const RefArgs& a, uint32_t i) {
    const float* p = reinterpret_cast<const float*>(a.positions + static_cast<int64_t>(i) * a.stride);
    return make_float3(p[0], p[1], p[2]);
}

__global__ void RefKernel(RefArgs a) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k < a.triangles) {
        int lo = 0, hi = a.prim_count - 1;  // last primitive whose base <= k
        while (lo < hi) {
            const int m = (lo + hi + 1) >> 1;
            if (a.tri_base[m] <= k) lo = m;
            else hi = m - 1;
        }
        const int32_t t = static_cast<int32_t>(k - a.tri_base[lo]);
        const uint64_t o = a.prim_first[lo] + static_cast<uint64_t>(t) * 3;
        const uint32_t i0 = a.indices[o], i1 = a.indices[o + 1], i2 = a.indices[o + 2];
        const uint64_t nv = static_cast<uint64_t>(a.vertex_count);
        if (i0 >= nv || i1 >= nv || i2 >= nv) {
            atomicOr(a.flags, kFlagNonFinite);
            return;
        }
        const float3 p0 = Vertex(a, i0), p1 = Vertex(a, i1), p2 = Vertex(a, i2);
        const float third = 1.0f / 3.0f;
        const float4 lo4 = make_float4(MinKeep(MinKeep(p0.x, p1.x), p2.x), MinKeep(MinKeep(p0.y, p1.y), p2.y),
                                       MinKeep(MinKeep(p0.z, p1.z), p2.z), __int_as_float(static_cast<int>(k)));
        const float4 hi4 = make_float4(MaxKeep(MaxKeep(p0.x, p1.x), p2.x), MaxKeep(MaxKeep(p0.y, p1.y), p2.y),
                                       MaxKeep(MaxKeep(p0.z, p1.z), p2.z), 0.0f);
        const float4 c4 = make_float4(__fmul_rn(__fadd_rn(__fadd_rn(p0.x, p1.x), p2.x), third),
                                      __fmul_rn(__fadd_rn(__fadd_rn(p0.y, p1.y), p2.y), third),
                                      __fmul_rn(__fadd_rn(__fadd_rn(p0.z, p1.z), p2.z), third), 0.0f);
        if (!(isfinite(lo4.x) && isfinite(lo4.y) && isfinite(lo4.z) && isfinite(hi4.x) && isfinite(hi4.y) &&
              isfinite(hi4.z) && isfinite(c4.x) && isfinite(c4.y) && isfinite(c4.z))) {
            atomicOr(a.flags, kFlagNonFinite);
            return;
        }
        a.refs[k] = DevRef{lo4, hi4, c4};
        a.prims[k] = yrc_bvh_primitive{0, lo, -1, t, static_cast<int32_t>(k)};
    } else if (k < a.triangles + a.sphere_count) {
        const int32_t s = static_cast<int32_t>(k - a.triangles);
        const yrc_sphere sp = a.spheres[s];
        const float r = sp.radius;
        const float4 lo4 = make_float4(__fsub_rn(sp.center[0], r), __fsub_rn(sp.center[1], r),
                                       __fsub_rn(sp.center[2], r), __int_as_float(static_cast<int>(k)));
        const float4 hi4 = make_float4(__fadd_rn(sp.center[0], r), __fadd_rn(sp.center[1], r),
                                       __fadd_rn(sp.center[2], r), 0.0f);
        const float4 c4 = make_float4(sp.center[0], sp.center[1], sp.center[2], 0.0f);
        if (!(r > 0.0f) || !(isfinite(lo4.x) && isfinite(lo4.y) && isfinite(lo4.z) && isfinite(hi4.x) &&
                             isfinite(hi4.y) && isfinite(hi4.z) && isfinite(c4.x) && isfinite(c4.y) && isfinite(c4.z))) {
            atomicOr(a.flags, kFlagNonFinite);
            return;
        }
        a.refs[k] = DevRef{lo4, hi4, c4};
        a.prims[k] = yrc_bvh_primitive{1, -1, s, -1, -1};
    }
}

__global__ void WideInitKernel(WideResult* wide, int count) {
    const int w = blockIdx.x;
    if (w >= count) return;
    for (int j = threadIdx.x; j < 12; j += blockDim.x) wide[w].keys[j] = (j % 2 == 0) ? kMinEmpty : kMaxEmpty;
    for (int j = threadIdx.x; j < 3 * kBuckets; j += blockDim.x) {
        (&wide[w].cnt[0][0])[j] = 0u;
        for (int q = 0; q < 6; ++q) (&wide[w].bins[0][0][0])[j * 6 + q] = q < 3 ? kMinEmpty : kMaxEmpty;
    }
}

struct SmallArgs {
    DevRef* refs;
    const SmallTask* tasks;
    int32_t count;
    yrc_bvh_node* local;  // subtree nodes at [2 * begin, 2 * begin + 2 * count - 1), local indices
    int32_t* size;        // nodes per subtree
    int32_t max_leaf;
    int* max_depth;
    int* flags;
    int32_t* host;  // per task: 1 when the host builds it (a median split)
};

// One thread builds the whole subtree of a range of at most kSmall refs, in
// the reference's serial order; node payloads are local (interior: right
// child's local index) or global (leaf: first slot = range begin).
__global__ void SmallKernel(SmallArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.count) return;
    const SmallTask task = a.tasks[t];
    DevRef* refs = a.refs;
    yrc_bvh_node* out = a.local + 2 * static_cast<int64_t>(task.begin);
    struct Entry {
        int16_t begin, end;  // relative to task.begin
        int16_t depth_off, parent;  // parent < 0: none; else local index whose right child this is
    };
    Entry stack[kMaxSmallDepth + 2];
    int sp = 0;
    stack[sp++] = Entry{0, static_cast<int16_t>(task.count), 0, -1};
    int next = 0, deepest = 0;
    while (sp > 0) {
        const Entry en = stack[--sp];
        const int b = task.begin + en.begin, e = task.begin + en.end, n = e - b;
        const int idx = next++;
        if (en.parent >= 0) out[en.parent].payload_offset = idx;
        const int depth = task.depth + en.depth_off;
        deepest = depth > deepest ? depth : deepest;
        FBox node, cen;
        Empty(node);
        Empty(cen);
        for (int i = b; i < e; ++i) {
            const DevRef r = refs[i];
            for (int ax = 0; ax < 3; ++ax) {
                node.lo[ax] = MinKeep(node.lo[ax], Comp(r.lo, ax));
                node.hi[ax] = MaxKeep(node.hi[ax], Comp(r.hi, ax));
                cen.lo[ax] = MinKeep(cen.lo[ax], Comp(r.c, ax));
                cen.hi[ax] = MaxKeep(cen.hi[ax], Comp(r.c, ax));
            }
        }
        yrc_bvh_node& self = out[idx];
        for (int ax = 0; ax < 3; ++ax) {
            self.bounds_min[ax] = node.lo[ax];
            self.bounds_max[ax] = node.hi[ax];
        }
        bool leaf = n <= a.max_leaf;
        int axis = -1, split = -1;
        float cext[3];
        for (int ax = 0; ax < 3; ++ax) cext[ax] = __fsub_rn(cen.hi[ax], cen.lo[ax]);
        if (!leaf) {
            int counts[3 * kBuckets];
            FBox boxes[3 * kBuckets];
            for (int j = 0; j < 3 * kBuckets; ++j) {
                counts[j] = 0;
                Empty(boxes[j]);
            }
            if (HalfArea2(node) > 0.0f) {
                for (int ax = 0; ax < 3; ++ax) {
                    if (cext[ax] < kDegenerateExtent) continue;
                    for (int i = b; i < e; ++i) {
                        const DevRef r = refs[i];
                        const int bk = ax * kBuckets + BucketOf(Comp(r.c, ax), cen.lo[ax], cext[ax]);
                        ++counts[bk];
                        FBox rb;
                        for (int q = 0; q < 3; ++q) {
                            rb.lo[q] = Comp(r.lo, q);
                            rb.hi[q] = Comp(r.hi, q);
                        }
                        MergeInto(boxes[bk], rb);
                    }
                }
            }
            float best_cost;
            const bool found = BestSplit(counts, boxes, node, cext, axis, split, best_cost);
            if (found && best_cost >= __int2float_rn(n)) {
                leaf = true;
            } else if (!found) {
                // A median split (std::nth_element): the host builds this
                // whole subtree with its serial builder. The partitions done
                // so far are kept; repeating a two-pointer partition on a
                // partitioned range moves nothing, so the host's build from
                // here equals a build from the start.
                a.host[t] = 1;
                atomicOr(a.flags, kFlagHostSubtree);
                a.size[t] = 0;
                return;
            }
        }
        if (leaf) {
            self.payload_offset = b;
            self.primitive_count = n;
            continue;
        }
        // Two-pointer partition (the reference's std::partition).
        const float lo = cen.lo[axis], extent = cext[axis];
        int first = b, last = e;
        for (;;) {
            while (first != last && BucketOf(Comp(refs[first].c, axis), lo, extent) <= split) ++first;
            if (first == last) break;
            --last;
            while (first != last && !(BucketOf(Comp(refs[last].c, axis), lo, extent) <= split)) --last;
            if (first == last) break;
            const DevRef x = refs[first];
            refs[first] = refs[last];
            refs[last] = x;
            ++first;
        }
        const int mid = first;
        if (mid == b || mid == e) {  // cannot happen when the SAH found both sides non-empty
            a.host[t] = 1;
            atomicOr(a.flags, kFlagHostSubtree);
            a.size[t] = 0;
            return;
        }
        self.primitive_count = 0;
        self.payload_offset = -1;
        if (sp + 2 > kMaxSmallDepth + 2) {
            atomicOr(a.flags, kFlagEmpty);
            break;
        }
        // Right pushed first so that the left subtree follows the node.
        stack[sp++] = Entry{static_cast<int16_t>(mid - task.begin), en.end, static_cast<int16_t>(en.depth_off + 1),
                            static_cast<int16_t>(idx)};
        stack[sp++] = Entry{en.begin, static_cast<int16_t>(mid - task.begin), static_cast<int16_t>(en.depth_off + 1),
                            -1};
    }
    a.size[t] = next;
    atomicMax(a.max_depth, deepest);
}

// Subtree sizes of one level of big nodes (children done).
__global__ void SizeKernel(const BigNode* big, int lo, int hi, const int32_t* small_size, int32_t* size) {
    const int id = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= hi) return;
    const BigNode& n = big[id];
    if (n.leaf) {
        size[id] = 1;
        return;
    }
    const int l = n.left >= 0 ? size[n.left] : small_size[-1 - n.left];
    const int r = n.right >= 0 ? size[n.right] : small_size[-1 - n.right];
    size[id] = 1 + l + r;
}

// Pre-order indices of the children of one level of big nodes.
__global__ void IndexKernel(const BigNode* big, int lo, int hi, const int32_t* size, const int32_t* small_size,
                            int32_t* index, int32_t* small_index) {
    const int id = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= hi) return;
    const BigNode& n = big[id];
    if (n.leaf) return;
    const int me = index[id];
    const int left_size = n.left >= 0 ? size[n.left] : small_size[-1 - n.left];
    if (n.left >= 0) index[n.left] = me + 1;
    else small_index[-1 - n.left] = me + 1;
    if (n.right >= 0) index[n.right] = me + 1 + left_size;
    else small_index[-1 - n.right] = me + 1 + left_size;
}

__global__ void WriteBigKernel(const BigNode* big, int count, const int32_t* index, const int32_t* small_index,
                               yrc_bvh_node* nodes, int total, int* max_depth, int* flags) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= count) return;
    if (index[id] < 0 || index[id] >= total) {
        atomicOr(flags, kFlagEmpty);
        return;
    }
    const BigNode& n = big[id];
    yrc_bvh_node o;
    for (int ax = 0; ax < 3; ++ax) {
        o.bounds_min[ax] = n.lo[ax];
        o.bounds_max[ax] = n.hi[ax];
    }
    if (n.leaf) {
        o.payload_offset = n.begin;
        o.primitive_count = n.count;
    } else {
        o.payload_offset = n.right >= 0 ? index[n.right] : small_index[-1 - n.right];
        o.primitive_count = 0;
    }
    nodes[index[id]] = o;
    atomicMax(max_depth, n.depth);
}

__global__ void WriteSmallKernel(const SmallTask* tasks, int count, const yrc_bvh_node* local, const int32_t* size,
                                 const int32_t* small_index, yrc_bvh_node* nodes, int total, int* flags) {
    const int t = blockIdx.x;
    if (t >= count) return;
    const SmallTask task = tasks[t];
    const int root = small_index[t];
    if (root < 0 || root + size[t] > total) {
        if (threadIdx.x == 0) atomicOr(flags, kFlagEmpty);
        return;
    }
    const yrc_bvh_node* src = local + 2 * static_cast<int64_t>(task.begin);
    for (int k = threadIdx.x; k < size[t]; k += blockDim.x) {
        yrc_bvh_node o = src[k];
        if (o.primitive_count == 0) o.payload_offset += root;
        nodes[root + k] = o;
    }
}

__global__ void SlotsKernel(const DevRef* refs, int64_t n, int32_t* slots) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i < n) slots[i] = __float_as_int(refs[i].lo.w);
}

unsigned Grid(int64_t n, int block) { return static_cast<unsigned>(std::max<int64_t>(1, (n + block - 1) / block)); }

// Device buffers of one build, freed together.
struct Buffers {
    std::vector<void*> ptrs;
    cudaError_t err = cudaSuccess;
    template <typename T>
    T* Alloc(int64_t n) {
        void* p = nullptr;
        if (err == cudaSuccess) err = cudaMalloc(&p, static_cast<size_t>(std::max<int64_t>(n, 1)) * sizeof(T));
        if (err == cudaSuccess) ptrs.push_back(p);
        return static_cast<T*>(p);
    }
    ~Buffers() {
        for (void* p : ptrs) cudaFree(p);
    }
};

}  // namespace

namespace {

// The hierarchy over n refs already in `d_refs` (reordered in place).
DevRef ToDevRef(const BuildRef& r) {
    float flat;
    std::memcpy(&flat, &r.flat_index, sizeof(flat));
    return DevRef{make_float4(r.bounds.lo.x, r.bounds.lo.y, r.bounds.lo.z, flat),
                  make_float4(r.bounds.hi.x, r.bounds.hi.y, r.bounds.hi.z, 0.0f),
                  make_float4(r.centroid.x, r.centroid.y, r.centroid.z, 0.0f)};
}

BuildRef ToBuildRef(const DevRef& d) {
    BuildRef r;
    std::memcpy(&r.flat_index, &d.lo.w, sizeof(r.flat_index));
    r.bounds.lo = Vec3{d.lo.x, d.lo.y, d.lo.z};
    r.bounds.hi = Vec3{d.hi.x, d.hi.y, d.hi.z};
    r.centroid = Vec3{d.c.x, d.c.y, d.c.z};
    return r;
}

// Copies device refs [begin, end) to the host as BuildRefs.
cudaError_t DownloadRefs(const DevRef* d_refs, int64_t begin, int64_t end, std::vector<BuildRef>& out) {
    std::vector<DevRef> dev(static_cast<size_t>(end - begin));
    const cudaError_t err = cudaMemcpy(dev.data(), d_refs + begin, sizeof(DevRef) * dev.size(), cudaMemcpyDeviceToHost);
    out.resize(dev.size());
    for (size_t i = 0; i < dev.size(); ++i) out[i] = ToBuildRef(dev[i]);
    return err;
}

cudaError_t UploadRefs(DevRef* d_refs, int64_t begin, const std::vector<BuildRef>& refs) {
    std::vector<DevRef> dev(refs.size());
    for (size_t i = 0; i < refs.size(); ++i) dev[i] = ToDevRef(refs[i]);
    return cudaMemcpy(d_refs + begin, dev.data(), sizeof(DevRef) * dev.size(), cudaMemcpyHostToDevice);
}

int BuildOnDevice(Buffers& B, DevRef* d_refs, int64_t n, const yrc_bvh_options& options, HostBvh& bvh,
                  std::string& error) {
    int32_t* d_tmp = B.Alloc<int32_t>(n);
    // Big nodes: each covers more than kSmall refs; the bound below is far
    // above what SAH trees use, and a build that would exceed it goes to the
    // host builder.
    const int64_t big_cap = std::min<int64_t>(2 * n, 2 * (n / kSmall + 1) * 40 + 64);
    BigNode* d_big = B.Alloc<BigNode>(big_cap);
    Range* d_ranges[2] = {B.Alloc<Range>(big_cap), B.Alloc<Range>(big_cap)};
    SmallTask* d_small = B.Alloc<SmallTask>(n);
    yrc_bvh_node* d_local = B.Alloc<yrc_bvh_node>(2 * n);
    int32_t* d_small_size = B.Alloc<int32_t>(n);
    int32_t* d_small_index = B.Alloc<int32_t>(n);
    int32_t* d_size = B.Alloc<int32_t>(big_cap);
    int32_t* d_index = B.Alloc<int32_t>(big_cap);
    unsigned* d_counts = B.Alloc<unsigned>(4);  // next ranges, big nodes, small tasks
    constexpr int kMaxWideRanges = 256;
    WideResult* d_wide = B.Alloc<WideResult>(kMaxWideRanges);
    int32_t* d_wide_of = B.Alloc<int32_t>(kMaxWideRanges);
    int32_t* d_wide_count = B.Alloc<int32_t>(kMaxWideRanges);
    const int64_t max_chunks = n / kChunk + kMaxWideRanges + 1;
    WideChunk* d_chunks = B.Alloc<WideChunk>(max_chunks);
    int* d_flags = B.Alloc<int>(2);             // flags, max depth
    int2* d_median = B.Alloc<int2>(big_cap);     // median ranges of a level
    int32_t* d_small_host = B.Alloc<int32_t>(n);  // per small task: built by the host
    if (B.err != cudaSuccess) {
        error = std::string("device BVH build: ") + cudaGetErrorString(B.err);
        return -1;
    }
    cudaError_t err = cudaSuccess;
    const int max_leaf = options.max_leaf_triangles;
    // Root: a big range (id 0), or a single small subtree.
    unsigned counts[4] = {0, 0, 0, 0};  // next ranges, big nodes, small tasks, median ranges
    std::vector<int> level_lo, level_hi;
    if (err == cudaSuccess) err = cudaMemset(d_flags, 0, 2 * sizeof(int));
    if (n > kSmall) {
        const Range root{0, static_cast<int32_t>(n), 1, 0};
        counts[0] = 0;
        counts[1] = 1;
        counts[2] = 0;
        if (err == cudaSuccess) err = cudaMemcpy(d_ranges[0], &root, sizeof(Range), cudaMemcpyHostToDevice);
        int ranges = 1, cur = 0, lo = 0;
        while (err == cudaSuccess && ranges > 0) {
            if (counts[1] + 2 * static_cast<int64_t>(ranges) > big_cap) return 0;  // very unbalanced: the host builder
            const unsigned zero = 0;
            err = cudaMemcpy(d_counts, &zero, sizeof(unsigned), cudaMemcpyHostToDevice);
            if (err == cudaSuccess) err = cudaMemcpy(d_counts + 1, counts + 1, 2 * sizeof(unsigned), cudaMemcpyHostToDevice);
            // Ranges larger than kWide (only in the top levels): bounds and
            // buckets reduced by one block per chunk first.
            bool use_wide = false;
            if (ranges <= kMaxWideRanges) {
                std::vector<Range> hr(static_cast<size_t>(ranges));
                err = cudaMemcpy(hr.data(), d_ranges[cur], sizeof(Range) * ranges, cudaMemcpyDeviceToHost);
                std::vector<int32_t> wide_of(static_cast<size_t>(ranges), -1), wide_count;
                std::vector<WideChunk> chunks;
                for (int q = 0; q < ranges && err == cudaSuccess; ++q) {
                    const Range& h = hr[static_cast<size_t>(q)];
                    if (h.end - h.begin <= kWide) continue;
                    const int slot = static_cast<int>(wide_count.size());
                    wide_of[static_cast<size_t>(q)] = slot;
                    wide_count.push_back(h.end - h.begin);
                    for (int b = h.begin; b < h.end; b += kChunk) chunks.push_back(WideChunk{b, std::min(h.end, b + kChunk), slot, 0});
                }
                if (!wide_count.empty() && err == cudaSuccess && static_cast<int64_t>(chunks.size()) <= max_chunks) {
                    use_wide = true;
                    const int nw = static_cast<int>(wide_count.size());
                    const unsigned nc = static_cast<unsigned>(chunks.size());
                    err = cudaMemcpy(d_wide_of, wide_of.data(), sizeof(int32_t) * ranges, cudaMemcpyHostToDevice);
                    if (err == cudaSuccess) err = cudaMemcpy(d_wide_count, wide_count.data(), sizeof(int32_t) * nw, cudaMemcpyHostToDevice);
                    if (err == cudaSuccess) err = cudaMemcpy(d_chunks, chunks.data(), sizeof(WideChunk) * nc, cudaMemcpyHostToDevice);
                    if (err == cudaSuccess) {
                        WideInitKernel<<<static_cast<unsigned>(nw), 64>>>(d_wide, nw);
                        WideBoundsKernel<<<nc, kBlock>>>(d_refs, d_chunks, d_wide);
                        WideBinsKernel<<<nc, kBlock>>>(d_refs, d_chunks, d_wide_count, d_wide, max_leaf);
                        err = cudaGetLastError();
                    }
                }
            }
            if (err == cudaSuccess) err = cudaMemcpy(d_counts + 3, &zero, sizeof(unsigned), cudaMemcpyHostToDevice);
            LevelArgs a{d_refs, d_tmp, d_ranges[cur], ranges, d_ranges[cur ^ 1], d_counts, d_big, d_counts + 1,
                        d_small, d_counts + 2, max_leaf, d_flags, use_wide ? d_wide_of : nullptr, d_wide,
                        d_median, d_counts + 3};
            if (err == cudaSuccess) {
                LevelKernel<<<static_cast<unsigned>(ranges), kBlock>>>(a);
                err = cudaGetLastError();
            }
            if (err == cudaSuccess) err = cudaMemcpy(counts, d_counts, 4 * sizeof(unsigned), cudaMemcpyDeviceToHost);
            // Median splits of this level (degenerate ranges): the host's
            // std::nth_element permutes each range before its children run.
            if (err == cudaSuccess && counts[3] > 0) {
                std::vector<int2> med(counts[3]);
                err = cudaMemcpy(med.data(), d_median, sizeof(int2) * med.size(), cudaMemcpyDeviceToHost);
                std::vector<BuildRef> range;
                for (size_t q = 0; q < med.size() && err == cudaSuccess; ++q) {
                    err = DownloadRefs(d_refs, med[q].x, med[q].y, range);
                    if (err != cudaSuccess) break;
                    MedianPartitionRange(range);
                    err = UploadRefs(d_refs, med[q].x, range);
                }
            }
            level_lo.push_back(lo);
            level_hi.push_back(lo + ranges);
            lo += ranges;
            ranges = static_cast<int>(counts[0]);
            cur ^= 1;
        }
    } else {
        const SmallTask only{0, static_cast<int32_t>(n), 1, 0};
        counts[2] = 1;
        if (err == cudaSuccess) err = cudaMemcpy(d_small, &only, sizeof(SmallTask), cudaMemcpyHostToDevice);
    }
    const int big_total = static_cast<int>(counts[1]);
    const int small_total = static_cast<int>(counts[2]);
    if (err == cudaSuccess && small_total > 0) {
        err = cudaMemset(d_small_host, 0, sizeof(int32_t) * small_total);
        SmallArgs s{d_refs, d_small, small_total, d_local, d_small_size, max_leaf, d_flags + 1, d_flags, d_small_host};
        if (err == cudaSuccess) {
            SmallKernel<<<Grid(small_total, 128), 128>>>(s);
            err = cudaGetLastError();
        }
    }
    int flags[2] = {0, 0};
    if (err == cudaSuccess) err = cudaMemcpy(flags, d_flags, 2 * sizeof(int), cudaMemcpyDeviceToHost);
    int32_t host_depth = 0;
    if (err == cudaSuccess && (flags[0] & kFlagHostSubtree)) {
        // Subtrees that met a median split: the host's serial builder, from
        // the refs as the device left them, into the task's local node slots.
        std::vector<SmallTask> tasks(static_cast<size_t>(small_total));
        std::vector<int32_t> host(static_cast<size_t>(small_total));
        err = cudaMemcpy(tasks.data(), d_small, sizeof(SmallTask) * tasks.size(), cudaMemcpyDeviceToHost);
        if (err == cudaSuccess) err = cudaMemcpy(host.data(), d_small_host, sizeof(int32_t) * host.size(), cudaMemcpyDeviceToHost);
        std::vector<BuildRef> range;
        std::vector<yrc_bvh_node> nodes;
        for (int t = 0; t < small_total && err == cudaSuccess; ++t) {
            if (!host[static_cast<size_t>(t)]) continue;
            const SmallTask& task = tasks[static_cast<size_t>(t)];
            err = DownloadRefs(d_refs, task.begin, task.begin + task.count, range);
            int32_t depth = 0;
            if (err == cudaSuccess && !BuildSubtreeHost(range, options, task.depth, nodes, depth, error)) return -1;
            for (yrc_bvh_node& node : nodes) {
                if (node.primitive_count > 0) node.payload_offset += task.begin;  // leaf: global first slot
            }
            if (err == cudaSuccess) err = UploadRefs(d_refs, task.begin, range);
            if (err == cudaSuccess) {
                err = cudaMemcpy(d_local + 2 * static_cast<int64_t>(task.begin), nodes.data(),
                                 sizeof(yrc_bvh_node) * nodes.size(), cudaMemcpyHostToDevice);
            }
            const int32_t size = static_cast<int32_t>(nodes.size());
            if (err == cudaSuccess) err = cudaMemcpy(d_small_size + t, &size, sizeof(int32_t), cudaMemcpyHostToDevice);
            host_depth = std::max(host_depth, depth);
        }
        flags[0] &= ~kFlagHostSubtree;
    }
    if (err != cudaSuccess) {
        error = std::string("device BVH build: ") + cudaGetErrorString(err);
        return -1;
    }
    if (flags[0] != 0) {
        error = "device BVH build: subtree stack exhausted";
        return -1;
    }
    if (err == cudaSuccess) err = cudaMemset(d_index, 0xff, sizeof(int32_t) * big_cap);
    if (err == cudaSuccess) err = cudaMemset(d_small_index, 0xff, sizeof(int32_t) * n);
    // Sizes bottom-up, indices top-down.
    for (int L = static_cast<int>(level_lo.size()) - 1; L >= 0 && err == cudaSuccess; --L) {
        SizeKernel<<<Grid(level_hi[L] - level_lo[L], 256), 256>>>(d_big, level_lo[L], level_hi[L], d_small_size, d_size);
        err = cudaGetLastError();
    }
    int32_t total = 0;
    if (big_total > 0) {
        const int32_t zero = 0;
        if (err == cudaSuccess) err = cudaMemcpy(d_index, &zero, sizeof(int32_t), cudaMemcpyHostToDevice);
        for (size_t L = 0; L < level_lo.size() && err == cudaSuccess; ++L) {
            IndexKernel<<<Grid(level_hi[L] - level_lo[L], 256), 256>>>(d_big, level_lo[L], level_hi[L], d_size,
                                                                        d_small_size, d_index, d_small_index);
            err = cudaGetLastError();
        }
        if (err == cudaSuccess) err = cudaMemcpy(&total, d_size, sizeof(int32_t), cudaMemcpyDeviceToHost);
    } else {
        const int32_t zero = 0;
        if (err == cudaSuccess) err = cudaMemcpy(d_small_index, &zero, sizeof(int32_t), cudaMemcpyHostToDevice);
        if (err == cudaSuccess) err = cudaMemcpy(&total, d_small_size, sizeof(int32_t), cudaMemcpyDeviceToHost);
    }
    yrc_bvh_node* d_nodes = B.Alloc<yrc_bvh_node>(total);
    int32_t* d_slots = B.Alloc<int32_t>(n);
    if (B.err != cudaSuccess) err = B.err;
    if (err == cudaSuccess && big_total > 0) {
        WriteBigKernel<<<Grid(big_total, 256), 256>>>(d_big, big_total, d_index, d_small_index, d_nodes, total,
                                                      d_flags + 1, d_flags);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess && small_total > 0) {
        WriteSmallKernel<<<static_cast<unsigned>(small_total), 32>>>(d_small, small_total, d_local, d_small_size,
                                                                    d_small_index, d_nodes, total, d_flags);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) {
        SlotsKernel<<<Grid(n, 256), 256>>>(d_refs, n, d_slots);
        err = cudaGetLastError();
    }
    bvh.nodes.resize(static_cast<size_t>(total));
    bvh.primitive_indices.resize(static_cast<size_t>(n));
    if (err == cudaSuccess) err = cudaMemcpy(bvh.nodes.data(), d_nodes, sizeof(yrc_bvh_node) * total, cudaMemcpyDeviceToHost);
    if (err == cudaSuccess) {
        err = cudaMemcpy(bvh.primitive_indices.data(), d_slots, sizeof(int32_t) * n, cudaMemcpyDeviceToHost);
    }
    if (err == cudaSuccess) err = cudaMemcpy(flags, d_flags, 2 * sizeof(int), cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) {
        error = std::string("device BVH build: ") + cudaGetErrorString(err);
        return -1;
    }
    if (flags[0] & ~kFlagHostSubtree) {
        error = "device BVH build: inconsistent node layout";
        return -1;
    }
    bvh.max_depth = std::max(flags[1], host_depth);
    return 1;
}

}  // namespace

int BuildHierarchyDevice(std::vector<BuildRef>& refs, const yrc_bvh_options& options, HostBvh& bvh,
                         std::string& error) {
    const int64_t n = static_cast<int64_t>(refs.size());
    if (n == 0) return 1;
    if (options.split_method != 0) return 0;  // median splits: the host builder
    if (n >= (int64_t{1} << 31) - 1) return 0;
    Buffers B;
    DevRef* d_refs = B.Alloc<DevRef>(n);
    if (B.err != cudaSuccess) {
        error = std::string("device BVH build: ") + cudaGetErrorString(B.err);
        return -1;
    }
    std::vector<DevRef> host(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) host[static_cast<size_t>(i)] = ToDevRef(refs[static_cast<size_t>(i)]);
    const cudaError_t err = cudaMemcpy(d_refs, host.data(), sizeof(DevRef) * n, cudaMemcpyHostToDevice);
    if (err != cudaSuccess) {
        error = std::string("device BVH build: ") + cudaGetErrorString(err);
        return -1;
    }
    return BuildOnDevice(B, d_refs, n, options, bvh, error);
}

int BuildFlatDevice(const yrc_geometry& g, const yrc_bvh_options& options, HostBvh& bvh, std::string& error) {
    if (options.split_method != 0) return 0;
    // Index ranges are checked on the host (as the reference does, per
    // primitive); per-triangle checks run on the device.
    std::vector<uint32_t> prim_first;
    std::vector<int32_t> tri_base;
    int64_t triangles = 0;
    for (int32_t p = 0; p < g.primitive_count; ++p) {
        const uint64_t first = g.primitives[p].first_index, count = g.primitives[p].index_count;
        const uint64_t total = static_cast<uint64_t>(g.index_count);
        if (first > total || count > total - first || count % 3 != 0) return 0;
        prim_first.push_back(g.primitives[p].first_index);
        tri_base.push_back(static_cast<int32_t>(triangles));
        triangles += static_cast<int64_t>(count / 3);
    }
    const int64_t n = triangles + g.sphere_count;
    if (n == 0 || n >= (int64_t{1} << 31) - 1) return 0;
    tri_base.push_back(static_cast<int32_t>(triangles));
    Buffers B;
    const int64_t pos_bytes = g.vertex_count > 0 ? (g.vertex_count - 1) * g.vertex_stride + 3 * sizeof(float) : 0;
    char* d_pos = B.Alloc<char>(pos_bytes);
    uint32_t* d_idx = B.Alloc<uint32_t>(g.index_count);
    uint32_t* d_first = B.Alloc<uint32_t>(static_cast<int64_t>(prim_first.size()));
    int32_t* d_base = B.Alloc<int32_t>(static_cast<int64_t>(tri_base.size()));
    yrc_sphere* d_spheres = B.Alloc<yrc_sphere>(g.sphere_count);
    DevRef* d_refs = B.Alloc<DevRef>(n);
    yrc_bvh_primitive* d_prims = B.Alloc<yrc_bvh_primitive>(n);
    int* d_flag = B.Alloc<int>(1);
    cudaError_t err = B.err;
    if (err == cudaSuccess && pos_bytes > 0) err = cudaMemcpy(d_pos, g.positions, pos_bytes, cudaMemcpyHostToDevice);
    if (err == cudaSuccess && g.index_count > 0) {
        err = cudaMemcpy(d_idx, g.indices, sizeof(uint32_t) * g.index_count, cudaMemcpyHostToDevice);
    }
    if (err == cudaSuccess && !prim_first.empty()) {
        err = cudaMemcpy(d_first, prim_first.data(), sizeof(uint32_t) * prim_first.size(), cudaMemcpyHostToDevice);
    }
    if (err == cudaSuccess) err = cudaMemcpy(d_base, tri_base.data(), sizeof(int32_t) * tri_base.size(), cudaMemcpyHostToDevice);
    if (err == cudaSuccess && g.sphere_count > 0) {
        err = cudaMemcpy(d_spheres, g.spheres, sizeof(yrc_sphere) * g.sphere_count, cudaMemcpyHostToDevice);
    }
    if (err == cudaSuccess) err = cudaMemset(d_flag, 0, sizeof(int));
    if (err == cudaSuccess) {
        RefArgs a{d_pos, g.vertex_stride, g.vertex_count, d_idx, d_first, d_base, g.primitive_count, triangles,
                  d_spheres, g.sphere_count, d_refs, d_prims, d_flag};
        RefKernel<<<Grid(n, 256), 256>>>(a);
        err = cudaGetLastError();
    }
    int flag = 0;
    if (err == cudaSuccess) err = cudaMemcpy(&flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) {
        error = std::string("device BVH build: ") + cudaGetErrorString(err);
        return -1;
    }
    if (flag) return 0;  // invalid geometry: the host build reports the reference's error
    const int r = BuildOnDevice(B, d_refs, n, options, bvh, error);
    if (r <= 0) return r;
    bvh.primitives.resize(static_cast<size_t>(n));
    err = cudaMemcpy(bvh.primitives.data(), d_prims, sizeof(yrc_bvh_primitive) * n, cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) {
        error = std::string("device BVH build: ") + cudaGetErrorString(err);
        return -1;
    }
    bvh.total_triangles = static_cast<int32_t>(triangles);
    bvh.total_spheres = g.sphere_count;
    return 1;
}

}  // namespace yrc
