// Ray reordering ahead of a traversal launch.
//
// Incoherent rays (origins anywhere in the scene, directions anywhere on the
// sphere) leave a warp's 32 lanes on 32 unrelated paths through the BVH: the
// lanes step through interior nodes and leaves out of phase and fetch
// unrelated nodes. Sorting the rays by a spatial key first puts rays that
// start close together and head the same way into the same warp, so they
// visit largely the same nodes in the same order.
//
// The key interleaves (Morton order) six quantised coordinates: the ray
// origin in the BVH's root box, and either the normalised direction in
// [-1, 1]^3 (kRayOrderDirection) or a second point a fixed distance along
// the ray (kRayOrderTwoPoint). Its top `bits` bits pick one of 2^bits bins,
// and a counting sort over the bins (histogram, exclusive scan, scatter)
// gives the permutation the traversal kernel reads its rays through. Rays
// within a bin keep no particular order; the traversal's results are per
// ray, so the order changes only which lanes share a warp, never a hit.
//
// Traffic per ray: 32 B ray read + 4 B key write + 4 B key read + 4 B index
// write, plus one histogram and one cursor atomic; the 2^bits counters stay
// in L2.
#include <cuda_runtime.h>

#include <cstdint>

#include "trace_kernels.hpp"

namespace yrc {
namespace {

constexpr int kOrderBlock = 256;
constexpr int kScanThreads = 1024;
constexpr int kScanPerThread = 4;
constexpr int kScanTile = kScanThreads * kScanPerThread;

struct RayKeyParams {
    float lo[3];
    float scale[3];    // quantisation levels per unit length along each axis
    float dir_scale;   // quantisation levels per unit of a direction component
    float length;      // distance to the second point (two-point keys)
    uint32_t levels;   // largest quantised value per coordinate
    int per_dim;       // bits per coordinate
    int shift;         // interleaved bits dropped at the bottom
    int mode;
};

__device__ __forceinline__ uint32_t Quantize(float v, float lo, float scale, uint32_t levels) {
    // fmaxf/fminf return the other operand for NaN, so a NaN coordinate
    // lands in bin 0 instead of an undefined conversion.
    const float q = fminf(fmaxf((v - lo) * scale, 0.0f), static_cast<float>(levels));
    return static_cast<uint32_t>(q);
}

// Adds each lane's 1 to counters[key]: lanes of a warp that share a key
// add their count once (coherent rays, e.g. from one camera, share bins);
// returns the counter's value before the lane's own increment.
__device__ __forceinline__ uint32_t WarpAtomicInc(uint32_t* counters, uint32_t key, unsigned valid) {
    const unsigned peers = __match_any_sync(valid, key);
    const int leader = __ffs(peers) - 1;
    const unsigned lane = threadIdx.x & 31u;
    uint32_t base = 0;
    if (static_cast<int>(lane) == leader) base = atomicAdd(counters + key, static_cast<uint32_t>(__popc(peers)));
    base = __shfl_sync(valid, base, leader);
    return base + static_cast<uint32_t>(__popc(peers & ((1u << lane) - 1u)));
}

__global__ void __launch_bounds__(kOrderBlock) RayKeyKernel(const float4* rays, int64_t count, RayKeyParams p,
                                                             uint32_t* keys, uint32_t* hist) {
    // Every lane of a warp runs the same iterations (uniform base), so the
    // warp-wide key matching sees the whole warp.
    for (int64_t base = blockIdx.x * static_cast<int64_t>(blockDim.x); base < count;
         base += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        const bool in = i < count;
        const unsigned valid = __ballot_sync(0xffffffffu, in);
        if (!in) continue;
        const float4 a = __ldg(rays + 2 * i);
        const float4 b = __ldg(rays + 2 * i + 1);
        const float len2 = b.x * b.x + b.y * b.y + b.z * b.z;
        const float inv = len2 > 0.0f ? rsqrtf(len2) : 0.0f;
        const float dx = b.x * inv, dy = b.y * inv, dz = b.z * inv;
        uint32_t q[6];
        q[0] = Quantize(a.x, p.lo[0], p.scale[0], p.levels);
        q[1] = Quantize(a.y, p.lo[1], p.scale[1], p.levels);
        q[2] = Quantize(a.z, p.lo[2], p.scale[2], p.levels);
        if (p.mode == kRayOrderDirection) {
            q[3] = Quantize(dx, -1.0f, p.dir_scale, p.levels);
            q[4] = Quantize(dy, -1.0f, p.dir_scale, p.levels);
            q[5] = Quantize(dz, -1.0f, p.dir_scale, p.levels);
        } else {
            q[3] = Quantize(a.x + dx * p.length, p.lo[0], p.scale[0], p.levels);
            q[4] = Quantize(a.y + dy * p.length, p.lo[1], p.scale[1], p.levels);
            q[5] = Quantize(a.z + dz * p.length, p.lo[2], p.scale[2], p.levels);
        }
        uint32_t key = 0;
        for (int bit = p.per_dim - 1; bit >= 0; --bit) {
#pragma unroll
            for (int k = 0; k < 6; ++k) key = (key << 1) | ((q[k] >> bit) & 1u);
        }
        key >>= p.shift;
        keys[i] = key;
        WarpAtomicInc(hist, key, valid);
    }
}

// Exclusive scan of v over the block (kScanThreads threads); *total gets
// the block's sum.
__device__ __forceinline__ uint32_t BlockExclusiveScan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warp_sums[kScanThreads / 32];
    const unsigned lane = threadIdx.x & 31u;
    const unsigned warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= static_cast<unsigned>(o)) x += y;
    }
    if (lane == 31u) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_sums[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= static_cast<unsigned>(o)) w += y;
        }
        warp_sums[lane] = w;
    }
    __syncthreads();
    const uint32_t prefix = warp ? warp_sums[warp - 1] : 0u;
    *total = warp_sums[kScanThreads / 32 - 1];
    return prefix + x - v;
}

// Sum of each kScanTile-counter tile.
__global__ void __launch_bounds__(kScanThreads) TileSumKernel(const uint32_t* counters, int64_t n,
                                                             uint32_t* tile_sums) {
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanTile;
    uint32_t s = 0;
    for (int k = threadIdx.x; k < kScanTile; k += kScanThreads) {
        const int64_t j = base + k;
        if (j < n) s += counters[j];
    }
    uint32_t total = 0;
    BlockExclusiveScan(s, &total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// In-place exclusive scan of one kScanTile tile per block, offset by the
// tile's entry in tile_offsets (already scanned), if given.
__global__ void __launch_bounds__(kScanThreads) TileScanKernel(uint32_t* counters, int64_t n,
                                                              const uint32_t* tile_offsets) {
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanTile + threadIdx.x * kScanPerThread;
    uint32_t v[kScanPerThread];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanPerThread; ++k) {
        v[k] = base + k < n ? counters[base + k] : 0u;
        s += v[k];
    }
    uint32_t total = 0;
    uint32_t run = BlockExclusiveScan(s, &total) + (tile_offsets ? tile_offsets[blockIdx.x] : 0u);
#pragma unroll
    for (int k = 0; k < kScanPerThread; ++k) {
        if (base + k < n) counters[base + k] = run;
        run += v[k];
    }
}

__global__ void __launch_bounds__(kOrderBlock) RayScatterKernel(const uint32_t* keys, int64_t count,
                                                                 uint32_t* offsets, uint32_t* order) {
    for (int64_t base = blockIdx.x * static_cast<int64_t>(blockDim.x); base < count;
         base += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        const bool in = i < count;
        const unsigned valid = __ballot_sync(0xffffffffu, in);
        if (!in) continue;
        const uint32_t pos = WarpAtomicInc(offsets, keys[i], valid);
        order[pos] = static_cast<uint32_t>(i);
    }
}

}  // namespace

int RayOrderBits(int64_t count, int requested) {
    if (requested > 0) return requested < kRayOrderMinBits ? kRayOrderMinBits
                              : requested > kRayOrderMaxBits ? kRayOrderMaxBits : requested;
    // About eight rays per bin.
    int lg = 0;
    while (lg < 62 && (int64_t{1} << (lg + 1)) <= count) ++lg;
    const int bits = lg - 3;
    return bits < kRayOrderMinBits ? kRayOrderMinBits : bits > kRayOrderMaxBits ? kRayOrderMaxBits : bits;
}

int64_t RayOrderTiles(int bits) { return ((int64_t{1} << bits) + kScanTile - 1) / kScanTile; }

cudaError_t OrderRays(const float4* rays, int64_t count, const AccelParams& accel, int mode, int bits, float length,
                      const RayOrderScratch& scratch, cudaStream_t stream, int sm_count) {
    const int64_t bins = int64_t{1} << bits;
    const int64_t tiles = RayOrderTiles(bits);
    if (tiles > kScanTile) return cudaErrorInvalidValue;  // one block scans the tile sums
    RayKeyParams p{};
    const int per_dim = (bits + 5) / 6;
    p.per_dim = per_dim;
    p.shift = 6 * per_dim - bits;
    p.levels = (1u << per_dim) - 1u;
    const float levels = static_cast<float>(1u << per_dim);
    float diag2 = 0.0f;
    for (int k = 0; k < 3; ++k) {
        const float extent = accel.root_hi[k] - accel.root_lo[k];
        p.lo[k] = accel.root_lo[k];
        p.scale[k] = extent > 0.0f ? levels / extent : 0.0f;
        diag2 += extent * extent;
    }
    p.dir_scale = levels * 0.5f;
    p.length = length * sqrtf(diag2);
    p.mode = mode;
    cudaError_t err = cudaMemsetAsync(scratch.hist, 0, static_cast<size_t>(bins) * sizeof(uint32_t), stream);
    if (err != cudaSuccess) return err;
    int64_t blocks = (count + kOrderBlock - 1) / kOrderBlock;
    const int64_t cap = static_cast<int64_t>(sm_count) * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    RayKeyKernel<<<static_cast<unsigned>(blocks), kOrderBlock, 0, stream>>>(rays, count, p, scratch.keys,
                                                                             scratch.hist);
    TileSumKernel<<<static_cast<unsigned>(tiles), kScanThreads, 0, stream>>>(scratch.hist, bins, scratch.tile_sums);
    TileScanKernel<<<1, kScanThreads, 0, stream>>>(scratch.tile_sums, tiles, nullptr);
    TileScanKernel<<<static_cast<unsigned>(tiles), kScanThreads, 0, stream>>>(scratch.hist, bins, scratch.tile_sums);
    RayScatterKernel<<<static_cast<unsigned>(blocks), kOrderBlock, 0, stream>>>(scratch.keys, count, scratch.hist,
                                                                                 scratch.order);
    return cudaGetLastError();
}

}  // namespace yrc
