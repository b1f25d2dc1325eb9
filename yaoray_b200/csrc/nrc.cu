// Neural radiance cache: a multiresolution hash-grid encoding of position
// plus spherical harmonics of the view direction and surface attributes,
// feeding a 64-wide, 5-hidden-layer ReLU MLP with an exp-activated RGB
// output; bf16 operands on the tcgen05 tensor cores with fp32 accumulation
// in TMEM; trained online with a relative-L2 loss and Adam.
//
// Kernels (one CTA of 128 threads per 128-row tile; persistent grids):
//   CacheInferKernel  encode + 6 forward GEMMs + exp           (inference)
//   CacheTrainKernel  encode + forward + loss + 6 x (dW, dX) backward GEMMs,
//                     weight gradients accumulated in TMEM across the CTA's
//                     tiles and flushed once, grid gradients scattered with
//                     float2 atomics, the touched entries listed once each
//   AdamKernel        fp32 master weights -> bf16 weights (all of them)
//   SparseGridAdamKernel  lazy Adam over the listed grid entries -> fp16 grid
//
// The reference renderer has no radiance cache; this file has no counterpart
// in it.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <random>
#include <string>
#include <vector>

#include "nrc.hpp"
#include "umma.cuh"
#include "yrc_internal.hpp"

namespace yrc {
namespace nrc {

constexpr int kLevels = 16;
constexpr int kLog2Table = 19;
constexpr int64_t kTable = int64_t(1) << kLog2Table;
constexpr int kWidth = 64;
constexpr int kLayers = 6;  // 5 hidden + output
constexpr int kTile = 128;
constexpr int kThreads = 128;
constexpr int kMatBytes = kTile * kWidth * 2;  // 128 rows x 64 bf16
constexpr int kWBytes = 64 * kWidth * 2;       // one 64 x 64 bf16 weight matrix
constexpr int kWeightCount = kLayers * 64 * kWidth;
constexpr int kQueryFloats = 16;
constexpr uint32_t kWaitTries = 1u << 24;
constexpr float kOClamp = 15.0f;
constexpr float kLossEps = 0.01f;
constexpr float kLr = 1.0e-2f;
constexpr double kBeta1 = 0.9, kBeta2 = 0.99;
constexpr float kAvgDecay = 0.99f;  // default decay of the parameter moving average
constexpr float kAdamEps = 1.0e-15f;
constexpr uint32_t kPrimeY = 2654435761u, kPrimeZ = 805459861u;

// Shared-memory plans (bytes from the dynamic shared memory base).
constexpr int kOffW = 0;                                   // 6 weight matrices
constexpr int kOffA = kOffW + kLayers * kWBytes;           // activations
constexpr int kInferSmem = kOffA + kMatBytes + 64;         // + barrier, TMEM slot
constexpr int kOffG = kOffA + kLayers * kMatBytes;         // training: gradient tile
// The dW GEMM reads its A operand (the gradient tile as MN-major, M = 128)
// up to 1 KB past the tile; the pad keeps even a transposed reading of the
// descriptor's two strides (13.6 KB past) inside this kernel's shared memory.
constexpr int kPadG = 14 * 1024;
constexpr int kOffBarTrain = kOffG + kMatBytes + kPadG;
constexpr int kTrainSmem = kOffBarTrain + 64;
constexpr uint32_t kTrainTmemCols = 512;  // [0, 64) activations / dX, [64 + 64 l, ...) dW_l
constexpr uint32_t kInferTmemCols = 64;

struct GridArgs {
    const __half2* table;  // [kLevels * kTable]
    float2* grad;          // same shape, training only
    // Training only: the entries this step's samples touched, as a bitmask
    // over [kLevels * kTable] and a compacted list (each entry once).
    uint32_t* touched;
    int32_t* touched_list;
    unsigned long long* touched_count;
    float scale[kLevels];
    int32_t side[kLevels];  // dense grid side, 0 when the level is hashed
    float lo[3];
    float inv;
};

// ------------------------------------------------------------ encoding

__device__ __forceinline__ void LevelCorners(const GridArgs& g, int l, const float p[3], uint32_t idx[8],
                                             float w[8]) {
    float f[3];
    int32_t b[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float x = __fmul_rn(p[k], g.scale[l]);
        const float fl = floorf(x);
        b[k] = static_cast<int32_t>(fl);
        f[k] = __fsub_rn(x, fl);
    }
    const int32_t side = g.side[l];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int32_t x = b[0] + (c & 1), y = b[1] + ((c >> 1) & 1), z = b[2] + ((c >> 2) & 1);
        if (side) {
            idx[c] = static_cast<uint32_t>(x + y * side + z * side * side);
        } else {
            idx[c] = (static_cast<uint32_t>(x) ^ (static_cast<uint32_t>(y) * kPrimeY) ^
                      (static_cast<uint32_t>(z) * kPrimeZ)) &
                     static_cast<uint32_t>(kTable - 1);
        }
        const float wx = (c & 1) ? f[0] : __fsub_rn(1.0f, f[0]);
        const float wy = ((c >> 1) & 1) ? f[1] : __fsub_rn(1.0f, f[1]);
        const float wz = ((c >> 2) & 1) ? f[2] : __fsub_rn(1.0f, f[2]);
        w[c] = __fmul_rn(__fmul_rn(wx, wy), wz);
    }
}

__device__ __forceinline__ void NormalisedPosition(const GridArgs& g, const float* q, float p[3]) {
#pragma unroll
    for (int k = 0; k < 3; ++k) p[k] = fminf(fmaxf(__fmul_rn(__fsub_rn(q[k], g.lo[k]), g.inv), 0.0f), 1.0f);
}

// The 64 network inputs of one query (see the query layout in yrcuda.h).
__device__ __forceinline__ void Encode(const GridArgs& g, const float* q, float x[kWidth]) {
    float p[3];
    NormalisedPosition(g, q, p);
#pragma unroll
    for (int l = 0; l < kLevels; ++l) {
        uint32_t idx[8];
        float w[8];
        LevelCorners(g, l, p, idx, w);
        float a0 = 0.0f, a1 = 0.0f;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const float2 v = __half22float2(g.table[static_cast<int64_t>(l) * kTable + idx[c]]);
            a0 = __fadd_rn(a0, __fmul_rn(v.x, w[c]));
            a1 = __fadd_rn(a1, __fmul_rn(v.y, w[c]));
        }
        x[2 * l] = a0;
        x[2 * l + 1] = a1;
    }
    // Real spherical harmonics, degrees 0-3, of the direction.
    const float dx = q[4], dy = q[5], dz = q[6];
    const float xx = dx * dx, yy = dy * dy, zz = dz * dz;
    x[32] = 0.28209479177387814f;
    x[33] = -0.48860251190291987f * dy;
    x[34] = 0.48860251190291987f * dz;
    x[35] = -0.48860251190291987f * dx;
    x[36] = 1.0925484305920792f * dx * dy;
    x[37] = -1.0925484305920792f * dy * dz;
    x[38] = 0.94617469575755997f * zz - 0.31539156525251999f;
    x[39] = -1.0925484305920792f * dx * dz;
    x[40] = 0.54627421529603959f * (xx - yy);
    x[41] = 0.59004358992664352f * dy * (-3.0f * xx + yy);
    x[42] = 2.8906114426405538f * dx * dy * dz;
    x[43] = 0.45704579946446572f * dy * (1.0f - 5.0f * zz);
    x[44] = 0.3731763325901154f * dz * (5.0f * zz - 3.0f);
    x[45] = 0.45704579946446572f * dx * (1.0f - 5.0f * zz);
    x[46] = 1.4453057213202769f * dz * (xx - yy);
    x[47] = 0.59004358992664352f * dx * (-xx + 3.0f * yy);
    x[48] = q[7] * 0.5f + 0.5f;
    x[49] = q[8] * 0.5f + 0.5f;
    x[50] = q[9] * 0.5f + 0.5f;
    x[51] = q[3];
    x[52] = q[10];
    x[53] = q[11];
    x[54] = q[12];
    x[55] = q[13];
    x[56] = q[14];
    x[57] = q[15];
    x[58] = 1.0f;
    x[59] = x[60] = x[61] = x[62] = x[63] = 0.0f;
}

// ------------------------------------------------------- smem row access

__device__ __forceinline__ uint32_t PackBf16(float a, float b) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// Row `r` of a 128 x 64 tile in the canonical layout, from 64 floats.
__device__ __forceinline__ void StoreRow(uint8_t* mat, int r, const float v[kWidth]) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        uint4 u;
        u.x = PackBf16(v[8 * c + 0], v[8 * c + 1]);
        u.y = PackBf16(v[8 * c + 2], v[8 * c + 3]);
        u.z = PackBf16(v[8 * c + 4], v[8 * c + 5]);
        u.w = PackBf16(v[8 * c + 6], v[8 * c + 7]);
        *reinterpret_cast<uint4*>(mat + umma::Canon64(r, 8 * c)) = u;
    }
}

// Columns 8c..8c+7 of row r as floats.
__device__ __forceinline__ void LoadChunk(const uint8_t* mat, int r, int c, float out[8]) {
    const uint4 u = *reinterpret_cast<const uint4*>(mat + umma::Canon64(r, 8 * c));
    const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w[k]));
        out[2 * k] = f.x;
        out[2 * k + 1] = f.y;
    }
}

// Copies the 6 bf16 weight matrices (row-major [out][in]) into shared memory.
__device__ __forceinline__ void LoadWeights(const __nv_bfloat16* w, uint8_t* smem_w) {
    for (int i = threadIdx.x; i < kLayers * 64 * 8; i += blockDim.x) {
        const int l = i / (64 * 8), rem = i % (64 * 8), r = rem / 8, c = rem % 8;
        const uint4 v = *reinterpret_cast<const uint4*>(w + static_cast<int64_t>(l) * 64 * kWidth + r * kWidth + 8 * c);
        *reinterpret_cast<uint4*>(smem_w + l * kWBytes + umma::Canon64(r, 8 * c)) = v;
    }
}

// 64 fp32 accumulator columns [col, col + 64) of this thread's TMEM lane.
__device__ __forceinline__ void LoadAcc64(uint32_t tmem, int col, float v[kWidth]) {
    const uint32_t base = tmem + ((static_cast<uint32_t>(threadIdx.x) & ~31u) << 16) + static_cast<uint32_t>(col);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float t[16];
        umma::Ld16(base + 16 * j, t);
#pragma unroll
        for (int k = 0; k < 16; ++k) v[16 * j + k] = t[k];
    }
    umma::WaitLd();
}

// Forward GEMM of layer l: D[128 x n] = A (128 x 64) * W_l^T, K = 64.
__device__ __forceinline__ void IssueForward(uint32_t tmem, uint32_t a, uint32_t w, int n) {
    const uint32_t id = umma::IDesc(128, n, false, false);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        umma::Mma(tmem, umma::Desc(a + 256 * k, 128, 1024), umma::Desc(w + 256 * k, 128, 1024), id, k > 0);
    }
}

// Waits for the tensor core; all threads agree on a timeout.
__device__ __forceinline__ bool Await(uint64_t* bar, uint32_t& phase, int* error) {
    const bool ok = umma::MbarWait(bar, phase, kWaitTries);
    phase ^= 1u;
    const bool any_fail = __syncthreads_or(!ok);
    if (any_fail) {
        if (threadIdx.x == 0) atomicOr(error, 1);
        return false;
    }
    umma::FenceAfterSync();
    return true;
}

// Makes this thread's shared-memory writes and TMEM reads visible before the
// next tensor-core instruction, then synchronises the CTA.
__device__ __forceinline__ void HandOff() {
    umma::FenceProxyAsync();
    umma::FenceBeforeSync();
    __syncthreads();
}

__device__ __forceinline__ float ExpOut(float o) { return expf(fminf(o, kOClamp)); }

// ----------------------------------------------------------- inference

__global__ void __launch_bounds__(kThreads) CacheInferKernel(GridArgs g, const __nv_bfloat16* weights,
                                                            const float* queries, int64_t n_max,
                                                            const unsigned long long* n_ptr, float4* out,
                                                            int* error) {
    // The query count: n_max, or min(*n_ptr, n_max) when it lives on the device.
    const int64_t n = n_ptr ? static_cast<int64_t>(min(*n_ptr, static_cast<unsigned long long>(n_max))) : n_max;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* sw = smem + kOffW;
    uint8_t* sa = smem + kOffA;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kOffA + kMatBytes);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kOffA + kMatBytes + 16);
    if (threadIdx.x < 32) umma::TmemAlloc(tmem_slot, kInferTmemCols);
    if (threadIdx.x == 0) umma::MbarInit(bar, 1);
    LoadWeights(weights, sw);
    umma::FenceBeforeSync();
    __syncthreads();
    umma::FenceAfterSync();
    const uint32_t tmem = *tmem_slot;
    const uint32_t a_addr = umma::SmemAddr(sa), w_addr = umma::SmemAddr(sw);
    uint32_t phase = 0;
    const int r = threadIdx.x;
    const int64_t tiles = (n + kTile - 1) / kTile;
    bool ok = true;
    for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        const int64_t row = t * kTile + r;
        float x[kWidth];
        if (row < n) {
            Encode(g, queries + row * kQueryFloats, x);
        } else {
#pragma unroll
            for (int k = 0; k < kWidth; ++k) x[k] = 0.0f;
        }
        StoreRow(sa, r, x);
        HandOff();
        for (int l = 0; l < kLayers && ok; ++l) {
            const int nn = l < kLayers - 1 ? 64 : 16;
            if (threadIdx.x == 0) {
                umma::FenceAfterSync();
                IssueForward(tmem, a_addr, w_addr + l * kWBytes, nn);
                umma::Commit(bar);
            }
            ok = Await(bar, phase, error);
            if (!ok) break;
            if (l < kLayers - 1) {
                float v[kWidth];
                LoadAcc64(tmem, 0, v);
#pragma unroll
                for (int k = 0; k < kWidth; ++k) v[k] = fmaxf(v[k], 0.0f);
                StoreRow(sa, r, v);  // in place: the GEMM that read the tile has completed
                HandOff();
            } else {
                float v[16];
                umma::Ld16(tmem + ((static_cast<uint32_t>(threadIdx.x) & ~31u) << 16), v);
                umma::WaitLd();
                if (row < n) out[row] = make_float4(ExpOut(v[0]), ExpOut(v[1]), ExpOut(v[2]), 0.0f);
                umma::FenceBeforeSync();
                __syncthreads();
            }
        }
    }
    umma::FenceBeforeSync();
    __syncthreads();
    if (threadIdx.x < 32) umma::TmemFree(tmem, kInferTmemCols);
}

// ------------------------------------------------------------ training

__global__ void __launch_bounds__(kThreads) CacheTrainKernel(GridArgs g, const __nv_bfloat16* weights,
                                                            float* weight_grad, const float* queries,
                                                            const float4* targets, int64_t n_max,
                                                            const unsigned long long* n_ptr, float* loss_sum,
                                                            int* error) {
    const int64_t n = n_ptr ? static_cast<int64_t>(min(*n_ptr, static_cast<unsigned long long>(n_max))) : n_max;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* sw = smem + kOffW;
    uint8_t* sa = smem + kOffA;  // a_0 .. a_5
    uint8_t* sg = smem + kOffG;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kOffBarTrain);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kOffBarTrain + 16);
    if (threadIdx.x < 32) umma::TmemAlloc(tmem_slot, kTrainTmemCols);
    if (threadIdx.x == 0) umma::MbarInit(bar, 1);
    LoadWeights(weights, sw);
    // The pad after the gradient tile is read (never used) by the dW GEMMs.
    for (int i = threadIdx.x; i < kPadG / 16; i += blockDim.x) {
        reinterpret_cast<uint4*>(sg + kMatBytes)[i] = make_uint4(0, 0, 0, 0);
    }
    umma::FenceBeforeSync();
    __syncthreads();
    umma::FenceAfterSync();
    const uint32_t tmem = *tmem_slot;
    const uint32_t a_addr = umma::SmemAddr(sa), w_addr = umma::SmemAddr(sw), g_addr = umma::SmemAddr(sg);
    uint32_t phase = 0;
    const int r = threadIdx.x;
    const int64_t tiles = (n + kTile - 1) / kTile;
    const float inv3n = n > 0 ? 1.0f / (3.0f * static_cast<float>(n)) : 0.0f;
    float my_loss = 0.0f;
    bool first = true, ok = true;
    for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        const int64_t row = t * kTile + r;
        const bool valid = row < n;
        {
            float x[kWidth];
            if (valid) {
                Encode(g, queries + row * kQueryFloats, x);
            } else {
#pragma unroll
                for (int k = 0; k < kWidth; ++k) x[k] = 0.0f;
            }
            StoreRow(sa, r, x);
        }
        HandOff();
        // Forward: a_{l+1} = bf16(relu(a_l W_l^T)); the output layer's first
        // three columns are o.
        for (int l = 0; l < kLayers && ok; ++l) {
            const int nn = l < kLayers - 1 ? 64 : 16;
            if (threadIdx.x == 0) {
                umma::FenceAfterSync();
                IssueForward(tmem, a_addr + l * kMatBytes, w_addr + l * kWBytes, nn);
                umma::Commit(bar);
            }
            ok = Await(bar, phase, error);
            if (!ok) break;
            float v[kWidth];
            if (l < kLayers - 1) {
                LoadAcc64(tmem, 0, v);
#pragma unroll
                for (int k = 0; k < kWidth; ++k) v[k] = fmaxf(v[k], 0.0f);
                StoreRow(sa + (l + 1) * kMatBytes, r, v);
            } else {
                float o[16];
                umma::Ld16(tmem + ((static_cast<uint32_t>(threadIdx.x) & ~31u) << 16), o);
                umma::WaitLd();
#pragma unroll
                for (int k = 0; k < kWidth; ++k) v[k] = 0.0f;
                if (valid) {
                    const float4 y = targets[row];
                    const float yk[3] = {y.x, y.y, y.z};
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const float rgb = ExpOut(o[k]);
                        const float denom = rgb * rgb + kLossEps;
                        const float diff = rgb - yk[k];
                        my_loss += diff * diff / denom;
                        const float drgb = (2.0f * diff / denom) * inv3n;
                        v[k] = o[k] < kOClamp ? drgb * rgb : 0.0f;
                    }
                }
                StoreRow(sg, r, v);
            }
            HandOff();
        }
        // Backward, output layer first.
        for (int l = kLayers - 1; l >= 0 && ok; --l) {
            if (threadIdx.x == 0) {
                umma::FenceAfterSync();
                // dW_l (+)= G^T a_l: M = 128 (rows >= 64 unused), N = 64, K = 128 rows.
                const uint32_t id_w = umma::IDesc(128, 64, true, true);
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    umma::Mma(tmem + 64 + 64 * l, umma::Desc(g_addr + 2048 * k, 1024, 128),
                              umma::Desc(a_addr + l * kMatBytes + 2048 * k, 1024, 128), id_w, !(first && k == 0));
                }
                // dX = G W_l: M = 128, N = 64 inputs, K = 64 outputs (16 for the output layer).
                const uint32_t id_x = umma::IDesc(128, 64, false, true);
                const int ks = l == kLayers - 1 ? 1 : 4;
                for (int k = 0; k < ks; ++k) {
                    umma::Mma(tmem, umma::Desc(g_addr + 256 * k, 128, 1024),
                              umma::Desc(w_addr + l * kWBytes + 2048 * k, 1024, 128), id_x, k > 0);
                }
                umma::Commit(bar);
            }
            ok = Await(bar, phase, error);
            if (!ok) break;
            float dx[kWidth];
            LoadAcc64(tmem, 0, dx);
            if (l > 0) {
                // dY_{l-1} = dX masked by relu'(a_l)
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    float a8[8];
                    LoadChunk(sa + l * kMatBytes, r, c, a8);
#pragma unroll
                    for (int k = 0; k < 8; ++k) dx[8 * c + k] = a8[k] > 0.0f ? dx[8 * c + k] : 0.0f;
                }
                StoreRow(sg, r, dx);
            } else {
                // Grid features: scatter d input / d feature with the
                // trilinear weights. Per level, the eight corners' gradient
                // reductions, touched-bit reads and bit sets are issued
                // together (eight requests in flight instead of one round
                // trip per corner), and the entries touched first this step
                // are appended to the optimiser's list with one counter
                // atomic per warp and level: the list counter is a single
                // address that every CTA updates, so its atomics serialise.
                // Every lane of the warp runs the loop (the warp-wide steps
                // need all of them); a lane without a sample touches nothing.
                const unsigned lane = threadIdx.x & 31u;
                float p[3] = {0.0f, 0.0f, 0.0f};
                if (valid) NormalisedPosition(g, queries + row * kQueryFloats, p);
#pragma unroll 1
                for (int lv = 0; lv < kLevels; ++lv) {
                    uint32_t idx[8];
                    float w[8];
                    LevelCorners(g, lv, p, idx, w);
                    const float d0 = dx[2 * lv], d1 = dx[2 * lv + 1];
                    int64_t e[8];
                    uint32_t seen[8];
                    uint32_t fresh = 0;  // bit c: corner c's entry was touched first by this lane
                    if (valid) {
#pragma unroll
                        for (int c = 0; c < 8; ++c) {
                            e[c] = static_cast<int64_t>(lv) * kTable + idx[c];
                            atomicAdd(g.grad + e[c], make_float2(w[c] * d0, w[c] * d1));
                        }
#pragma unroll
                        for (int c = 0; c < 8; ++c) seen[c] = g.touched[e[c] >> 5];
#pragma unroll
                        for (int c = 0; c < 8; ++c) {
                            // A bit already set was listed by whoever set it;
                            // of the threads that set it now, atomicOr tells
                            // exactly one that it came first.
                            const uint32_t bit = 1u << (e[c] & 31);
                            if (!(seen[c] & bit) && !(atomicOr(g.touched + (e[c] >> 5), bit) & bit)) {
                                fresh |= 1u << c;
                            }
                        }
                    }
                    // Warp prefix sum of the new entries, one counter atomic.
                    const uint32_t mine = static_cast<uint32_t>(__popc(fresh));
                    uint32_t incl = mine;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                        if (lane >= static_cast<unsigned>(o)) incl += y;
                    }
                    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
                    if (total) {
                        unsigned long long base = 0;
                        if (lane == 0) base = atomicAdd(g.touched_count, static_cast<unsigned long long>(total));
                        base = __shfl_sync(0xffffffffu, base, 0);
                        unsigned long long at = base + (incl - mine);
#pragma unroll
                        for (int c = 0; c < 8; ++c) {
                            if (fresh & (1u << c)) g.touched_list[at++] = static_cast<int32_t>(e[c]);
                        }
                    }
                }
            }
            HandOff();
        }
        first = false;
    }
    // Flush the weight gradients accumulated in TMEM (rows 0..63 live in the
    // lanes of warps 0 and 1).
    if (ok && !first && threadIdx.x < 64) {
        for (int l = 0; l < kLayers; ++l) {
            float v[kWidth];
            LoadAcc64(tmem, 64 + 64 * l, v);
            const int rows = l == kLayers - 1 ? 16 : 64;
            if (r < rows) {
#pragma unroll 8
                for (int k = 0; k < kWidth; ++k) atomicAdd(weight_grad + l * 4096 + r * kWidth + k, v[k]);
            }
        }
    }
    // loss: warp sums, one atomic per warp
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) my_loss += __shfl_xor_sync(0xffffffffu, my_loss, off);
    if ((threadIdx.x & 31) == 0 && loss_sum) atomicAdd(loss_sum, my_loss);
    umma::FenceBeforeSync();
    __syncthreads();
    if (threadIdx.x < 32) umma::TmemFree(tmem, kTrainTmemCols);
}

// ---------------------------------------------------------------- Adam

// The step's constants: bias corrections c1 = 1 - beta1^t, c2 = 1 - beta2^t
// (t read from the device so that a captured graph replays correctly) and
// the moving average's decay min(avg_decay, (1 + t) / (10 + t)).
struct AdamStep {
    float c1, c2, decay, keep;
};

__device__ inline AdamStep MakeAdamStep(const int64_t* step, float avg_decay) {
    const double t = static_cast<double>(*step);
    AdamStep a;
    a.c1 = static_cast<float>(1.0 - pow(kBeta1, t));
    a.c2 = static_cast<float>(1.0 - pow(kBeta2, t));
    a.decay = static_cast<float>(fmin(static_cast<double>(avg_decay), (1.0 + t) / (10.0 + t)));
    a.keep = static_cast<float>(1.0 - static_cast<double>(a.decay));
    return a;
}

// One parameter's Adam update in the operation order of the oracle, then
// its moving average (Polyak averaging); returns (parameter, average).
__device__ __forceinline__ float2 AdamUpdate(const AdamStep& a, float& p, float& m, float& v, float g, float& avg) {
    const float b1 = static_cast<float>(kBeta1), b2 = static_cast<float>(kBeta2);
    const float nb1 = static_cast<float>(1.0 - kBeta1), nb2 = static_cast<float>(1.0 - kBeta2);
    const float mi = __fadd_rn(__fmul_rn(m, b1), __fmul_rn(nb1, g));
    const float vi = __fadd_rn(__fmul_rn(v, b2), __fmul_rn(__fmul_rn(nb2, g), g));
    m = mi;
    v = vi;
    const float mhat = __fdiv_rn(mi, a.c1);
    const float vhat = __fdiv_rn(vi, a.c2);
    const float step = __fdiv_rn(__fmul_rn(kLr, mhat), __fadd_rn(__fsqrt_rn(vhat), kAdamEps));
    p = __fsub_rn(p, step);
    avg = __fadd_rn(__fmul_rn(a.decay, avg), __fmul_rn(a.keep, p));
    return make_float2(p, avg);
}

// Adam over every parameter (the network weights); `half_out` / `bf16_out`
// receive the rounded copy read by the kernels, likewise for the average.
__global__ void AdamKernel(float* p, float* m, float* v, const float* grad, int64_t count, const int64_t* step,
                           __half* half_out, __nv_bfloat16* bf16_out, float* avg, __half* avg_half,
                           __nv_bfloat16* avg_bf16, float avg_decay) {
    const AdamStep a = MakeAdamStep(step, avg_decay);
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        float pi = p[i], mi = m[i], vi = v[i], ai = avg[i];
        AdamUpdate(a, pi, mi, vi, grad[i], ai);
        p[i] = pi;
        m[i] = mi;
        v[i] = vi;
        avg[i] = ai;
        if (half_out) half_out[i] = __float2half_rn(pi);
        if (bf16_out) bf16_out[i] = __float2bfloat16_rn(pi);
        if (avg_half) avg_half[i] = __float2half_rn(ai);
        if (avg_bf16) avg_bf16[i] = __float2bfloat16_rn(ai);
    }
}

// Lazy Adam over the grid: only the entries this step's samples touched
// (the compacted list the training kernel wrote) update their two features,
// moments and averages, with the dense kernel's arithmetic; an entry no
// sample reached keeps its state, as sparse Adam variants do (PyTorch's
// SparseAdam). Each listed entry's gradient and touched bit are cleared for
// the next step, so no pass over the whole table is needed.
__global__ void SparseGridAdamKernel(float2* p, float2* m, float2* v, float2* grad, uint32_t* touched,
                                     const int32_t* list, const unsigned long long* count, const int64_t* step,
                                     __half2* half_out, float2* avg, __half2* avg_half, float avg_decay) {
    const AdamStep a = MakeAdamStep(step, avg_decay);
    const int64_t n = static_cast<int64_t>(*count);
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t e = list[i];
        touched[e >> 5] = 0u;  // every listed entry of the word clears it alike
        float2 pe = p[e], me = m[e], ve = v[e], ae = avg[e];
        const float2 ge = grad[e];
        AdamUpdate(a, pe.x, me.x, ve.x, ge.x, ae.x);
        AdamUpdate(a, pe.y, me.y, ve.y, ge.y, ae.y);
        p[e] = pe;
        m[e] = me;
        v[e] = ve;
        avg[e] = ae;
        grad[e] = make_float2(0.0f, 0.0f);
        half_out[e] = __floats2half2_rn(pe.x, pe.y);
        avg_half[e] = __floats2half2_rn(ae.x, ae.y);
    }
}

__global__ void StepKernel(int64_t* step) { ++*step; }

__global__ void RoundKernel(const float* p, int64_t count, __half* half_out, __nv_bfloat16* bf16_out) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (half_out) half_out[i] = __float2half_rn(p[i]);
        if (bf16_out) bf16_out[i] = __float2bfloat16_rn(p[i]);
    }
}

// Grid initialisation: U(-1e-4, 1e-4) from a hash of (seed, index).
__global__ void InitGridKernel(float* p, int64_t count, uint64_t seed) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        uint64_t z = seed + 0x9E3779B97F4A7C15ull * static_cast<uint64_t>(i + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        const float u = static_cast<float>(z >> 40) * (1.0f / 16777216.0f);
        p[i] = (u * 2.0f - 1.0f) * 1.0e-4f;
    }
}

}  // namespace nrc
}  // namespace yrc

// ----------------------------------------------------------------- C ABI

struct yrc_nrc {
    int device = 0;
    int sm_count = 0;
    yrc::nrc::GridArgs grid{};
    __half* table = nullptr;        // kLevels * kTable * 2
    float* table_master = nullptr;  // fp32 master
    float* table_m = nullptr;
    float* table_v = nullptr;
    float* table_grad = nullptr;    // zero between steps (the grid optimiser clears what it used)
    uint32_t* touched_mask = nullptr;       // entries touched this step, zero between steps
    int32_t* touched_list = nullptr;        // kLevels * kTable
    unsigned long long* touched_count = nullptr;
    __nv_bfloat16* w = nullptr;  // kWeightCount
    float* w_master = nullptr;
    float* w_m = nullptr;
    float* w_v = nullptr;
    float* w_grad = nullptr;
    // Exponential moving average of the parameters (fp32) and its rounded
    // copies, which the path tracer may query instead of the raw ones.
    float* table_avg_master = nullptr;
    __half* table_avg = nullptr;
    float* w_avg_master = nullptr;
    __nv_bfloat16* w_avg = nullptr;
    float avg_decay = yrc::nrc::kAvgDecay;
    float* loss = nullptr;  // device scalar (sum of per-sample losses)
    int* error = nullptr;
    int64_t* step = nullptr;  // device: optimiser steps taken
    std::mutex mutex;
};

namespace yrc {
namespace nrc {
namespace {

yrc_status CudaFailN(cudaError_t err, const char* what) {
    return Fail(YRC_ERR_CUDA, std::string("radiance cache: ") + what + ": " + cudaGetErrorString(err));
}

constexpr int64_t kGridParams = kLevels * kTable * 2;

unsigned Blocks(int64_t count, int sm_count) {
    const int64_t want = (count + 255) / 256;
    const int64_t cap = static_cast<int64_t>(sm_count) * 16;
    return static_cast<unsigned>(want < 1 ? 1 : (want > cap ? cap : want));
}

void FreeAll(yrc_nrc* c) {
    void* ptrs[] = {c->table,  c->table_master,     c->table_m,   c->table_v,      c->table_grad,
                    c->w,      c->w_master,         c->w_m,       c->w_v,          c->w_grad,
                    c->table_avg_master, c->table_avg, c->w_avg_master, c->w_avg, c->loss,
                    c->error,  c->step, c->touched_mask, c->touched_list, c->touched_count};
    for (void* p : ptrs) cudaFree(p);
}

// Gradients of n pairs (n_ptr: the count on the device, at most n).
yrc_status LaunchTrain(yrc_nrc* c, const float* queries, const float* targets, int64_t n,
                       const unsigned long long* n_ptr, cudaStream_t st) {
    // The grid gradients and touched bits are zero already (cleared per
    // entry by the grid optimiser); the compacted list starts empty.
    cudaError_t err = cudaMemsetAsync(c->touched_count, 0, sizeof(unsigned long long), st);
    if (err == cudaSuccess) err = cudaMemsetAsync(c->w_grad, 0, sizeof(float) * kWeightCount, st);
    if (err == cudaSuccess) err = cudaMemsetAsync(c->loss, 0, sizeof(float), st);
    if (err != cudaSuccess) return CudaFailN(err, "clearing gradients");
    if (n <= 0) return Ok();
    GridArgs g = c->grid;
    g.grad = reinterpret_cast<float2*>(c->table_grad);
    g.touched = c->touched_mask;
    g.touched_list = c->touched_list;
    g.touched_count = c->touched_count;
    const int64_t tiles = (n + kTile - 1) / kTile;
    const int64_t blocks = tiles < c->sm_count ? tiles : c->sm_count;  // one CTA per SM (TMEM, smem)
    CacheTrainKernel<<<static_cast<unsigned>(blocks), kThreads, kTrainSmem, st>>>(
        g, c->w, c->w_grad, queries, reinterpret_cast<const float4*>(targets), n, n_ptr, c->loss, c->error);
    err = cudaGetLastError();
    if (err != cudaSuccess) return CudaFailN(err, "training launch");
    return Ok();
}

yrc_status LaunchAdam(yrc_nrc* c, cudaStream_t st) {
    StepKernel<<<1, 1, 0, st>>>(c->step);
    AdamKernel<<<Blocks(kWeightCount, c->sm_count), 256, 0, st>>>(c->w_master, c->w_m, c->w_v, c->w_grad,
                                                                  kWeightCount, c->step, nullptr, c->w,
                                                                  c->w_avg_master, nullptr, c->w_avg, c->avg_decay);
    SparseGridAdamKernel<<<static_cast<unsigned>(c->sm_count) * 8, 256, 0, st>>>(
        reinterpret_cast<float2*>(c->table_master), reinterpret_cast<float2*>(c->table_m),
        reinterpret_cast<float2*>(c->table_v), reinterpret_cast<float2*>(c->table_grad), c->touched_mask,
        c->touched_list, c->touched_count, c->step, reinterpret_cast<__half2*>(c->table),
        reinterpret_cast<float2*>(c->table_avg_master), reinterpret_cast<__half2*>(c->table_avg), c->avg_decay);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return CudaFailN(err, "optimiser launch");
    return Ok();
}

yrc_status CheckError(yrc_nrc* c) {
    int e = 0;
    const cudaError_t err = cudaMemcpy(&e, c->error, sizeof(int), cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) return CudaFailN(err, "reading the status word");
    if (e) {
        cudaMemset(c->error, 0, sizeof(int));
        return Fail(YRC_ERR_DEVICE_FAULT, "radiance cache: a tensor-core wait timed out");
    }
    return Ok();
}

// Rounded copies of the master parameters, and the moving average restarted
// at them (weights and/or grid).
cudaError_t ResetAverage(yrc_nrc* c, bool weights, bool grid) {
    cudaError_t err = cudaSuccess;
    if (weights) {
        RoundKernel<<<Blocks(kWeightCount, c->sm_count), 256>>>(c->w_master, kWeightCount, nullptr, c->w);
        err = cudaMemcpy(c->w_avg_master, c->w_master, sizeof(float) * kWeightCount, cudaMemcpyDeviceToDevice);
        RoundKernel<<<Blocks(kWeightCount, c->sm_count), 256>>>(c->w_master, kWeightCount, nullptr, c->w_avg);
    }
    if (grid && err == cudaSuccess) {
        RoundKernel<<<Blocks(kGridParams, c->sm_count), 256>>>(c->table_master, kGridParams, c->table, nullptr);
        err = cudaMemcpy(c->table_avg_master, c->table_master, sizeof(float) * kGridParams,
                         cudaMemcpyDeviceToDevice);
        RoundKernel<<<Blocks(kGridParams, c->sm_count), 256>>>(c->table_master, kGridParams, c->table_avg, nullptr);
    }
    if (err == cudaSuccess) err = cudaDeviceSynchronize();
    return err;
}

}  // namespace

yrc_status Infer(yrc_nrc* c, const float* queries, int64_t n, const unsigned long long* n_ptr, float* rgb,
                 cudaStream_t st, bool averaged) {
    if (n <= 0) return Ok();
    const int64_t tiles = (n + kTile - 1) / kTile;
    int per_sm = 0;
    cudaError_t err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, CacheInferKernel, kThreads, kInferSmem);
    if (err != cudaSuccess) return CudaFailN(err, "occupancy");
    if (per_sm < 1) per_sm = 1;
    const int64_t cap = static_cast<int64_t>(per_sm) * c->sm_count;
    const int64_t blocks = tiles < cap ? tiles : cap;
    GridArgs g = c->grid;
    if (averaged) g.table = reinterpret_cast<const __half2*>(c->table_avg);
    CacheInferKernel<<<static_cast<unsigned>(blocks), kThreads, kInferSmem, st>>>(
        g, averaged ? c->w_avg : c->w, queries, n, n_ptr, reinterpret_cast<float4*>(rgb), c->error);
    err = cudaGetLastError();
    if (err != cudaSuccess) return CudaFailN(err, "inference launch");
    return Ok();
}

yrc_status TrainStep(yrc_nrc* c, const float* queries, const float* targets, int64_t n,
                     const unsigned long long* n_ptr, cudaStream_t st) {
    yrc_status s = LaunchTrain(c, queries, targets, n, n_ptr, st);
    if (s != YRC_OK) return s;
    return LaunchAdam(c, st);
}

}  // namespace nrc
}  // namespace yrc

extern "C" {

yrc_status yrc_nrc_create(const float box_lo[3], float box_extent, uint64_t seed, yrc_nrc** out) {
    using namespace yrc;
    using namespace yrc::nrc;
    if (!out || !box_lo || !(box_extent > 0.0f) || !std::isfinite(box_extent)) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_nrc_create: bad argument");
    }
    *out = nullptr;
    auto* c = new (std::nothrow) yrc_nrc();
    if (!c) return Fail(YRC_ERR_OUT_OF_MEMORY, "yrc_nrc_create: host allocation failed");
    cudaGetDevice(&c->device);
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device);
    const double b = std::exp(std::log(2048.0 / 16.0) / (kLevels - 1));
    for (int l = 0; l < kLevels; ++l) {
        const float s = static_cast<float>(16.0 * std::pow(b, l));
        c->grid.scale[l] = s;
        const int64_t side = static_cast<int64_t>(std::ceil(static_cast<double>(s))) + 2;
        c->grid.side[l] = side * side * side <= kTable ? static_cast<int32_t>(side) : 0;
    }
    for (int k = 0; k < 3; ++k) c->grid.lo[k] = box_lo[k];
    c->grid.inv = 1.0f / box_extent;
    cudaError_t err = cudaSuccess;
    auto alloc = [&](auto** p, size_t bytes) {
        if (err == cudaSuccess) err = cudaMalloc(reinterpret_cast<void**>(p), bytes);
    };
    alloc(&c->table, sizeof(__half) * kGridParams);
    alloc(&c->table_master, sizeof(float) * kGridParams);
    alloc(&c->table_m, sizeof(float) * kGridParams);
    alloc(&c->table_v, sizeof(float) * kGridParams);
    alloc(&c->table_grad, sizeof(float) * kGridParams);
    alloc(&c->touched_mask, sizeof(uint32_t) * (kLevels * kTable / 32));
    alloc(&c->touched_list, sizeof(int32_t) * kLevels * kTable);
    alloc(&c->touched_count, sizeof(unsigned long long));
    alloc(&c->w, sizeof(__nv_bfloat16) * kWeightCount);
    alloc(&c->w_master, sizeof(float) * kWeightCount);
    alloc(&c->w_m, sizeof(float) * kWeightCount);
    alloc(&c->w_v, sizeof(float) * kWeightCount);
    alloc(&c->w_grad, sizeof(float) * kWeightCount);
    alloc(&c->table_avg_master, sizeof(float) * kGridParams);
    alloc(&c->table_avg, sizeof(__half) * kGridParams);
    alloc(&c->w_avg_master, sizeof(float) * kWeightCount);
    alloc(&c->w_avg, sizeof(__nv_bfloat16) * kWeightCount);
    alloc(&c->loss, sizeof(float));
    alloc(&c->error, sizeof(int));
    alloc(&c->step, sizeof(int64_t));
    if (err == cudaSuccess) err = cudaFuncSetAttribute(CacheTrainKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       kTrainSmem);
    if (err == cudaSuccess) err = cudaFuncSetAttribute(CacheInferKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       kInferSmem);
    if (err != cudaSuccess) {
        FreeAll(c);
        delete c;
        return CudaFailN(err, "allocation");
    }
    c->grid.table = reinterpret_cast<const __half2*>(c->table);
    // Xavier-uniform weights (output rows 3..15 and rows 16..63 of the
    // output matrix zero), grid U(-1e-4, 1e-4), zero optimiser state.
    std::vector<float> w(kWeightCount, 0.0f);
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<float> unit(-1.0f, 1.0f);
    for (int l = 0; l < kLayers; ++l) {
        const int rows = l == kLayers - 1 ? 3 : 64;
        const float a = std::sqrt(6.0f / static_cast<float>(kWidth + (l == kLayers - 1 ? 3 : kWidth)));
        for (int r = 0; r < rows; ++r)
            for (int k = 0; k < kWidth; ++k) w[static_cast<size_t>(l) * 4096 + r * kWidth + k] = a * unit(rng);
    }
    err = cudaMemcpy(c->w_master, w.data(), sizeof(float) * kWeightCount, cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemset(c->w_m, 0, sizeof(float) * kWeightCount);
    if (err == cudaSuccess) err = cudaMemset(c->w_v, 0, sizeof(float) * kWeightCount);
    if (err == cudaSuccess) err = cudaMemset(c->table_m, 0, sizeof(float) * kGridParams);
    if (err == cudaSuccess) err = cudaMemset(c->table_v, 0, sizeof(float) * kGridParams);
    if (err == cudaSuccess) err = cudaMemset(c->table_grad, 0, sizeof(float) * kGridParams);
    if (err == cudaSuccess) err = cudaMemset(c->touched_mask, 0, sizeof(uint32_t) * (kLevels * kTable / 32));
    if (err == cudaSuccess) err = cudaMemset(c->touched_count, 0, sizeof(unsigned long long));
    if (err == cudaSuccess) err = cudaMemset(c->error, 0, sizeof(int));
    if (err == cudaSuccess) err = cudaMemset(c->step, 0, sizeof(int64_t));
    if (err == cudaSuccess) {
        InitGridKernel<<<Blocks(kGridParams, c->sm_count), 256>>>(c->table_master, kGridParams, seed);
        err = ResetAverage(c, true, true);
    }
    if (err != cudaSuccess) {
        FreeAll(c);
        delete c;
        return CudaFailN(err, "initialisation");
    }
    *out = c;
    return Ok();
}

void yrc_nrc_destroy(yrc_nrc* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    yrc::nrc::FreeAll(c);
    delete c;
}

yrc_status yrc_nrc_copy_state(yrc_nrc* dst, yrc_nrc* src) {
    using namespace yrc;
    using namespace yrc::nrc;
    if (!dst || !src || dst == src) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_nrc_copy_state: bad argument");
    if (dst->device != src->device) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_nrc_copy_state: caches on different devices");
    }
    std::scoped_lock lock(dst->mutex, src->mutex);
    cudaSetDevice(src->device);
    cudaError_t err = cudaDeviceSynchronize();
    auto copy = [&](void* d, const void* s_, size_t bytes) {
        if (err == cudaSuccess) err = cudaMemcpy(d, s_, bytes, cudaMemcpyDeviceToDevice);
    };
    copy(dst->table, src->table, sizeof(__half) * kGridParams);
    copy(dst->table_master, src->table_master, sizeof(float) * kGridParams);
    copy(dst->table_m, src->table_m, sizeof(float) * kGridParams);
    copy(dst->table_v, src->table_v, sizeof(float) * kGridParams);
    copy(dst->w, src->w, sizeof(__nv_bfloat16) * kWeightCount);
    copy(dst->w_master, src->w_master, sizeof(float) * kWeightCount);
    copy(dst->w_m, src->w_m, sizeof(float) * kWeightCount);
    copy(dst->w_v, src->w_v, sizeof(float) * kWeightCount);
    copy(dst->table_avg_master, src->table_avg_master, sizeof(float) * kGridParams);
    copy(dst->table_avg, src->table_avg, sizeof(__half) * kGridParams);
    copy(dst->w_avg_master, src->w_avg_master, sizeof(float) * kWeightCount);
    copy(dst->w_avg, src->w_avg, sizeof(__nv_bfloat16) * kWeightCount);
    copy(dst->step, src->step, sizeof(int64_t));
    if (err != cudaSuccess) return CudaFailN(err, "state copy");
    // The encoding's box and level scales; the table pointer stays dst's own.
    for (int l = 0; l < kLevels; ++l) {
        dst->grid.scale[l] = src->grid.scale[l];
        dst->grid.side[l] = src->grid.side[l];
    }
    for (int k = 0; k < 3; ++k) dst->grid.lo[k] = src->grid.lo[k];
    dst->grid.inv = src->grid.inv;
    dst->avg_decay = src->avg_decay;
    return Ok();
}

yrc_status yrc_nrc_set_params(yrc_nrc* c, const float* weights, const float* grid) {
    using namespace yrc;
    using namespace yrc::nrc;
    if (!c) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_nrc_set_params: null cache");
    std::lock_guard<std::mutex> lock(c->mutex);
    cudaSetDevice(c->device);
    cudaError_t err = cudaSuccess;
    if (weights) err = cudaMemcpy(c->w_master, weights, sizeof(float) * kWeightCount, cudaMemcpyHostToDevice);
    if (grid && err == cudaSuccess) {
        err = cudaMemcpy(c->table_master, grid, sizeof(float) * kGridParams, cudaMemcpyHostToDevice);
    }
    if (err == cudaSuccess) err = ResetAverage(c, weights != nullptr, grid != nullptr);
    if (err != cudaSuccess) return CudaFailN(err, "setting parameters");
    return Ok();
}

namespace {
yrc_status GetParams(yrc_nrc* c, const float* w_src, const float* grid_src, float* weights, float* grid) {
    using namespace yrc;
    using namespace yrc::nrc;
    std::lock_guard<std::mutex> lock(c->mutex);
    cudaSetDevice(c->device);
    cudaError_t err = cudaDeviceSynchronize();
    if (weights && err == cudaSuccess) {
        err = cudaMemcpy(weights, w_src, sizeof(float) * kWeightCount, cudaMemcpyDeviceToHost);
    }
    if (grid && err == cudaSuccess) {
        err = cudaMemcpy(grid, grid_src, sizeof(float) * kGridParams, cudaMemcpyDeviceToHost);
    }
    if (err != cudaSuccess) return CudaFailN(err, "reading parameters");
    return Ok();
}
}  // namespace

yrc_status yrc_nrc_get_params(yrc_nrc* c, float* weights, float* grid) {
    if (!c) return yrc::Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_nrc_get_params: null cache");
    return GetParams(c, c->w_master, c->table_master, weights, grid);
}

yrc_status yrc_nrc_set_average_decay(yrc_nrc* c, float decay) {
    if (!c || !(decay >= 0.0f && decay < 1.0f)) {
        return yrc::Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_nrc_set_average_decay: bad argument");
    }
    std::lock_guard<std::mutex> lock(c->mutex);
    c->avg_decay = decay;
    return yrc::Ok();
}

yrc_status yrc_nrc_get_averaged_params(yrc_nrc* c, float* weights, float* grid) {
    if (!c) return yrc::Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_nrc_get_averaged_params: null cache");
    return GetParams(c, c->w_avg_master, c->table_avg_master, weights, grid);
}

yrc_status yrc_nrc_infer(yrc_nrc* c, const float* queries, int64_t n, float* rgb, void* stream) {
    using namespace yrc;
    if (!c || n < 0 || (n > 0 && (!queries || !rgb))) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_nrc_infer: bad argument");
    std::lock_guard<std::mutex> lock(c->mutex);
    cudaSetDevice(c->device);
    return nrc::Infer(c, queries, n, nullptr, rgb, static_cast<cudaStream_t>(stream), false);
}

yrc_status yrc_nrc_gradients(yrc_nrc* c, const float* queries, const float* targets, int64_t n, float* weight_grads,
                             float* grid_grads, float* loss) {
    using namespace yrc;
    using namespace yrc::nrc;
    if (!c || n < 0 || (n > 0 && (!queries || !targets))) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_nrc_gradients: bad argument");
    }
    std::lock_guard<std::mutex> lock(c->mutex);
    cudaSetDevice(c->device);
    yrc_status s = LaunchTrain(c, queries, targets, n, nullptr, nullptr);
    if (s != YRC_OK) return s;
    cudaError_t err = cudaDeviceSynchronize();
    if (err != cudaSuccess) return CudaFailN(err, "gradients");
    s = CheckError(c);
    if (s != YRC_OK) return s;
    if (weight_grads) err = cudaMemcpy(weight_grads, c->w_grad, sizeof(float) * kWeightCount, cudaMemcpyDeviceToHost);
    if (grid_grads && err == cudaSuccess) {
        err = cudaMemcpy(grid_grads, c->table_grad, sizeof(float) * kGridParams, cudaMemcpyDeviceToHost);
    }
    if (loss && err == cudaSuccess) {
        float sum = 0.0f;
        err = cudaMemcpy(&sum, c->loss, sizeof(float), cudaMemcpyDeviceToHost);
        *loss = n > 0 ? sum / (3.0f * static_cast<float>(n)) : 0.0f;
    }
    // No optimiser step follows: restore the zero gradients and touched bits
    // the next training step starts from.
    if (err == cudaSuccess) err = cudaMemset(c->table_grad, 0, sizeof(float) * kGridParams);
    if (err == cudaSuccess) err = cudaMemset(c->touched_mask, 0, sizeof(uint32_t) * (kLevels * kTable / 32));
    if (err != cudaSuccess) return CudaFailN(err, "reading gradients");
    return Ok();
}

yrc_status yrc_nrc_train_step(yrc_nrc* c, const float* queries, const float* targets, int64_t n, float* loss_out,
                              void* stream) {
    using namespace yrc;
    using namespace yrc::nrc;
    if (!c || n < 0 || (n > 0 && (!queries || !targets))) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_nrc_train_step: bad argument");
    }
    std::lock_guard<std::mutex> lock(c->mutex);
    cudaSetDevice(c->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    yrc_status s = TrainStep(c, queries, targets, n, nullptr, st);
    if (s != YRC_OK) return s;
    if (loss_out) {
        const cudaError_t err = cudaMemcpyAsync(loss_out, c->loss, sizeof(float), cudaMemcpyDeviceToDevice, st);
        if (err != cudaSuccess) return CudaFailN(err, "loss copy");
    }
    return Ok();
}

yrc_status yrc_nrc_check(yrc_nrc* c) {
    using namespace yrc;
    if (!c) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_nrc_check: null cache");
    std::lock_guard<std::mutex> lock(c->mutex);
    cudaSetDevice(c->device);
    const cudaError_t err = cudaDeviceSynchronize();
    if (err != cudaSuccess) return nrc::CudaFailN(err, "synchronize");
    return nrc::CheckError(c);
}

}  // extern "C"
