// Device evaluation of the sampling primitives the render kernels use, for
// callers (and tests) that check the device's sample values against the
// reference's: the per-pixel sampler (Sampler, src/sampling/sampler.cpp:
// 122-310), PCG32 (include/yaoray/core/rng.hpp:15-48) and
// SeedForPixelSample (sampler.cpp:304-310). The kernels call the same
// device functions as the render path (sampler.cuh).
#include <cuda_runtime.h>

#include <string>

#include "sampler.cuh"
#include "yrc_internal.hpp"

namespace yrc {
namespace {

__global__ void SamplerEvalKernel(int32_t kind, uint64_t seed, int32_t spp, const int4* queries_xy_s_b,
                                  const int2* queries_dim_lane, int64_t n, int32_t two_d, float* out) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const int4 q = queries_xy_s_b[i];
    const int2 dl = queries_dim_lane[i];
    PixelSampler s;
    s.Init(kind, seed, q.x, q.y, q.z, spp);
    const int bounce = q.w < 0 ? 0 : q.w;
    if (two_d) {
        float x, y;
        s.Sample2D(static_cast<uint32_t>(dl.x), bounce, x, y, dl.y);
        out[2 * i] = x;
        out[2 * i + 1] = y;
    } else {
        out[i] = s.Sample1D(static_cast<uint32_t>(dl.x), bounce, dl.y);
    }
}

__global__ void RngEvalKernel(const uint64_t* seeds, int64_t n, int32_t draws, float* out) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    Pcg32 rng;
    rng.Seed(seeds[i]);
    for (int32_t k = 0; k < draws; ++k) out[i * draws + k] = rng.NextFloat();
}

__global__ void PixelSeedEvalKernel(uint64_t seed, const int64_t* queries, int64_t n, uint64_t* out) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    out[i] = SeedForPixelSample(seed, static_cast<int>(queries[3 * i]), static_cast<int>(queries[3 * i + 1]),
                                static_cast<int>(queries[3 * i + 2]));
}

unsigned Blocks(int64_t n) { return static_cast<unsigned>((n + 255) / 256); }

// Device copies of host inputs and outputs, freed together.
struct Scratch {
    void* p[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaError_t err = cudaSuccess;
    void* Alloc(int k, size_t bytes) {
        if (err == cudaSuccess) err = cudaMalloc(&p[k], bytes > 0 ? bytes : 1);
        return p[k];
    }
    ~Scratch() {
        for (void* q : p) cudaFree(q);
    }
};

yrc_status Done(cudaError_t err, const char* what) {
    if (err != cudaSuccess) return Fail(YRC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
    return Ok();
}

}  // namespace
}  // namespace yrc

extern "C" {

yrc_status yrc_sampler_eval(int32_t kind, uint64_t seed, int32_t spp, const int32_t* queries, int64_t n,
                            int32_t two_d, float* out) {
    using namespace yrc;
    if (n < 0 || (n > 0 && (!queries || !out)) || kind < 0 || kind > 3) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_sampler_eval: bad argument");
    }
    if (n == 0) return Ok();
    std::vector<int4> a(static_cast<size_t>(n));
    std::vector<int2> b(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) {
        const int32_t* r = queries + 6 * i;
        a[static_cast<size_t>(i)] = make_int4(r[0], r[1], r[2], r[3]);
        b[static_cast<size_t>(i)] = make_int2(r[4], r[5]);
    }
    const size_t out_bytes = sizeof(float) * static_cast<size_t>(n) * (two_d ? 2 : 1);
    Scratch s;
    auto* da = static_cast<int4*>(s.Alloc(0, sizeof(int4) * a.size()));
    auto* db = static_cast<int2*>(s.Alloc(1, sizeof(int2) * b.size()));
    auto* dout = static_cast<float*>(s.Alloc(2, out_bytes));
    cudaError_t err = s.err;
    if (err == cudaSuccess) err = cudaMemcpy(da, a.data(), sizeof(int4) * a.size(), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemcpy(db, b.data(), sizeof(int2) * b.size(), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) {
        SamplerEvalKernel<<<Blocks(n), 256>>>(kind, seed, spp, da, db, n, two_d, dout);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemcpy(out, dout, out_bytes, cudaMemcpyDeviceToHost);
    return Done(err, "yrc_sampler_eval");
}

yrc_status yrc_rng_eval(const uint64_t* seeds, int64_t n, int32_t draws, float* out) {
    using namespace yrc;
    if (n < 0 || draws < 0 || (n > 0 && (!seeds || !out))) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_rng_eval: bad argument");
    if (n == 0 || draws == 0) return Ok();
    Scratch s;
    auto* ds = static_cast<uint64_t*>(s.Alloc(0, sizeof(uint64_t) * static_cast<size_t>(n)));
    auto* dout = static_cast<float*>(s.Alloc(1, sizeof(float) * static_cast<size_t>(n) * draws));
    cudaError_t err = s.err;
    if (err == cudaSuccess) err = cudaMemcpy(ds, seeds, sizeof(uint64_t) * static_cast<size_t>(n), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) {
        RngEvalKernel<<<Blocks(n), 256>>>(ds, n, draws, dout);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) {
        err = cudaMemcpy(out, dout, sizeof(float) * static_cast<size_t>(n) * draws, cudaMemcpyDeviceToHost);
    }
    return Done(err, "yrc_rng_eval");
}

yrc_status yrc_pixel_seed_eval(uint64_t seed, const int64_t* queries, int64_t n, uint64_t* out) {
    using namespace yrc;
    if (n < 0 || (n > 0 && (!queries || !out))) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_pixel_seed_eval: bad argument");
    if (n == 0) return Ok();
    Scratch s;
    auto* dq = static_cast<int64_t*>(s.Alloc(0, sizeof(int64_t) * 3 * static_cast<size_t>(n)));
    auto* dout = static_cast<uint64_t*>(s.Alloc(1, sizeof(uint64_t) * static_cast<size_t>(n)));
    cudaError_t err = s.err;
    if (err == cudaSuccess) err = cudaMemcpy(dq, queries, sizeof(int64_t) * 3 * static_cast<size_t>(n), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) {
        PixelSeedEvalKernel<<<Blocks(n), 256>>>(seed, dq, n, dout);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemcpy(out, dout, sizeof(uint64_t) * static_cast<size_t>(n), cudaMemcpyDeviceToHost);
    return Done(err, "yrc_pixel_seed_eval");
}

}  // extern "C"
