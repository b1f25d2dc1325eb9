// Measured BRDFs: host-side warp construction (PiecewiseLinear2D's
// constructor, include/yaoray/shading/piecewise_linear_2d.hpp, as
// LoadMeasuredBrdf builds the five warps, src/shading/measured_brdf.cpp:
// 150-189), upload, and C-ABI entry points that evaluate / sample a measured
// BRDF on the device for callers that compare it with the reference's.
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "measured.hpp"
#include "yrc_internal.hpp"

namespace yrc {
namespace {

struct HostWarp {
    int32_t size_x = 0, size_y = 0;
    std::vector<float> data, marginal, conditional;
    std::vector<float> params[3];
    uint32_t param_size[3] = {1, 1, 1};
    uint32_t param_stride[3] = {0, 0, 0};
    float patch_x = 0, patch_y = 0, inv_x = 0, inv_y = 0;
};

// The constructor's steps: slices over the parameter grid (last parameter
// varies fastest); with CDFs, per slice the row CDFs and the marginal CDF of
// the row integrals (trapezoids summed in double), everything normalised by
// the total; without, the values scaled by the cell area (and, when asked,
// normalised by their mean cell average).
HostWarp BuildWarp(const float* data, int xs, int ys, int dims, const int* res, const float* const* values,
                   bool normalize, bool build_cdf) {
    HostWarp w;
    w.size_x = xs;
    w.size_y = ys;
    w.patch_x = 1.f / static_cast<float>(xs - 1);
    w.patch_y = 1.f / static_cast<float>(ys - 1);
    w.inv_x = static_cast<float>(xs - 1);
    w.inv_y = static_cast<float>(ys - 1);
    uint32_t slices = 1;
    for (int i = dims - 1; i >= 0; --i) {
        const int pr = res[i] < 1 ? 1 : res[i];
        w.param_size[i] = static_cast<uint32_t>(pr);
        w.params[i].assign(values[i], values[i] + pr);
        w.param_stride[i] = pr > 1 ? slices : 0;
        slices *= w.param_size[i];
    }
    const size_t n_values = static_cast<size_t>(xs) * static_cast<size_t>(ys);
    w.data.assign(static_cast<size_t>(slices) * n_values, 0.f);
    if (build_cdf) {
        w.marginal.assign(static_cast<size_t>(slices) * ys, 0.f);
        w.conditional.assign(static_cast<size_t>(slices) * n_values, 0.f);
        for (uint32_t s = 0; s < slices; ++s) {
            const float* in = data + s * n_values;
            float* cond = w.conditional.data() + s * n_values;
            float* marg = w.marginal.data() + static_cast<size_t>(s) * ys;
            float* out = w.data.data() + s * n_values;
            for (int y = 0; y < ys; ++y) {
                double sum = 0.0;
                size_t i = static_cast<size_t>(y) * xs;
                cond[i] = 0.f;
                for (int x = 0; x < xs - 1; ++x, ++i) {
                    sum += 0.5 * (static_cast<double>(in[i]) + static_cast<double>(in[i + 1]));
                    cond[i + 1] = static_cast<float>(sum);
                }
            }
            marg[0] = 0.f;
            double sum = 0.0;
            for (int y = 0; y < ys - 1; ++y) {
                sum += 0.5 * (static_cast<double>(cond[static_cast<size_t>(y + 1) * xs - 1]) +
                              static_cast<double>(cond[static_cast<size_t>(y + 2) * xs - 1]));
                marg[y + 1] = static_cast<float>(sum);
            }
            const float total = marg[ys - 1];
            if (total > 0.f && std::isfinite(total)) {
                const float norm = 1.f / total;
                for (size_t i = 0; i < n_values; ++i) cond[i] *= norm;
                for (int i = 0; i < ys; ++i) marg[i] *= norm;
                for (size_t i = 0; i < n_values; ++i) out[i] = in[i] * norm;
            } else {
                for (size_t i = 0; i < n_values; ++i) out[i] = in[i];
            }
        }
    } else {
        for (uint32_t s = 0; s < slices; ++s) {
            const float* in = data + s * n_values;
            float* out = w.data.data() + s * n_values;
            float norm = 1.f / (w.inv_x * w.inv_y);
            if (normalize) {
                double sum = 0.0;
                for (int y = 0; y < ys - 1; ++y) {
                    size_t i = static_cast<size_t>(y) * xs;
                    for (int x = 0; x < xs - 1; ++x, ++i) {
                        const float avg = 0.25f * (in[i] + in[i + 1] + in[i + xs] + in[i + 1 + xs]);
                        sum += static_cast<double>(avg);
                    }
                }
                norm = (sum > 0.0 && std::isfinite(sum)) ? static_cast<float>(1.0 / sum) : 1.f;
            }
            for (size_t k = 0; k < n_values; ++k) out[k] = in[k] * norm;
        }
    }
    return w;
}

// Appends a warp's arrays to `blob`; returns the device warp with offsets in
// place of pointers (fixed up by Relocate).
DevWarp Pack(const HostWarp& w, std::vector<float>& blob) {
    DevWarp d{};
    auto put = [&](const std::vector<float>& v) {
        const size_t at = blob.size();
        blob.insert(blob.end(), v.begin(), v.end());
        return reinterpret_cast<const float*>(at);
    };
    d.data = put(w.data);
    d.marginal = put(w.marginal);
    d.conditional = put(w.conditional);
    for (int i = 0; i < 3; ++i) {
        d.param_values[i] = put(w.params[i]);
        d.param_size[i] = w.param_size[i];
        d.param_stride[i] = w.param_stride[i];
    }
    d.size_x = w.size_x;
    d.size_y = w.size_y;
    d.patch_x = w.patch_x;
    d.patch_y = w.patch_y;
    d.inv_patch_x = w.inv_x;
    d.inv_patch_y = w.inv_y;
    return d;
}

void Relocate(DevWarp& d, const float* base) {
    auto fix = [&](const float*& p) { p = base + reinterpret_cast<size_t>(p); };
    fix(d.data);
    fix(d.marginal);
    fix(d.conditional);
    for (int i = 0; i < 3; ++i) fix(d.param_values[i]);
}

__global__ void MeasuredEvalKernel(const DevMeasuredBrdf* m, const float* q, int64_t n, float* f, float* pdf) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const float* r = q + 9 * i;
    const V3 wo{r[0], r[1], r[2]}, wi{r[3], r[4], r[5]}, nn{r[6], r[7], r[8]};
    const V3 v = EvalMeasured(*m, wo, wi, nn);
    f[3 * i] = v.x;
    f[3 * i + 1] = v.y;
    f[3 * i + 2] = v.z;
    pdf[i] = PdfMeasuredBrdf(*m, wo, wi, nn);
}

__global__ void MeasuredSampleKernel(const DevMeasuredBrdf* m, const float* q, int64_t n, float* out) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const float* r = q + 8 * i;
    const BsdfSample s = SampleMeasuredBrdf(*m, V3{r[0], r[1], r[2]}, V3{r[3], r[4], r[5]}, r[6], r[7]);
    float* o = out + 8 * i;
    o[0] = s.wi.x;
    o[1] = s.wi.y;
    o[2] = s.wi.z;
    o[3] = s.weight.x;
    o[4] = s.weight.y;
    o[5] = s.weight.z;
    o[6] = s.pdf;
    o[7] = s.valid ? 1.0f : 0.0f;
}

yrc_status CheckBrdf(const yrc_measured_brdf& b, int32_t i) {
    const std::string where = "measured BRDF " + std::to_string(i) + ": ";
    if (b.n_theta_i < 1 || b.n_phi_i < 1 || b.n_wavelengths < 1 || b.ndf_rows < 2 || b.ndf_cols < 2 ||
        b.vndf_rows < 2 || b.vndf_cols < 2 || b.res < 2 || !b.theta_i || !b.phi_i || !b.wavelengths || !b.ndf ||
        !b.sigma || !b.vndf || !b.luminance || !b.spectra) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, where + "missing arrays or grids smaller than 2 x 2");
    }
    if (b.n_phi_i > 2) return Fail(YRC_ERR_UNSUPPORTED, where + "anisotropic measured BRDF not supported (isotropic-only)");
    return Ok();
}

}  // namespace

void MeasuredSet::Release() {
    for (void* p : blocks) cudaFree(p);
    blocks.clear();
    brdfs = nullptr;
    count = 0;
    bytes = 0;
}

yrc_status UploadMeasured(const yrc_measured_brdf* brdfs, int32_t count, MeasuredSet& out) {
    out.Release();
    if (count < 0 || (count > 0 && !brdfs)) return Fail(YRC_ERR_INVALID_ARGUMENT, "invalid measured BRDF array");
    for (int32_t i = 0; i < count; ++i) {
        const yrc_status st = CheckBrdf(brdfs[i], i);
        if (st != YRC_OK) return st;
    }
    if (count == 0) return Ok();
    std::vector<DevMeasuredBrdf> host(static_cast<size_t>(count));
    std::vector<std::vector<float>> blobs(static_cast<size_t>(count));
    for (int32_t i = 0; i < count; ++i) {
        const yrc_measured_brdf& b = brdfs[i];
        std::vector<float>& blob = blobs[static_cast<size_t>(i)];
        const int none[1] = {1};
        const float* no_values[1] = {nullptr};
        const int p2[2] = {b.n_phi_i, b.n_theta_i};
        const float* v2[2] = {b.phi_i, b.theta_i};
        const int p3[3] = {b.n_phi_i, b.n_theta_i, b.n_wavelengths};
        const float* v3[3] = {b.phi_i, b.theta_i, b.wavelengths};
        DevMeasuredBrdf& d = host[static_cast<size_t>(i)];
        d.ndf = Pack(BuildWarp(b.ndf, b.ndf_cols, b.ndf_rows, 0, none, no_values, false, false), blob);
        d.sigma = Pack(BuildWarp(b.sigma, b.ndf_cols, b.ndf_rows, 0, none, no_values, false, false), blob);
        d.vndf = Pack(BuildWarp(b.vndf, b.vndf_cols, b.vndf_rows, 2, p2, v2, true, true), blob);
        d.luminance = Pack(BuildWarp(b.luminance, b.res, b.res, 2, p2, v2, true, true), blob);
        d.spectra = Pack(BuildWarp(b.spectra, b.res, b.res, 3, p3, v3, false, false), blob);
        d.isotropic = b.n_phi_i <= 2 ? 1 : 0;
    }
    cudaError_t err = cudaSuccess;
    for (int32_t i = 0; i < count && err == cudaSuccess; ++i) {
        const std::vector<float>& blob = blobs[static_cast<size_t>(i)];
        void* p = nullptr;
        err = cudaMalloc(&p, sizeof(float) * std::max<size_t>(blob.size(), 1));
        if (err != cudaSuccess) break;
        out.blocks.push_back(p);
        out.bytes += static_cast<int64_t>(sizeof(float) * blob.size());
        err = cudaMemcpy(p, blob.data(), sizeof(float) * blob.size(), cudaMemcpyHostToDevice);
        DevMeasuredBrdf& d = host[static_cast<size_t>(i)];
        const float* base = static_cast<const float*>(p);
        Relocate(d.ndf, base);
        Relocate(d.sigma, base);
        Relocate(d.vndf, base);
        Relocate(d.luminance, base);
        Relocate(d.spectra, base);
    }
    void* table = nullptr;
    if (err == cudaSuccess) err = cudaMalloc(&table, sizeof(DevMeasuredBrdf) * host.size());
    if (err == cudaSuccess) {
        out.blocks.push_back(table);
        err = cudaMemcpy(table, host.data(), sizeof(DevMeasuredBrdf) * host.size(), cudaMemcpyHostToDevice);
    }
    if (err != cudaSuccess) {
        out.Release();
        return Fail(YRC_ERR_CUDA, std::string("measured BRDF upload: ") + cudaGetErrorString(err));
    }
    out.brdfs = static_cast<DevMeasuredBrdf*>(table);
    out.count = count;
    return Ok();
}

}  // namespace yrc

extern "C" {

yrc_status yrc_measured_eval(const yrc_measured_brdf* brdf, const float* queries, int64_t n, float* f, float* pdf) {
    using namespace yrc;
    if (!brdf || n < 0 || (n > 0 && (!queries || !f || !pdf))) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_measured_eval: bad argument");
    }
    MeasuredSet set;
    yrc_status st = UploadMeasured(brdf, 1, set);
    if (st != YRC_OK || n == 0) return st;
    float *dq = nullptr, *df = nullptr, *dp = nullptr;
    cudaError_t err = cudaMalloc(&dq, sizeof(float) * 9 * static_cast<size_t>(n));
    if (err == cudaSuccess) err = cudaMalloc(&df, sizeof(float) * 3 * static_cast<size_t>(n));
    if (err == cudaSuccess) err = cudaMalloc(&dp, sizeof(float) * static_cast<size_t>(n));
    if (err == cudaSuccess) err = cudaMemcpy(dq, queries, sizeof(float) * 9 * static_cast<size_t>(n), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) {
        MeasuredEvalKernel<<<static_cast<unsigned>((n + 127) / 128), 128>>>(set.brdfs, dq, n, df, dp);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemcpy(f, df, sizeof(float) * 3 * static_cast<size_t>(n), cudaMemcpyDeviceToHost);
    if (err == cudaSuccess) err = cudaMemcpy(pdf, dp, sizeof(float) * static_cast<size_t>(n), cudaMemcpyDeviceToHost);
    cudaFree(dq);
    cudaFree(df);
    cudaFree(dp);
    set.Release();
    if (err != cudaSuccess) return Fail(YRC_ERR_CUDA, std::string("yrc_measured_eval: ") + cudaGetErrorString(err));
    return Ok();
}

yrc_status yrc_measured_sample(const yrc_measured_brdf* brdf, const float* queries, int64_t n, float* out) {
    using namespace yrc;
    if (!brdf || n < 0 || (n > 0 && (!queries || !out))) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_measured_sample: bad argument");
    }
    MeasuredSet set;
    yrc_status st = UploadMeasured(brdf, 1, set);
    if (st != YRC_OK || n == 0) return st;
    float *dq = nullptr, *dout = nullptr;
    cudaError_t err = cudaMalloc(&dq, sizeof(float) * 8 * static_cast<size_t>(n));
    if (err == cudaSuccess) err = cudaMalloc(&dout, sizeof(float) * 8 * static_cast<size_t>(n));
    if (err == cudaSuccess) err = cudaMemcpy(dq, queries, sizeof(float) * 8 * static_cast<size_t>(n), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) {
        MeasuredSampleKernel<<<static_cast<unsigned>((n + 127) / 128), 128>>>(set.brdfs, dq, n, dout);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemcpy(out, dout, sizeof(float) * 8 * static_cast<size_t>(n), cudaMemcpyDeviceToHost);
    cudaFree(dq);
    cudaFree(dout);
    set.Release();
    if (err != cudaSuccess) return Fail(YRC_ERR_CUDA, std::string("yrc_measured_sample: ") + cudaGetErrorString(err));
    return Ok();
}

}  // extern "C"
