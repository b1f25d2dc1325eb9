// Device evaluation of the path tracer's scattering functions, for callers
// (and tests) that check them one by one against the reference's:
// EvaluateBsdf / PdfBsdf / SampleBsdf (src/shading/bsdf.cpp:17-310, with the
// microfacet lobes of src/shading/bsdf_microfacet.cpp:16-298 and the
// stochastic layered walk of src/shading/bsdf_layered.cpp:13-349) and
// TabulatedBSSRDF's Sr / Sample_Sr / Pdf_Sr / Pdf_Sp
// (src/shading/bssrdf.cpp:153-266). The kernels call the same device
// functions as the render stages (bsdf.cuh, bssrdf.cuh); this unit is
// compiled without fused multiply-adds, like the render kernels.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "bsdf.cuh"
#include "bssrdf.cuh"
#include "render_types.hpp"
#include "yrc_internal.hpp"

namespace yrc {
namespace {

__device__ __forceinline__ V3 Row3(const float* r) { return V3{r[0], r[1], r[2]}; }

// Per query: f = EvaluateBsdf(wo, wi, n, rng), then pdf = PdfBsdf(wo, wi, n,
// rng) with the same PCG32 stream, as a path vertex evaluates a light sample.
__global__ void BsdfEvalKernel(Mat m, const float* queries, const uint64_t* seeds, int64_t n, float* f, float* pdf) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const float* q = queries + 9 * i;
    Pcg32 rng;
    rng.Seed(seeds[i]);
    const V3 c = EvalBsdf(m, Row3(q), Row3(q + 3), Row3(q + 6), rng);
    const float p = PdfBsdf(m, Row3(q), Row3(q + 3), Row3(q + 6), rng);
    f[3 * i] = c.x;
    f[3 * i + 1] = c.y;
    f[3 * i + 2] = c.z;
    pdf[i] = p;
}

// Per query (wo, n, u): SampleBsdf -> (wi, weight, pdf, valid, specular).
__global__ void BsdfSampleKernel(Mat m, const float* queries, const uint64_t* seeds, int64_t n, float* out) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const float* q = queries + 8 * i;
    Pcg32 rng;
    rng.Seed(seeds[i]);
    const BsdfSample s = SampleBsdf(m, Row3(q), Row3(q + 3), q[6], q[7], rng);
    float* o = out + 9 * i;
    o[0] = s.wi.x;
    o[1] = s.wi.y;
    o[2] = s.wi.z;
    o[3] = s.weight.x;
    o[4] = s.weight.y;
    o[5] = s.weight.z;
    o[6] = s.pdf;
    o[7] = s.valid ? 1.0f : 0.0f;
    o[8] = s.specular ? 1.0f : 0.0f;
}

__global__ void BssrdfEvalKernel(TabBssrdf b, const int32_t* channels, const float* u, const float* r, int64_t n,
                                 float* sample_r, float* pdf_sr, float* sr) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const int ch = channels[i];
    sample_r[i] = BssrdfSampleSr(b, ch, u[i]);
    pdf_sr[i] = BssrdfPdfSr(b, ch, r[i]);
    const V3 s = BssrdfSr(b, r[i]);
    sr[3 * i] = s.x;
    sr[3 * i + 1] = s.y;
    sr[3 * i + 2] = s.z;
}

// Per query: 18 floats (po, ss, ts, ns, pi, ni) -> Pdf_Sp.
__global__ void BssrdfPdfSpKernel(TabBssrdf b, const float* q, int64_t n, float* pdf) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const float* p = q + 18 * i;
    pdf[i] = BssrdfPdfSp(b, Row3(p), Row3(p + 3), Row3(p + 6), Row3(p + 9), Row3(p + 12), Row3(p + 15));
}

unsigned Blocks(int64_t n) { return static_cast<unsigned>((n + 255) / 256); }

// Device buffers of one call, freed together.
struct Buffers {
    std::vector<void*> p;
    cudaError_t err = cudaSuccess;
    template <typename T>
    T* Upload(const T* host, size_t count) {
        void* d = nullptr;
        if (err == cudaSuccess) err = cudaMalloc(&d, count > 0 ? count * sizeof(T) : 1);
        if (err == cudaSuccess) p.push_back(d);
        if (err == cudaSuccess && host && count > 0) err = cudaMemcpy(d, host, count * sizeof(T), cudaMemcpyHostToDevice);
        return static_cast<T*>(d);
    }
    template <typename T>
    T* Alloc(size_t count) {
        return Upload<T>(nullptr, count);
    }
    ~Buffers() {
        for (void* q : p) cudaFree(q);
    }
};

// The part of a yrc_material the BSDFs read (the render path's LoadMat).
Mat MatOf(const yrc_material& m) {
    Mat r{};
    r.kind = m.kind;
    r.reflectance = V3{m.reflectance[0], m.reflectance[1], m.reflectance[2]};
    r.ior = m.ior;
    r.ur = m.uroughness;
    r.vr = m.vroughness;
    r.coating_ior = m.coating_ior;
    r.coat_thickness = m.coat_thickness;
    r.coat_absorption = V3{m.coat_absorption[0], m.coat_absorption[1], m.coat_absorption[2]};
    r.coat_maxdepth = m.coat_maxdepth;
    r.coat_nsamples = m.coat_nsamples;
    r.measured = nullptr;
    return r;
}

bool BsdfKindSupported(int32_t kind) {
    return kind >= YRC_MAT_DIFFUSE && kind <= YRC_MAT_SUBSURFACE_EXIT && kind != YRC_MAT_MEASURED;
}

// TabulatedBSSRDF(sigma_a, sigma_s, eta, table) with the table in device
// memory (the render path's MakeTabBssrdf).
bool MakeDeviceBssrdf(const yrc_bssrdf_table* t, const float sigma_a[3], const float sigma_s[3], float eta,
                      Buffers& buf, TabBssrdf& b) {
    const size_t rc = static_cast<size_t>(t->rho_count), nc = static_cast<size_t>(t->radius_count);
    DevBssrdf d{};
    d.rho_count = t->rho_count;
    d.radius_count = t->radius_count;
    d.rho = buf.Upload(t->rho_samples, rc);
    d.radius = buf.Upload(t->radius_samples, nc);
    d.profile = buf.Upload(t->profile, rc * nc);
    d.rho_eff = buf.Upload(t->rho_eff, rc);
    d.profile_cdf = buf.Upload(t->profile_cdf, rc * nc);
    // MakeTabBssrdf's per-channel extinction and albedo, on the host.
    for (int k = 0; k < 3; ++k) {
        b.st[k] = sigma_a[k] + sigma_s[k];
        b.rho[k] = b.st[k] != 0.0f ? sigma_s[k] / b.st[k] : 0.0f;
    }
    b.eta = eta;
    b.table = d;
    return buf.err == cudaSuccess;
}

bool TableValid(const yrc_bssrdf_table* t) {
    return t && t->rho_count >= 4 && t->radius_count >= 4 && t->rho_samples && t->radius_samples && t->profile &&
           t->rho_eff && t->profile_cdf;
}

yrc_status Done(cudaError_t err, const char* what) {
    if (err != cudaSuccess) return Fail(YRC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
    return Ok();
}

}  // namespace
}  // namespace yrc

extern "C" {

yrc_status yrc_bsdf_eval(const yrc_material* material, const float* queries, const uint64_t* seeds, int64_t n,
                         float* f, float* pdf) {
    using namespace yrc;
    if (!material || n < 0 || (n > 0 && (!queries || !seeds || !f || !pdf))) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_bsdf_eval: bad argument");
    }
    if (!BsdfKindSupported(material->kind)) {
        return Fail(YRC_ERR_UNSUPPORTED, "yrc_bsdf_eval: material kind " + std::to_string(material->kind) +
                                             " (measured BRDFs have yrc_measured_eval)");
    }
    if (n == 0) return Ok();
    Buffers b;
    const size_t un = static_cast<size_t>(n);
    const float* dq = b.Upload(queries, 9 * un);
    const uint64_t* ds = b.Upload(seeds, un);
    float* df = b.Alloc<float>(3 * un);
    float* dp = b.Alloc<float>(un);
    cudaError_t err = b.err;
    if (err == cudaSuccess) {
        BsdfEvalKernel<<<Blocks(n), 256>>>(MatOf(*material), dq, ds, n, df, dp);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemcpy(f, df, 3 * un * sizeof(float), cudaMemcpyDeviceToHost);
    if (err == cudaSuccess) err = cudaMemcpy(pdf, dp, un * sizeof(float), cudaMemcpyDeviceToHost);
    return Done(err, "yrc_bsdf_eval");
}

yrc_status yrc_bsdf_sample(const yrc_material* material, const float* queries, const uint64_t* seeds, int64_t n,
                           float* out) {
    using namespace yrc;
    if (!material || n < 0 || (n > 0 && (!queries || !seeds || !out))) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_bsdf_sample: bad argument");
    }
    if (!BsdfKindSupported(material->kind)) {
        return Fail(YRC_ERR_UNSUPPORTED, "yrc_bsdf_sample: material kind " + std::to_string(material->kind) +
                                             " (measured BRDFs have yrc_measured_sample)");
    }
    if (n == 0) return Ok();
    Buffers b;
    const size_t un = static_cast<size_t>(n);
    const float* dq = b.Upload(queries, 8 * un);
    const uint64_t* ds = b.Upload(seeds, un);
    float* dout = b.Alloc<float>(9 * un);
    cudaError_t err = b.err;
    if (err == cudaSuccess) {
        BsdfSampleKernel<<<Blocks(n), 256>>>(MatOf(*material), dq, ds, n, dout);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemcpy(out, dout, 9 * un * sizeof(float), cudaMemcpyDeviceToHost);
    return Done(err, "yrc_bsdf_sample");
}

yrc_status yrc_bssrdf_eval(const yrc_bssrdf_table* table, const float sigma_a[3], const float sigma_s[3], float eta,
                           const int32_t* channels, const float* u, const float* r, int64_t n, float* sample_r,
                           float* pdf_sr, float* sr) {
    using namespace yrc;
    if (!TableValid(table) || !sigma_a || !sigma_s || n < 0 ||
        (n > 0 && (!channels || !u || !r || !sample_r || !pdf_sr || !sr))) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_bssrdf_eval: bad argument");
    }
    for (int64_t i = 0; i < n; ++i) {
        if (channels[i] < 0 || channels[i] > 2) return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_bssrdf_eval: channel not 0..2");
    }
    if (n == 0) return Ok();
    Buffers b;
    TabBssrdf tab;
    MakeDeviceBssrdf(table, sigma_a, sigma_s, eta, b, tab);
    const size_t un = static_cast<size_t>(n);
    const int32_t* dc = b.Upload(channels, un);
    const float* du = b.Upload(u, un);
    const float* dr = b.Upload(r, un);
    float* ds = b.Alloc<float>(un);
    float* dp = b.Alloc<float>(un);
    float* dsr = b.Alloc<float>(3 * un);
    cudaError_t err = b.err;
    if (err == cudaSuccess) {
        BssrdfEvalKernel<<<Blocks(n), 256>>>(tab, dc, du, dr, n, ds, dp, dsr);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemcpy(sample_r, ds, un * sizeof(float), cudaMemcpyDeviceToHost);
    if (err == cudaSuccess) err = cudaMemcpy(pdf_sr, dp, un * sizeof(float), cudaMemcpyDeviceToHost);
    if (err == cudaSuccess) err = cudaMemcpy(sr, dsr, 3 * un * sizeof(float), cudaMemcpyDeviceToHost);
    return Done(err, "yrc_bssrdf_eval");
}

yrc_status yrc_bssrdf_pdf_sp(const yrc_bssrdf_table* table, const float sigma_a[3], const float sigma_s[3], float eta,
                             const float* queries, int64_t n, float* pdf) {
    using namespace yrc;
    if (!TableValid(table) || !sigma_a || !sigma_s || n < 0 || (n > 0 && (!queries || !pdf))) {
        return Fail(YRC_ERR_INVALID_ARGUMENT, "yrc_bssrdf_pdf_sp: bad argument");
    }
    if (n == 0) return Ok();
    Buffers b;
    TabBssrdf tab;
    MakeDeviceBssrdf(table, sigma_a, sigma_s, eta, b, tab);
    const size_t un = static_cast<size_t>(n);
    const float* dq = b.Upload(queries, 18 * un);
    float* dp = b.Alloc<float>(un);
    cudaError_t err = b.err;
    if (err == cudaSuccess) {
        BssrdfPdfSpKernel<<<Blocks(n), 256>>>(tab, dq, n, dp);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemcpy(pdf, dp, un * sizeof(float), cudaMemcpyDeviceToHost);
    return Done(err, "yrc_bssrdf_pdf_sp");
}

}  // extern "C"
