// Reference-order float arithmetic usable from host C++ and CUDA device code.
//
// Bit-exact parity with the reference CPU build requires (a) the same
// expression order and (b) no fused multiply-add: the reference is compiled
// for baseline x86-64 (SSE2), which has no FMA, so every a*b+c rounds twice.
// On the device each operation therefore goes through an explicitly rounded
// intrinsic (__fmul_rn etc. are never contracted by nvcc); on the host the
// translation units are compiled with -ffp-contract=off.
#pragma once

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define YRC_HD __host__ __device__ __forceinline__
#else
#define YRC_HD inline
#endif

#if defined(__CUDA_ARCH__)
#define YRC_MUL(a, b) __fmul_rn((a), (b))
#define YRC_ADD(a, b) __fadd_rn((a), (b))
#define YRC_SUB(a, b) __fsub_rn((a), (b))
#define YRC_DIV(a, b) __fdiv_rn((a), (b))
#define YRC_RCP(a) __frcp_rn(a)
#else
#define YRC_MUL(a, b) ((a) * (b))
#define YRC_ADD(a, b) ((a) + (b))
#define YRC_SUB(a, b) ((a) - (b))
#define YRC_DIV(a, b) ((a) / (b))
#define YRC_RCP(a) (1.0f / (a))
#endif

namespace yrc {

// TransformPoint (src/core/transform.cpp:30-36): column-major, evaluated
// left to right: ((m0*x + m4*y) + m8*z) + m12.
YRC_HD void TransformPointRef(const float* m, const float* p, float* out) {
    for (int r = 0; r < 3; ++r) {
        float acc = YRC_ADD(YRC_MUL(m[r], p[0]), YRC_MUL(m[4 + r], p[1]));
        acc = YRC_ADD(acc, YRC_MUL(m[8 + r], p[2]));
        out[r] = YRC_ADD(acc, m[12 + r]);
    }
}

// TransformVector (transform.cpp:38-44): no translation.
YRC_HD void TransformVectorRef(const float* m, const float* v, float* out) {
    for (int r = 0; r < 3; ++r) {
        const float acc = YRC_ADD(YRC_MUL(m[r], v[0]), YRC_MUL(m[4 + r], v[1]));
        out[r] = YRC_ADD(acc, YRC_MUL(m[8 + r], v[2]));
    }
}

// IsInvertibleAffine (src/accel/two_level_bvh.cpp:27-36): all entries finite
// and |det(upper 3x3)| > 1e-12 with the reference's cofactor order.
inline bool IsInvertibleAffineRef(const float* m) {
    for (int i = 0; i < 16; ++i) {
        if (!std::isfinite(m[i])) return false;
    }
    const float det = m[0] * (m[5] * m[10] - m[9] * m[6]) - m[4] * (m[1] * m[10] - m[9] * m[2]) +
                      m[8] * (m[1] * m[6] - m[5] * m[2]);
    return std::isfinite(det) && std::fabs(det) > 1.0e-12f;
}

// Inverse (src/core/transform.cpp:147-197): 4x4 adjugate / determinant with
// the cofactor sums written in the reference's term order; identity when
// |det| <= 1e-12. The term order is part of the contract: world_to_object is
// used by the two-level traversal and must match bit for bit.
inline void InverseRef(const float* a, float* o) {
    o[0] = a[5] * a[10] * a[15] - a[5] * a[11] * a[14] - a[9] * a[6] * a[15] + a[9] * a[7] * a[14] +
           a[13] * a[6] * a[11] - a[13] * a[7] * a[10];
    o[4] = -a[4] * a[10] * a[15] + a[4] * a[11] * a[14] + a[8] * a[6] * a[15] - a[8] * a[7] * a[14] -
           a[12] * a[6] * a[11] + a[12] * a[7] * a[10];
    o[8] = a[4] * a[9] * a[15] - a[4] * a[11] * a[13] - a[8] * a[5] * a[15] + a[8] * a[7] * a[13] +
           a[12] * a[5] * a[11] - a[12] * a[7] * a[9];
    o[12] = -a[4] * a[9] * a[14] + a[4] * a[10] * a[13] + a[8] * a[5] * a[14] - a[8] * a[6] * a[13] -
            a[12] * a[5] * a[10] + a[12] * a[6] * a[9];
    o[1] = -a[1] * a[10] * a[15] + a[1] * a[11] * a[14] + a[9] * a[2] * a[15] - a[9] * a[3] * a[14] -
           a[13] * a[2] * a[11] + a[13] * a[3] * a[10];
    o[5] = a[0] * a[10] * a[15] - a[0] * a[11] * a[14] - a[8] * a[2] * a[15] + a[8] * a[3] * a[14] +
           a[12] * a[2] * a[11] - a[12] * a[3] * a[10];
    o[9] = -a[0] * a[9] * a[15] + a[0] * a[11] * a[13] + a[8] * a[1] * a[15] - a[8] * a[3] * a[13] -
           a[12] * a[1] * a[11] + a[12] * a[3] * a[9];
    o[13] = a[0] * a[9] * a[14] - a[0] * a[10] * a[13] - a[8] * a[1] * a[14] + a[8] * a[2] * a[13] +
            a[12] * a[1] * a[10] - a[12] * a[2] * a[9];
    o[2] = a[1] * a[6] * a[15] - a[1] * a[7] * a[14] - a[5] * a[2] * a[15] + a[5] * a[3] * a[14] +
           a[13] * a[2] * a[7] - a[13] * a[3] * a[6];
    o[6] = -a[0] * a[6] * a[15] + a[0] * a[7] * a[14] + a[4] * a[2] * a[15] - a[4] * a[3] * a[14] -
           a[12] * a[2] * a[7] + a[12] * a[3] * a[6];
    o[10] = a[0] * a[5] * a[15] - a[0] * a[7] * a[13] - a[4] * a[1] * a[15] + a[4] * a[3] * a[13] +
            a[12] * a[1] * a[7] - a[12] * a[3] * a[5];
    o[14] = -a[0] * a[5] * a[14] + a[0] * a[6] * a[13] + a[4] * a[1] * a[14] - a[4] * a[2] * a[13] -
            a[12] * a[1] * a[6] + a[12] * a[2] * a[5];
    o[3] = -a[1] * a[6] * a[11] + a[1] * a[7] * a[10] + a[5] * a[2] * a[11] - a[5] * a[3] * a[10] -
           a[9] * a[2] * a[7] + a[9] * a[3] * a[6];
    o[7] = a[0] * a[6] * a[11] - a[0] * a[7] * a[10] - a[4] * a[2] * a[11] + a[4] * a[3] * a[10] +
           a[8] * a[2] * a[7] - a[8] * a[3] * a[6];
    o[11] = -a[0] * a[5] * a[11] + a[0] * a[7] * a[9] + a[4] * a[1] * a[11] - a[4] * a[3] * a[9] -
            a[8] * a[1] * a[7] + a[8] * a[3] * a[5];
    o[15] = a[0] * a[5] * a[10] - a[0] * a[6] * a[9] - a[4] * a[1] * a[10] + a[4] * a[2] * a[9] +
            a[8] * a[1] * a[6] - a[8] * a[2] * a[5];
    const float det = a[0] * o[0] + a[1] * o[4] + a[2] * o[8] + a[3] * o[12];
    if (std::fabs(det) <= 1.0e-12f) {
        for (int i = 0; i < 16; ++i) o[i] = (i % 5 == 0) ? 1.0f : 0.0f;
        return;
    }
    const float inv_det = 1.0f / det;
    for (int i = 0; i < 16; ++i) o[i] *= inv_det;
}

}  // namespace yrc
