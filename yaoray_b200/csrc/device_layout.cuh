// Device-resident traversal layout and the exact ray/box, ray/triangle and
// ray/sphere tests of the reference, for sm_100a.
//
// Layout (all 16-byte aligned, fetched with 128-bit read-only loads):
//
//  NodePair (64 B): one per INTERIOR node of the reference's binary BVH. It
//    holds both children's boxes, so visiting an interior node is one 64-byte
//    fetch instead of two 32-byte fetches at unrelated addresses (left child
//    at index+1, right child at payload_offset in RenderBvhNode).
//      a = (L.lo.x, L.lo.y, L.lo.z, L.hi.x)   b = (L.hi.y, L.hi.z, R.lo.x, R.lo.y)
//      c = (R.lo.z, R.hi.x, R.hi.y, R.hi.z)   d = (L.ref, R.ref, -, -)
//    A child ref >= 0 is the child's NodePair index, kLeafBit|... (negative)
//    is a leaf: ~first_record; kAbsentRef marks a child the reference would
//    not test (index outside the node array).
//
//  Record (48 B): one per leaf primitive slot, in leaf order, so a leaf is a
//    contiguous record run whose last entry carries kLast. A triangle stores
//    p0 and the edges p1-p0, p2-p0 exactly as the reference computes them
//    (IEEE subtraction is deterministic, so precomputing them changes no bit):
//      v0 = (p0.xyz, id)   v1 = (e1.xyz, flags)   v2 = (e2.xyz, mesh primitive)
//    A sphere stores (center.xyz, sphere index), (radius, 0, 0, flags).
//    In a TLAS an instance record stores (0,0,0, instance index), flags.
//
//  Instance (80 B, two-level only): the reference's world_to_object rows in
//    TransformPoint order plus the BLAS root box and root ref.
#pragma once

#include <cstdint>
#include <cstring>

#include <cuda_runtime.h>

#include "yrc_math_host.hpp"

namespace yrc {

// Bit casts usable in host code (the device has __int_as_float etc.).
inline float IntBits(int32_t i) {
    float f;
    std::memcpy(&f, &i, sizeof(f));
    return f;
}
inline int32_t FloatBits(float f) {
    int32_t i;
    std::memcpy(&i, &f, sizeof(i));
    return i;
}

constexpr int32_t kAbsentRef = INT32_MIN;

// Record kinds (flags bits 1..3).
enum RecordKind : int32_t {
    kRecTriangle = 0,
    kRecSphere = 1,
    kRecSkipCountTriangle = 2,  // slot counted as a triangle test, never hits
    kRecSkipCountSphere = 3,    // slot counted as a sphere test, never hits
    kRecSkip = 4,               // slot skipped without a count
    kRecInstance = 5,           // TLAS: descend into an instance's BLAS
};
constexpr int32_t kRecLast = 1;  // flags bit 0: last record of its leaf

struct alignas(16) NodePair {
    float4 a, b, c;
    int4 d;
};
static_assert(sizeof(NodePair) == 64, "NodePair must be 64 bytes");

// Four-wide node collapsed from the binary pairs (flat, triangle-only BVHs):
// child boxes in SoA form (lo x / hi x / lo y / hi y / lo z / hi z of the
// four children), child refs (wide node index, ~record for a leaf, or
// kAbsentRef), padded to one 128-byte line. The boxes are the binary tree's
// own node boxes, so the same slab tests run on them; the binary nodes that
// the collapse skips contain their children, and the slab test's rounding is
// monotone, so a box that passes implies that every skipped ancestor passes.
struct alignas(16) WideNode {
    float4 lox, hix, loy, hiy, loz, hiz;
    int4 ref;
    float4 pad;
};
static_assert(sizeof(WideNode) == 128, "WideNode must be 128 bytes");

struct alignas(16) Record {
    float4 v0, v1, v2;
};
static_assert(sizeof(Record) == 48, "Record must be 48 bytes");

struct alignas(16) Instance {
    float4 row0, row1, row2;  // (m[r], m[4+r], m[8+r], m[12+r]) of world_to_object
    float4 box_a;             // BLAS root lo.xyz, hi.x
    float4 box_b;             // hi.y, hi.z, root ref (int bits), BLAS root is a leaf (unused)
};
static_assert(sizeof(Instance) == 80, "Instance must be 80 bytes");

// Everything a trace kernel needs, passed by value.
struct AccelParams {
    const NodePair* pairs;
    const Record* records;
    const Instance* instances;
    float root_lo[3];
    float root_hi[3];
    int32_t root_ref;     // kAbsentRef for an empty BVH
    int32_t two_level;    // 1: records at the root level are TLAS records
    int32_t stack_limit;  // deepest stack the traversal may need (host-computed)
    const WideNode* wide;      // four-wide copy of a flat triangle-only BVH, or nullptr
    int32_t wide_root;         // wide node index, ~record (leaf root) or kAbsentRef
    int32_t wide_stack_limit;  // deepest stack of the four-wide traversal
};

#if defined(__CUDACC__)

// RayBoundsPrecompute (include/yaoray/core/bounds.hpp:50-66).
struct RayPre {
    float o[3];
    float d[3];
    float inv[3];
    unsigned neg;  // bit a: signbit(inv[a])
};

__device__ __forceinline__ void Precompute(RayPre& r) {
    r.neg = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        r.inv[a] = __frcp_rn(r.d[a]);  // IEEE 1.0f / d
        r.neg |= (__float_as_uint(r.inv[a]) >> 31) << a;
    }
}

// IntersectBounds (bounds.hpp:68-90): comparison-select updates keep the
// interval on a NaN (0 * inf on a slab plane), inclusive t_max >= t_min.
__device__ __forceinline__ bool SlabTest(const RayPre& r, float lx, float ly, float lz, float hx, float hy,
                                         float hz, float tmin, float tmax, float& entry) {
    const float lo[3] = {lx, ly, lz};
    const float hi[3] = {hx, hy, hz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const bool n = (r.neg >> a) & 1u;
        const float nb = n ? hi[a] : lo[a];
        const float fb = n ? lo[a] : hi[a];
        const float an = __fmul_rn(__fsub_rn(nb, r.o[a]), r.inv[a]);
        const float af = __fmul_rn(__fsub_rn(fb, r.o[a]), r.inv[a]);
        tmin = an > tmin ? an : tmin;
        tmax = af < tmax ? af : tmax;
    }
    entry = tmin;
    return tmax >= tmin;
}

// SlabTest for an interval that holds no NaN, which is the case for every
// box test after the root box passed SlabTest: a NaN ray t_min or t_max
// fails that test (no comparison with it holds), and the interval then only
// takes values that compared in order. With NaN-free bounds, fmaxf / fminf
// give the comparison-selects' results: a NaN plane distance leaves the
// bound unchanged in both forms, and where they differ in the sign of a zero
// no later comparison (t_max >= t_min, the entry orders, the stack culls)
// changes. One min / max instruction per update instead of a compare and a
// select.
__device__ __forceinline__ bool SlabTestInterval(const RayPre& r, float lx, float ly, float lz, float hx, float hy,
                                                 float hz, float tmin, float tmax, float& entry) {
    const float lo[3] = {lx, ly, lz};
    const float hi[3] = {hx, hy, hz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const bool n = (r.neg >> a) & 1u;
        const float nb = n ? hi[a] : lo[a];
        const float fb = n ? lo[a] : hi[a];
        const float an = __fmul_rn(__fsub_rn(nb, r.o[a]), r.inv[a]);
        const float af = __fmul_rn(__fsub_rn(fb, r.o[a]), r.inv[a]);
        tmin = fmaxf(an, tmin);
        tmax = fminf(af, tmax);
    }
    entry = tmin;
    return tmax >= tmin;
}

// Dot / Cross in the reference's order (include/yaoray/core/vec.hpp:155-165).
__device__ __forceinline__ float Dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return __fadd_rn(__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), __fmul_rn(az, bz));
}

// Closest-hit candidate state (the reference's BvhHit "nearest").
struct Nearest {
    float t;
    int32_t id;    // flat triangle index, -2 - sphere, or -1
    int32_t prim;  // mesh primitive of a triangle hit, else -1
    float u, v;
    bool hit;
};

// IntersectTriangle (src/accel/bvh_traversal.cpp:52-121): Moller-Trumbore with
// |det| < 1e-8 rejection, u in [0,1], v >= 0, u+v <= 1, t in (t_min, nearest.t]
// and the equal-t tie broken toward the smaller flat_triangle_index.
// Returns true when the candidate was accepted.
__device__ __forceinline__ bool TriangleTest(const RayPre& r, const float4 v0, const float4 v1, const float4 v2,
                                             float tmin, Nearest& best) {
    const float e1x = v1.x, e1y = v1.y, e1z = v1.z;
    const float e2x = v2.x, e2y = v2.y, e2z = v2.z;
    // pvec = Cross(d, e2)
    const float px = __fsub_rn(__fmul_rn(r.d[1], e2z), __fmul_rn(r.d[2], e2y));
    const float py = __fsub_rn(__fmul_rn(r.d[2], e2x), __fmul_rn(r.d[0], e2z));
    const float pz = __fsub_rn(__fmul_rn(r.d[0], e2y), __fmul_rn(r.d[1], e2x));
    const float det = Dot3(e1x, e1y, e1z, px, py, pz);
    if (fabsf(det) < 1.0e-8f) return false;
    const float inv_det = __frcp_rn(det);
    const float tx = __fsub_rn(r.o[0], v0.x);
    const float ty = __fsub_rn(r.o[1], v0.y);
    const float tz = __fsub_rn(r.o[2], v0.z);
    const float u = __fmul_rn(Dot3(tx, ty, tz, px, py, pz), inv_det);
    if (u < 0.0f || u > 1.0f) return false;
    // qvec = Cross(tvec, e1)
    const float qx = __fsub_rn(__fmul_rn(ty, e1z), __fmul_rn(tz, e1y));
    const float qy = __fsub_rn(__fmul_rn(tz, e1x), __fmul_rn(tx, e1z));
    const float qz = __fsub_rn(__fmul_rn(tx, e1y), __fmul_rn(ty, e1x));
    const float v = __fmul_rn(Dot3(r.d[0], r.d[1], r.d[2], qx, qy, qz), inv_det);
    if (v < 0.0f || __fadd_rn(u, v) > 1.0f) return false;
    const float t = __fmul_rn(Dot3(e2x, e2y, e2z, qx, qy, qz), inv_det);
    if (t <= tmin || t > best.t) return false;
    const int32_t id = __float_as_int(v0.w);
    if (t == best.t && best.hit && best.id >= 0 && id >= best.id) return false;
    best.hit = true;
    best.t = t;
    best.id = id;
    best.prim = __float_as_int(v2.w);
    best.u = u;
    best.v = v;
    return true;
}

// IntersectSphere (src/geometry/intersection.cpp:108-128) followed by the
// caller's strict `hit.t >= nearest.t` rejection and SphereUv
// (intersection.cpp:145-151). t is bit-exact (IEEE sqrt and divide); the UV
// uses CUDA's atan2f/acosf, which may differ from the host libm in the last ulp.
__device__ __forceinline__ bool SphereTest(const RayPre& r, const float4 v0, const float4 v1, float tmin,
                                           Nearest& best) {
    const float ocx = __fsub_rn(r.o[0], v0.x);
    const float ocy = __fsub_rn(r.o[1], v0.y);
    const float ocz = __fsub_rn(r.o[2], v0.z);
    const float radius = v1.x;
    const float a = Dot3(r.d[0], r.d[1], r.d[2], r.d[0], r.d[1], r.d[2]);
    const float b = __fmul_rn(2.0f, Dot3(ocx, ocy, ocz, r.d[0], r.d[1], r.d[2]));
    const float c = __fsub_rn(Dot3(ocx, ocy, ocz, ocx, ocy, ocz), __fmul_rn(radius, radius));
    const float disc = __fsub_rn(__fmul_rn(b, b), __fmul_rn(__fmul_rn(4.0f, a), c));
    if (disc < 0.0f) return false;
    const float sq = __fsqrt_rn(disc);
    const float inv_2a = __fdiv_rn(0.5f, a);
    const float tmax = best.t;
    float t = __fmul_rn(__fsub_rn(-b, sq), inv_2a);
    if (!(t > tmin && t < tmax)) {
        t = __fmul_rn(__fadd_rn(-b, sq), inv_2a);
        if (!(t > tmin && t < tmax)) return false;
    }
    if (t >= best.t) return false;
    // hit point = origin + direction * t; normal = Normalize(hit - center)
    const float hx = __fadd_rn(r.o[0], __fmul_rn(r.d[0], t));
    const float hy = __fadd_rn(r.o[1], __fmul_rn(r.d[1], t));
    const float hz = __fadd_rn(r.o[2], __fmul_rn(r.d[2], t));
    float nx = __fsub_rn(hx, v0.x), ny = __fsub_rn(hy, v0.y), nz = __fsub_rn(hz, v0.z);
    const float len = __fsqrt_rn(Dot3(nx, ny, nz, nx, ny, nz));
    if (len > 0.0f) {
        nx = __fdiv_rn(nx, len);
        ny = __fdiv_rn(ny, len);
        nz = __fdiv_rn(nz, len);
    } else {
        nx = ny = nz = 0.0f;
    }
    const float pi = 3.14159265358979323846f;
    const float cy = fminf(fmaxf(ny, -1.0f), 1.0f);
    best.hit = true;
    best.t = t;
    best.id = -2 - __float_as_int(v0.w);
    best.prim = -1;
    best.u = __fdiv_rn(__fadd_rn(atan2f(nx, nz), pi), __fmul_rn(2.0f, pi));
    best.v = __fdiv_rn(__fsub_rn(pi, acosf(cy)), pi);
    return true;
}

#endif  // __CUDACC__

}  // namespace yrc
