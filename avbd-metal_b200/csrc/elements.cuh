// elements.cuh — device helpers shared by the element-contact pipelines
// (Planar-DAT in cloth.cu, isotropic OGC in ogc.cu): closest-point queries,
// sorted-neighbourhood membership, the soft persistence map lookup and the
// soft-contact record writer.
//
// Follows Shaders/25_cloth.metal (closestPtTriangle :27-63, softKeyHash /
// softMapFind :79-99, softEmit :269-333, eeClosestSegSeg :632-648).
#pragma once
#include "../../include/avbd.h"
#include "dmath.cuh"
#include "kernels.h"

namespace avbd {
namespace {

constexpr float DAT_GEOMETRY_EPS = 1.0e-8f;
constexpr float DAT_TIME_MARGIN = 1.0e-3f;
constexpr float EE_INTERIOR_EPS = 0.02f;
constexpr float FLT_BIG_ = 3.402823466e38f;

struct I3 { int x, y, z; };

__device__ __forceinline__ I3 cell_of(float3 p, float cs) {
    return I3{(int)floorf(p.x / cs), (int)floorf(p.y / cs), (int)floorf(p.z / cs)};
}
__device__ __forceinline__ uint32_t elem_hash(I3 c, uint32_t size) { return cell_hash(c.x, c.y, c.z, 0u, size); }
__device__ __forceinline__ I3 imin3(I3 a, I3 b) { return I3{min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)}; }
__device__ __forceinline__ I3 imax3(I3 a, I3 b) { return I3{max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)}; }
__device__ __forceinline__ I3 iadd(I3 a, int s) { return I3{a.x + s, a.y + s, a.z + s}; }
__device__ __forceinline__ float3 vmin(float3 a, float3 b) { return mk3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
__device__ __forceinline__ float3 vmax(float3 a, float3 b) { return mk3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }

// Closest point on a triangle (Ericson 5.1.5; 25_cloth.metal:27-63).
__device__ float3 closest_pt_triangle(float3 p, float3 a, float3 b, float3 c, float3& bary) {
    const float3 ab = b - a, ac = c - a, ap = p - a;
    const float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) { bary = mk3(1, 0, 0); return a; }
    const float3 bp = p - b;
    const float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) { bary = mk3(0, 1, 0); return b; }
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        const float v = d1 / mx(d1 - d3, 1e-12f);
        bary = mk3(1 - v, v, 0);
        return a + ab * v;
    }
    const float3 cp = p - c;
    const float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) { bary = mk3(0, 0, 1); return c; }
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        const float w = d2 / mx(d2 - d6, 1e-12f);
        bary = mk3(1 - w, 0, w);
        return a + ac * w;
    }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        const float w = (d4 - d3) / mx((d4 - d3) + (d5 - d6), 1e-12f);
        bary = mk3(0, 1 - w, w);
        return b + (c - b) * w;
    }
    const float denom = va + vb + vc;
    if (fabsf(denom) < 1e-20f) { bary = mk3(1, 0, 0); return a; }
    const float v = vb / denom, w = vc / denom;
    bary = mk3(1 - v - w, v, w);
    return a + ab * v + ac * w;
}

// Closest parameters of two segments (25_cloth.metal:632-648).
__device__ void closest_seg_seg(float3 p0, float3 p1, float3 q0, float3 q1, float& s, float& t) {
    const float3 d1 = p1 - p0, d2 = q1 - q0, r = p0 - q0;
    const float a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    s = 0.0f;
    t = 0.0f;
    if (a <= 1e-12f && e <= 1e-12f) return;
    if (a <= 1e-12f) { t = clampf(f / e, 0.0f, 1.0f); return; }
    const float c = dot(d1, r);
    if (e <= 1e-12f) { s = clampf(-c / a, 0.0f, 1.0f); return; }
    const float b = dot(d1, d2);
    const float denom = a * e - b * b;
    if (fabsf(denom) > 1e-12f) s = clampf((b * f - c * e) / denom, 0.0f, 1.0f);
    t = (b * s + f) / e;
    if (t < 0.0f) { t = 0.0f; s = clampf(-c / a, 0.0f, 1.0f); }
    else if (t > 1.0f) { t = 1.0f; s = clampf((b - c) / a, 0.0f, 1.0f); }
}

__device__ __forceinline__ bool nbr_contains(const uint32_t* list, uint32_t s, uint32_t e, uint32_t x) {
    uint32_t lo = s, hi = e;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (list[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo < e && list[lo] == x;
}

__device__ __forceinline__ bool pair_excluded(const DevPtrs& d, uint32_t n, uint32_t a, uint32_t b) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t ex = d.exclusions[2 * mid], ey = d.exclusions[2 * mid + 1];
        if (ex < a || (ex == a && ey < b)) lo = mid + 1; else hi = mid;
    }
    return lo < n && d.exclusions[2 * lo] == a && d.exclusions[2 * lo + 1] == b;
}

__device__ __forceinline__ uint32_t soft_key_hash(uint32_t a, uint32_t b, uint32_t cap) {
    uint32_t h = (a * 0x9E3779B1u) ^ (b * 0x85EBCA77u);
    h ^= h >> 16;
    h *= 0xC2B2AE3Du;
    h ^= h >> 13;
    return h & (cap - 1u);
}

__device__ int soft_map_find(const Params& P, const DevPtrs& d, uint32_t keyA, uint32_t keyB) {
    uint32_t h = soft_key_hash(keyA, keyB, P.softMapCapacity);
    for (uint32_t probe = 0; probe < 64; probe++) {
        const uint32_t ka = d.softKeyA[h];
        if (ka == 0u) return -1;
        if (ka == keyA + 1u && d.softKeyB[h] == keyB) return (int)d.softVal[h];
        h = (h + 1u) & (P.softMapCapacity - 1u);
    }
    return -1;
}

__device__ float soft_prev_side(const Params& P, const DevPtrs& d, uint32_t keyA, uint32_t keyB, float proposed) {
    const int prev = soft_map_find(P, d, keyA, keyB);
    if (prev < 0) return proposed;
    const uint32_t flags = __float_as_uint(d.prevSoft[prev].anchorA.w);
    return (flags & SCF_SIDE_NEG) ? -1.0f : 1.0f;
}

__device__ __forceinline__ float soft_lambda_cap(const Params& P, float minMass) {
    return mn(P.lambdaMax, mx(10.0f, 1.0e5f * minMass));
}

// Warm start from the persistence map and write one record
// (softEmit, 25_cloth.metal:273-333).
__device__ void soft_write(const Params& P, const DevPtrs& d, uint32_t slot, uint4 ids, float4 weights, float3 n,
                           float friction, float3 anchorA, float C0n, float restT, float lamCap, float minMass,
                           uint32_t kind, bool rigidA, bool roundA, bool sideNeg, uint32_t keyA, uint32_t keyB) {
    float3 lam = s3(0), pen = s3(0);
    const int prev = soft_map_find(P, d, keyA, keyB);
    if (prev >= 0) {
        const SoftContactGPU& o = d.prevSoft[prev];
        lam = xyz(o.lambda) * (P.alpha * P.gamma);
        pen = xyz(o.penalty);
        float3 t1o, t2o, t1n, t2n;
        orthonormal(xyz(o.normal), t1o, t2o);
        orthonormal(n, t1n, t2n);
        const float3 lt = t1o * lam.y + t2o * lam.z;
        lam.y = dot(t1n, lt);
        lam.z = dot(t2n, lt);
    }
    const float penFloor = mx(PENALTY_MIN, minMass / (P.dt * P.dt));
    pen = clamp3(pen * P.gamma, s3(penFloor), s3(PENALTY_MAX));
    if (slot >= P.maxSoft) return;
    const uint32_t flags = (rigidA ? SCF_RIGID_A : 0u) | (sideNeg ? SCF_SIDE_NEG : 0u) | (kind << SCF_KIND_SHIFT) |
                           (roundA ? SCF_ROUND_A : 0u);
    SoftContactGPU& sc = d.soft[slot];
    sc.ids = u4{ids.x, ids.y, ids.z, ids.w};
    sc.normal = tof4(n, friction);
    sc.anchorA = tof4(rigidA ? anchorA : mk3(restT, 0, 0), __uint_as_float(flags));
    sc.weights = tof4(weights);
    sc.C0 = f4{C0n, 0.0f, 0.0f, lamCap};
    sc.lambda = tof4(lam, __uint_as_float(keyA));
    sc.penalty = tof4(pen, __uint_as_float(keyB));
}

}  // namespace
}  // namespace avbd
