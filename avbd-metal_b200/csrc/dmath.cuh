// dmath.cuh — float32 vector, quaternion and 3x3 helpers for the solver
// kernels (the device side of 00_common.metal:50-228 of the reference).
//
// The solver kernels are compiled with -fmad=false and IEEE division/sqrt,
// and every helper below evaluates its terms in one fixed order, so a frame
// computed here is reproducible bit for bit and agrees with a serial float32
// evaluation of the same expressions.
#pragma once
#include <cstdint>
#include "avbd_types.h"

namespace avbd {

struct M3 { float3 r0, r1, r2; };

__device__ __forceinline__ float3 mk3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 s3(float s) { return make_float3(s, s, s); }
__device__ __forceinline__ float3 xyz(float4 v) { return make_float3(v.x, v.y, v.z); }
__device__ __forceinline__ float3 xyz(f4 v) { return make_float3(v.x, v.y, v.z); }
__device__ __forceinline__ float4 mk4(float3 v, float w) { return make_float4(v.x, v.y, v.z, w); }
__device__ __forceinline__ float4 tof(f4 v) { return make_float4(v.x, v.y, v.z, v.w); }
__device__ __forceinline__ f4 tof4(float4 v) { return f4{v.x, v.y, v.z, v.w}; }
__device__ __forceinline__ f4 tof4(float3 v, float w) { return f4{v.x, v.y, v.z, w}; }

__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return mk3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return mk3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return mk3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 operator/(float3 a, float s) { return mk3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float3& operator+=(float3& a, float3 b) { a = a + b; return a; }
__device__ __forceinline__ float3& operator-=(float3& a, float3 b) { a = a - b; return a; }
__device__ __forceinline__ float3& operator*=(float3& a, float s) { a = a * s; return a; }
__device__ __forceinline__ float4 operator+(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ float4 operator*(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
__device__ __forceinline__ float4 operator/(float4 a, float s) { return make_float4(a.x / s, a.y / s, a.z / s, a.w / s); }
__device__ __forceinline__ float4 neg4(float4 a) { return make_float4(-a.x, -a.y, -a.z, -a.w); }

// Ordered min/max/clamp with explicit comparisons (NaN falls to the second arm).
__device__ __forceinline__ float mn(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float mx(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return mn(mx(x, lo), hi); }
__device__ __forceinline__ float3 mn3(float3 a, float3 b) { return mk3(mn(a.x, b.x), mn(a.y, b.y), mn(a.z, b.z)); }
__device__ __forceinline__ float3 mx3(float3 a, float3 b) { return mk3(mx(a.x, b.x), mx(a.y, b.y), mx(a.z, b.z)); }
__device__ __forceinline__ float3 clamp3(float3 v, float3 lo, float3 hi) { return mn3(mx3(v, lo), hi); }
__device__ __forceinline__ float3 abs3(float3 v) { return mk3(fabsf(v.x), fabsf(v.y), fabsf(v.z)); }
__device__ __forceinline__ float comp(float3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
__device__ __forceinline__ void setcomp(float3& v, int i, float s) { if (i == 0) v.x = s; else if (i == 1) v.y = s; else v.z = s; }

__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float dot4(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
    return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// 1/sqrt with IEEE division and square root (not the approximate rsqrt).
__device__ __forceinline__ float rsq(float x) { return 1.0f / sqrtf(x); }
__device__ __forceinline__ float len3(float3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ float dist3(float3 a, float3 b) { return len3(a - b); }
__device__ __forceinline__ float dist2(float3 a, float3 b) { float3 d = a - b; return dot(d, d); }
__device__ __forceinline__ float3 nrm3(float3 a) { return a * rsq(dot(a, a)); }
__device__ __forceinline__ float4 nrm4(float4 a) { return a * rsq(dot4(a, a)); }

__device__ __forceinline__ bool finite_bits(float x) { return (__float_as_uint(x) & 0x7F800000u) != 0x7F800000u; }
__device__ __forceinline__ bool finite3(float3 v) { return finite_bits(v.x) && finite_bits(v.y) && finite_bits(v.z); }

__device__ __forceinline__ M3 m3_zero() { return M3{s3(0), s3(0), s3(0)}; }
__device__ __forceinline__ M3 m3_diag(float3 d) { return M3{mk3(d.x, 0, 0), mk3(0, d.y, 0), mk3(0, 0, d.z)}; }
__device__ __forceinline__ M3 m3_identity() { return m3_diag(s3(1)); }
__device__ __forceinline__ float3 m3_mul(const M3& m, float3 v) { return mk3(dot(m.r0, v), dot(m.r1, v), dot(m.r2, v)); }
__device__ __forceinline__ float3 m3_col(const M3& m, int i) { return mk3(comp(m.r0, i), comp(m.r1, i), comp(m.r2, i)); }
__device__ __forceinline__ M3 m3_transpose(const M3& m) { return M3{m3_col(m, 0), m3_col(m, 1), m3_col(m, 2)}; }
__device__ __forceinline__ M3 m3_mulm(const M3& a, const M3& b) {
    M3 bt = m3_transpose(b);
    return M3{mk3(dot(a.r0, bt.r0), dot(a.r0, bt.r1), dot(a.r0, bt.r2)),
              mk3(dot(a.r1, bt.r0), dot(a.r1, bt.r1), dot(a.r1, bt.r2)),
              mk3(dot(a.r2, bt.r0), dot(a.r2, bt.r1), dot(a.r2, bt.r2))};
}
__device__ __forceinline__ M3 m3_add(const M3& a, const M3& b) { return M3{a.r0 + b.r0, a.r1 + b.r1, a.r2 + b.r2}; }
__device__ __forceinline__ M3 m3_scale(const M3& a, float s) { return M3{a.r0 * s, a.r1 * s, a.r2 * s}; }
__device__ __forceinline__ M3 m3_outer(float3 a, float3 b) { return M3{b * a.x, b * a.y, b * a.z}; }
__device__ __forceinline__ M3 m3_skew(float3 r) { return M3{mk3(0, -r.z, r.y), mk3(r.z, 0, -r.x), mk3(-r.y, r.x, 0)}; }
__device__ __forceinline__ M3 m3_diagonalize(const M3& m) {
    return m3_diag(mk3(len3(m3_col(m, 0)), len3(m3_col(m, 1)), len3(m3_col(m, 2))));
}

// Quaternions: (x, y, z) imaginary, w real.
__device__ __forceinline__ float4 q_mul(float4 a, float4 b) {
    return make_float4(a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
                       a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
                       a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w,
                       a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z);
}
__device__ __forceinline__ float4 q_conj(float4 q) { return make_float4(-q.x, -q.y, -q.z, q.w); }
__device__ __forceinline__ float4 q_inv(float4 q) { return q_conj(q) / dot4(q, q); }
__device__ __forceinline__ float3 q_rotate(float4 q, float3 v) {
    float3 u = xyz(q);
    float3 t = 2.0f * cross(u, v);
    return v + q.w * t + cross(u, t);
}
__device__ __forceinline__ M3 world_inertia(float4 q, float3 p) {
    float3 c0 = q_rotate(q, mk3(1, 0, 0));
    float3 c1 = q_rotate(q, mk3(0, 1, 0));
    float3 c2 = q_rotate(q, mk3(0, 0, 1));
    return m3_add(m3_add(m3_scale(m3_outer(c0, c0), p.x), m3_scale(m3_outer(c1, c1), p.y)),
                  m3_scale(m3_outer(c2, c2), p.z));
}
// Tangent-space difference, canonicalised to w >= 0.
__device__ __forceinline__ float3 q_sub(float4 a, float4 b) {
    float4 r = q_mul(a, q_inv(b));
    if (r.w < 0.0f) r = neg4(r);
    return xyz(r) * 2.0f;
}
__device__ __forceinline__ float4 q_addw(float4 q, float3 w) {
    float4 dq = q_mul(mk4(w, 0.0f), q);
    return nrm4(q + dq * 0.5f);
}
__device__ __forceinline__ float3 xform(float3 p, float4 q, float3 v) { return q_rotate(q, v) + p; }

// Jacobi-preconditioned, pivot-clamped LDL^T solve of the 6x6 block system
// [aLin aCross^T; aCross aAng] x = b.
__device__ __forceinline__ void solve6x6(const M3& aLin, const M3& aAng, const M3& aCross,
                                         float3 bLin, float3 bAng, float3& xLin, float3& xAng) {
    float s1 = rsq(mx(aLin.r0.x, 1e-30f));
    float s2 = rsq(mx(aLin.r1.y, 1e-30f));
    float s3_ = rsq(mx(aLin.r2.z, 1e-30f));
    float s4 = rsq(mx(aAng.r0.x, 1e-30f));
    float s5 = rsq(mx(aAng.r1.y, 1e-30f));
    float s6 = rsq(mx(aAng.r2.z, 1e-30f));
    const float A11 = 1.0f, A22 = 1.0f, A33 = 1.0f, A44 = 1.0f, A55 = 1.0f, A66 = 1.0f;
    float A21 = aLin.r1.x * s2 * s1;
    float A31 = aLin.r2.x * s3_ * s1, A32 = aLin.r2.y * s3_ * s2;
    float A41 = aCross.r0.x * s4 * s1, A42 = aCross.r0.y * s4 * s2, A43 = aCross.r0.z * s4 * s3_;
    float A51 = aCross.r1.x * s5 * s1, A52 = aCross.r1.y * s5 * s2, A53 = aCross.r1.z * s5 * s3_,
          A54 = aAng.r1.x * s5 * s4;
    float A61 = aCross.r2.x * s6 * s1, A62 = aCross.r2.y * s6 * s2, A63 = aCross.r2.z * s6 * s3_,
          A64 = aAng.r2.x * s6 * s4, A65 = aAng.r2.y * s6 * s5;
    bLin = mk3(bLin.x * s1, bLin.y * s2, bLin.z * s3_);
    bAng = mk3(bAng.x * s4, bAng.y * s5, bAng.z * s6);
    float L21 = A21 / A11, L31 = A31 / A11, L41 = A41 / A11, L51 = A51 / A11, L61 = A61 / A11;
    const float eps = 1e-6f;
    float D1 = mx(A11, eps);
    float D2 = mx(A22 - L21 * L21 * D1, eps);
    float L32 = (A32 - L21 * L31 * D1) / D2;
    float L42 = (A42 - L21 * L41 * D1) / D2;
    float L52 = (A52 - L21 * L51 * D1) / D2;
    float L62 = (A62 - L21 * L61 * D1) / D2;
    float D3 = mx(A33 - (L31 * L31 * D1 + L32 * L32 * D2), eps);
    float L43 = (A43 - L31 * L41 * D1 - L32 * L42 * D2) / D3;
    float L53 = (A53 - L31 * L51 * D1 - L32 * L52 * D2) / D3;
    float L63 = (A63 - L31 * L61 * D1 - L32 * L62 * D2) / D3;
    float D4 = mx(A44 - (L41 * L41 * D1 + L42 * L42 * D2 + L43 * L43 * D3), eps);
    float L54 = (A54 - L41 * L51 * D1 - L42 * L52 * D2 - L43 * L53 * D3) / D4;
    float L64 = (A64 - L41 * L61 * D1 - L42 * L62 * D2 - L43 * L63 * D3) / D4;
    float D5 = mx(A55 - (L51 * L51 * D1 + L52 * L52 * D2 + L53 * L53 * D3 + L54 * L54 * D4), eps);
    float L65 = (A65 - L51 * L61 * D1 - L52 * L62 * D2 - L53 * L63 * D3 - L54 * L64 * D4) / D5;
    float D6 = mx(A66 - (L61 * L61 * D1 + L62 * L62 * D2 + L63 * L63 * D3 + L64 * L64 * D4
                         + L65 * L65 * D5), eps);
    float y1 = bLin.x;
    float y2 = bLin.y - L21 * y1;
    float y3 = bLin.z - L31 * y1 - L32 * y2;
    float y4 = bAng.x - L41 * y1 - L42 * y2 - L43 * y3;
    float y5 = bAng.y - L51 * y1 - L52 * y2 - L53 * y3 - L54 * y4;
    float y6 = bAng.z - L61 * y1 - L62 * y2 - L63 * y3 - L64 * y4 - L65 * y5;
    float z1 = y1 / D1, z2 = y2 / D2, z3 = y3 / D3, z4 = y4 / D4, z5 = y5 / D5, z6 = y6 / D6;
    xAng.z = z6;
    xAng.y = z5 - L65 * xAng.z;
    xAng.x = z4 - L54 * xAng.y - L64 * xAng.z;
    xLin.z = z3 - L43 * xAng.x - L53 * xAng.y - L63 * xAng.z;
    xLin.y = z2 - L32 * xLin.z - L42 * xAng.x - L52 * xAng.y - L62 * xAng.z;
    xLin.x = z1 - L21 * xLin.y - L31 * xLin.z - L41 * xAng.x - L51 * xAng.y - L61 * xAng.z;
    xLin = mk3(xLin.x * s1, xLin.y * s2, xLin.z * s3_);
    xAng = mk3(xAng.x * s4, xAng.y * s5, xAng.z * s6);
}

__device__ __forceinline__ void orthonormal(float3 n, float3& t1, float3& t2) {
    t1 = fabsf(n.x) > fabsf(n.z) ? mk3(-n.y, n.x, 0) : mk3(0, -n.z, n.y);
    t1 = nrm3(t1);
    t2 = cross(n, t1);
}

// atan2 evaluated with a fixed float32 operation sequence, so host and device
// agree bit for bit (the libm and CUDA atan2f may differ in the last ulp).
// Method: reduce to a = min/max in [0, 1]; for a > tan(pi/12) use
// atan(a) = pi/6 + atan((sqrt(3) a - 1) / (sqrt(3) + a)) (Cody & Waite's
// argument reduction), leaving |z| <= tan(pi/12) where the Maclaurin series
// z - z^3/3 + ... + z^13/13 is exact to float32; then undo the octant and
// quadrant symmetries.  Accuracy: a few ulp.
__device__ __forceinline__ float atan2_series(float y, float x) {
    if (y != y || x != x) return x + y;
    const float ax = fabsf(x), ay = fabsf(y);
    const float hi = ax > ay ? ax : ay, lo = ax > ay ? ay : ax;
    float r;
    if (hi == 0.0f) {
        r = 0.0f;
    } else {
        const float a = lo / hi;
        const bool big = a > 0.267949192431122706f;                  // tan(pi/12)
        const float z = big ? (1.73205080756887729f * a - 1.0f) / (1.73205080756887729f + a) : a;
        const float z2 = z * z;
        float p = 1.0f / 13.0f;
        p = p * z2 - 1.0f / 11.0f;
        p = p * z2 + 1.0f / 9.0f;
        p = p * z2 - 1.0f / 7.0f;
        p = p * z2 + 1.0f / 5.0f;
        p = p * z2 - 1.0f / 3.0f;
        p = p * z2 + 1.0f;
        r = z * p;
        if (big) r = 0.523598775598298873f + r;                      // pi/6
        if (ay > ax) r = 1.57079632679489662f - r;                   // pi/2
    }
    if (signbit(x)) r = 3.14159265358979324f - r;                    // pi
    return signbit(y) ? -r : r;
}

__device__ __forceinline__ float combine_friction(float a, float b, uint32_t mode) {
    if (mode == 1u) return a * b;
    if (mode == 2u) return mn(a, b);
    if (mode == 3u) return mx(a, b);
    if (mode == 4u) return 0.5f * (a + b);
    return sqrtf(mx(a * b, 0.0f));
}

// Spatial hash of an integer cell, salted by collision group.
__device__ __forceinline__ uint32_t cell_hash(int cx, int cy, int cz, uint32_t group, uint32_t size) {
    uint32_t h = ((uint32_t)cx * 92837111u) ^ ((uint32_t)cy * 689287499u) ^ ((uint32_t)cz * 283923481u);
    h ^= group * 0x9e3779b9u;
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    return h & (size - 1u);
}
__device__ __forceinline__ void cell_coord(float3 p, float cs, int& x, int& y, int& z) {
    x = (int)floorf(p.x / cs);
    y = (int)floorf(p.y / cs);
    z = (int)floorf(p.z / cs);
}
__device__ __forceinline__ uint32_t pair_map_hash(uint32_t a, uint32_t b, uint32_t cap) {
    uint32_t h = (a * 73856093u) ^ (b * 19349663u);
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    return h & (cap - 1u);
}

// Conservative test that a ball (p, reach) misses the box [lo, hi]: true
// only when it lies farther than reach plus a rounding allowance.
__device__ __forceinline__ bool ball_misses_box(float3 p, float reach, float4 lo, float4 hi) {
    const float dx = fmaxf(fmaxf(lo.x - p.x, p.x - hi.x), 0.0f);
    const float dy = fmaxf(fmaxf(lo.y - p.y, p.y - hi.y), 0.0f);
    const float dz = fmaxf(fmaxf(lo.z - p.z, p.z - hi.z), 0.0f);
    const float scale = fmaxf(fmaxf(fabsf(p.x), fabsf(p.y)), fmaxf(fabsf(p.z), reach));
    const float r = reach * 1.0001f + scale * 1.0e-5f + 1.0e-6f;
    return dx * dx + dy * dy + dz * dz > r * r;
}

// Hinge twist of qB relative to qAr about `axis` (B local), in (-pi, pi].
__device__ __forceinline__ float twist_angle(float4 qAr, float4 qB, float3 axis) {
    float4 r = q_mul(q_inv(qAr), qB);
    if (r.w < 0.0f) r = neg4(r);
    return 2.0f * atan2_series(dot(xyz(r), axis), r.w);
}
__device__ __forceinline__ float wrap_pi(float x) {
    return x - 6.2831853f * floorf((x + 3.14159265f) / 6.2831853f);
}

}  // namespace avbd
