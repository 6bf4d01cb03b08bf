// oracle_math.h — float32 vector/quaternion/3x3 helpers of the CPU oracle.
//
// TEST INFRASTRUCTURE.  The oracle is a serial CPU restatement of the
// reference solver; only tests/, __graft_entry__.smoke() and the
// cpu_baseline leg of bench.py may load it.  Nothing in the product links it.
//
// Every operation is written out in a fixed evaluation order with IEEE
// float32 rounding (compile with -ffp-contract=off, no -ffast-math) so the
// oracle is a bit-level reference for the CUDA kernels, which are compiled
// with -fmad=false and follow the same order.
//
// Follows Sources/PhysicsAVBD/Shaders/00_common.metal:50-228.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

namespace oracle {

struct F3 { float x, y, z; };
struct F4 { float x, y, z, w; };
struct U4 { uint32_t x, y, z, w; };

static inline F3 f3(float x, float y, float z) { return F3{x, y, z}; }
static inline F3 f3s(float s) { return F3{s, s, s}; }
static inline F4 f4(float x, float y, float z, float w) { return F4{x, y, z, w}; }
static inline F4 f4(F3 v, float w) { return F4{v.x, v.y, v.z, w}; }
static inline F3 xyz(F4 v) { return F3{v.x, v.y, v.z}; }

static inline F3 operator+(F3 a, F3 b) { return F3{a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline F3 operator-(F3 a, F3 b) { return F3{a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline F3 operator-(F3 a) { return F3{-a.x, -a.y, -a.z}; }
static inline F3 operator*(F3 a, float s) { return F3{a.x * s, a.y * s, a.z * s}; }
static inline F3 operator*(float s, F3 a) { return F3{s * a.x, s * a.y, s * a.z}; }
static inline F3 operator*(F3 a, F3 b) { return F3{a.x * b.x, a.y * b.y, a.z * b.z}; }
static inline F3 operator/(F3 a, float s) { return F3{a.x / s, a.y / s, a.z / s}; }
static inline F3& operator+=(F3& a, F3 b) { a = a + b; return a; }
static inline F3& operator-=(F3& a, F3 b) { a = a - b; return a; }
static inline F3& operator*=(F3& a, float s) { a = a * s; return a; }

static inline F4 operator+(F4 a, F4 b) { return F4{a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
static inline F4 operator-(F4 a) { return F4{-a.x, -a.y, -a.z, -a.w}; }
static inline F4 operator*(F4 a, float s) { return F4{a.x * s, a.y * s, a.z * s, a.w * s}; }
static inline F4 operator/(F4 a, float s) { return F4{a.x / s, a.y / s, a.z / s, a.w / s}; }

static inline float fmin_(float a, float b) { return a < b ? a : b; }
static inline float fmax_(float a, float b) { return a > b ? a : b; }
static inline float clampf_(float x, float lo, float hi) { return fmin_(fmax_(x, lo), hi); }
static inline F3 fmin3(F3 a, F3 b) { return F3{fmin_(a.x, b.x), fmin_(a.y, b.y), fmin_(a.z, b.z)}; }
static inline F3 fmax3(F3 a, F3 b) { return F3{fmax_(a.x, b.x), fmax_(a.y, b.y), fmax_(a.z, b.z)}; }
static inline F3 clamp3(F3 v, F3 lo, F3 hi) { return fmin3(fmax3(v, lo), hi); }
static inline F3 abs3(F3 v) { return F3{std::fabs(v.x), std::fabs(v.y), std::fabs(v.z)}; }
static inline float comp(F3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
static inline void setcomp(F3& v, int i, float s) { if (i == 0) v.x = s; else if (i == 1) v.y = s; else v.z = s; }

static inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float dot4(F4 a, F4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
static inline F3 cross(F3 a, F3 b) {
    return F3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
static inline float rsqrt_(float x) { return 1.0f / std::sqrt(x); }
static inline float length(F3 a) { return std::sqrt(dot(a, a)); }
static inline float distance(F3 a, F3 b) { return length(a - b); }
static inline float distance2(F3 a, F3 b) { F3 d = a - b; return dot(d, d); }
static inline F3 normalize(F3 a) { return a * rsqrt_(dot(a, a)); }
static inline F4 normalize4(F4 a) { return a * rsqrt_(dot4(a, a)); }

static inline uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
static inline float bitsf(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
// Fast-math-safe finiteness test on the exponent bits (00_common.metal:130).
static inline bool finite_bits(float x) { return (fbits(x) & 0x7F800000u) != 0x7F800000u; }
static inline bool finite3(F3 v) { return finite_bits(v.x) && finite_bits(v.y) && finite_bits(v.z); }

// Row-major 3x3: mul(v) = (r0.v, r1.v, r2.v).
struct M3 { F3 r0, r1, r2; };
static inline M3 m3_zero() { return M3{f3s(0), f3s(0), f3s(0)}; }
static inline M3 m3_diag(F3 d) { return M3{f3(d.x, 0, 0), f3(0, d.y, 0), f3(0, 0, d.z)}; }
static inline M3 m3_identity() { return m3_diag(f3s(1)); }
static inline F3 m3_mul(const M3& m, F3 v) { return F3{dot(m.r0, v), dot(m.r1, v), dot(m.r2, v)}; }
static inline F3 m3_col(const M3& m, int i) {
    return F3{comp(m.r0, i), comp(m.r1, i), comp(m.r2, i)};
}
static inline M3 m3_transpose(const M3& m) { return M3{m3_col(m, 0), m3_col(m, 1), m3_col(m, 2)}; }
static inline M3 m3_mulm(const M3& a, const M3& b) {
    M3 bt = m3_transpose(b);
    return M3{F3{dot(a.r0, bt.r0), dot(a.r0, bt.r1), dot(a.r0, bt.r2)},
              F3{dot(a.r1, bt.r0), dot(a.r1, bt.r1), dot(a.r1, bt.r2)},
              F3{dot(a.r2, bt.r0), dot(a.r2, bt.r1), dot(a.r2, bt.r2)}};
}
static inline M3 m3_add(const M3& a, const M3& b) { return M3{a.r0 + b.r0, a.r1 + b.r1, a.r2 + b.r2}; }
static inline M3 m3_scale(const M3& a, float s) { return M3{a.r0 * s, a.r1 * s, a.r2 * s}; }
static inline M3 m3_outer(F3 a, F3 b) { return M3{b * a.x, b * a.y, b * a.z}; }
static inline M3 m3_skew(F3 r) { return M3{f3(0, -r.z, r.y), f3(r.z, 0, -r.x), f3(-r.y, r.x, 0)}; }
static inline M3 m3_diagonalize(const M3& m) {
    return m3_diag(F3{length(m3_col(m, 0)), length(m3_col(m, 1)), length(m3_col(m, 2))});
}

// Quaternions (x, y, z imaginary; w real).
static inline F4 q_mul(F4 a, F4 b) {
    return F4{a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
              a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
              a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w,
              a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
static inline F4 q_conj(F4 q) { return F4{-q.x, -q.y, -q.z, q.w}; }
static inline F4 q_inv(F4 q) { return q_conj(q) / dot4(q, q); }
static inline F3 q_rotate(F4 q, F3 v) {
    F3 u = xyz(q);
    F3 t = 2.0f * cross(u, v);
    return v + q.w * t + cross(u, t);
}
static inline M3 world_inertia(F4 q, F3 p) {
    F3 c0 = q_rotate(q, f3(1, 0, 0));
    F3 c1 = q_rotate(q, f3(0, 1, 0));
    F3 c2 = q_rotate(q, f3(0, 0, 1));
    return m3_add(m3_add(m3_scale(m3_outer(c0, c0), p.x), m3_scale(m3_outer(c1, c1), p.y)),
                  m3_scale(m3_outer(c2, c2), p.z));
}
// Tangent-space difference with w >= 0 canonicalisation (00_common.metal:113-117).
static inline F3 q_sub(F4 a, F4 b) {
    F4 r = q_mul(a, q_inv(b));
    if (r.w < 0.0f) r = -r;
    return xyz(r) * 2.0f;
}
static inline F4 q_addw(F4 q, F3 w) {
    F4 dq = q_mul(f4(w, 0.0f), q);
    return normalize4(q + dq * 0.5f);
}
static inline F3 xform(F3 p, F4 q, F3 v) { return q_rotate(q, v) + p; }

// Jacobi-preconditioned, pivot-clamped 6x6 LDL^T (00_common.metal:137-221).
static inline void solve6x6(const M3& aLin, const M3& aAng, const M3& aCross,
                            F3 bLin, F3 bAng, F3& xLin, F3& xAng) {
    float s1 = rsqrt_(fmax_(aLin.r0.x, 1e-30f));
    float s2 = rsqrt_(fmax_(aLin.r1.y, 1e-30f));
    float s3 = rsqrt_(fmax_(aLin.r2.z, 1e-30f));
    float s4 = rsqrt_(fmax_(aAng.r0.x, 1e-30f));
    float s5 = rsqrt_(fmax_(aAng.r1.y, 1e-30f));
    float s6 = rsqrt_(fmax_(aAng.r2.z, 1e-30f));
    const float A11 = 1.0f, A22 = 1.0f, A33 = 1.0f, A44 = 1.0f, A55 = 1.0f, A66 = 1.0f;
    float A21 = aLin.r1.x * s2 * s1;
    float A31 = aLin.r2.x * s3 * s1, A32 = aLin.r2.y * s3 * s2;
    float A41 = aCross.r0.x * s4 * s1, A42 = aCross.r0.y * s4 * s2, A43 = aCross.r0.z * s4 * s3;
    float A51 = aCross.r1.x * s5 * s1, A52 = aCross.r1.y * s5 * s2, A53 = aCross.r1.z * s5 * s3,
          A54 = aAng.r1.x * s5 * s4;
    float A61 = aCross.r2.x * s6 * s1, A62 = aCross.r2.y * s6 * s2, A63 = aCross.r2.z * s6 * s3,
          A64 = aAng.r2.x * s6 * s4, A65 = aAng.r2.y * s6 * s5;
    bLin = F3{bLin.x * s1, bLin.y * s2, bLin.z * s3};
    bAng = F3{bAng.x * s4, bAng.y * s5, bAng.z * s6};
    float L21 = A21 / A11, L31 = A31 / A11, L41 = A41 / A11, L51 = A51 / A11, L61 = A61 / A11;
    const float eps = 1e-6f;
    float D1 = fmax_(A11, eps);
    float D2 = fmax_(A22 - L21 * L21 * D1, eps);
    float L32 = (A32 - L21 * L31 * D1) / D2;
    float L42 = (A42 - L21 * L41 * D1) / D2;
    float L52 = (A52 - L21 * L51 * D1) / D2;
    float L62 = (A62 - L21 * L61 * D1) / D2;
    float D3 = fmax_(A33 - (L31 * L31 * D1 + L32 * L32 * D2), eps);
    float L43 = (A43 - L31 * L41 * D1 - L32 * L42 * D2) / D3;
    float L53 = (A53 - L31 * L51 * D1 - L32 * L52 * D2) / D3;
    float L63 = (A63 - L31 * L61 * D1 - L32 * L62 * D2) / D3;
    float D4 = fmax_(A44 - (L41 * L41 * D1 + L42 * L42 * D2 + L43 * L43 * D3), eps);
    float L54 = (A54 - L41 * L51 * D1 - L42 * L52 * D2 - L43 * L53 * D3) / D4;
    float L64 = (A64 - L41 * L61 * D1 - L42 * L62 * D2 - L43 * L63 * D3) / D4;
    float D5 = fmax_(A55 - (L51 * L51 * D1 + L52 * L52 * D2 + L53 * L53 * D3 + L54 * L54 * D4), eps);
    float L65 = (A65 - L51 * L61 * D1 - L52 * L62 * D2 - L53 * L63 * D3 - L54 * L64 * D4) / D5;
    float D6 = fmax_(A66 - (L61 * L61 * D1 + L62 * L62 * D2 + L63 * L63 * D3 + L64 * L64 * D4
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
    xLin = F3{xLin.x * s1, xLin.y * s2, xLin.z * s3};
    xAng = F3{xAng.x * s4, xAng.y * s5, xAng.z * s6};
}

static inline void orthonormal(F3 n, F3& t1, F3& t2) {
    t1 = std::fabs(n.x) > std::fabs(n.z) ? f3(-n.y, n.x, 0) : f3(0, -n.z, n.y);
    t1 = normalize(t1);
    t2 = cross(n, t1);
}

// atan2 evaluated with a fixed float32 operation sequence, so host and device
// agree bit for bit (the libm and CUDA atan2f may differ in the last ulp).
// Method: reduce to a = min/max in [0, 1]; for a > tan(pi/12) use
// atan(a) = pi/6 + atan((sqrt(3) a - 1) / (sqrt(3) + a)) (Cody & Waite's
// argument reduction), leaving |z| <= tan(pi/12) where the Maclaurin series
// z - z^3/3 + ... + z^13/13 is exact to float32; then undo the octant and
// quadrant symmetries.  Accuracy: a few ulp.
static inline float atan2_series(float y, float x) {
    if (y != y || x != x) return x + y;
    const float ax = std::fabs(x), ay = std::fabs(y);
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
    if (std::signbit(x)) r = 3.14159265358979324f - r;                    // pi
    return std::signbit(y) ? -r : r;
}

static inline float combine_friction(float a, float b, uint32_t mode) {
    if (mode == 1u) return a * b;
    if (mode == 2u) return fmin_(a, b);
    if (mode == 3u) return fmax_(a, b);
    if (mode == 4u) return 0.5f * (a + b);
    return std::sqrt(fmax_(a * b, 0.0f));
}

}  // namespace oracle
