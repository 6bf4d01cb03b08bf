// cpu_solver.cpp — "Oracle B": the reference's CPU solver restated in C++.
//
// TEST INFRASTRUCTURE AND CPU BASELINE, NOT PRODUCT CODE.  Only tests/ and
// bench.py's CPU legs load it (oracle/cpu_solver.py).
//
// The reference ships a rigid-only CPU implementation of AVBD that it calls
// the ground truth of its Metal solver (Sources/PhysicsAVBD/CPU/CPUSolver.swift:4-7).
// It differs from the GPU path by design — an O(n^2) sphere broadphase,
// Gauss-Seidel over bodies in index order instead of colors, the
// unpreconditioned 6x6 LDL^T (SimCore/Math/Math.swift:163-226), no
// speculative contact margin, no trust region — so it is not the parity
// oracle of the CUDA path; it is the reference's own CPU algorithm, timed
// single-threaded as the reference runs it, and a sanity check.
//
// Followed:
//   CPUSolver.step             CPU/CPUSolver.swift:211-315
//   CPUManifold                CPU/CPUManifold.swift:36-210 (initialize, forceAndC,
//                              updatePrimal, updateDual)
//   CPUJoint, CPUSpring        CPU/CPUForces.swift:14-248
//   collideBoxBox + helpers    CPU/CPUCollide.swift:1-468
//   collideSphereSphere/Box    CPU/CPUCollide.swift:270-418
//   quatSub/quatAdd, Mat3Rows,
//   worldInertiaRows, solve6x6 SimCore/Math/Math.swift:58-226
// Shapes: boxes and spheres (the tori and capsules of CPUCollide.swift:470-848
// are not restated; a scene with them is refused at creation).
// Quaternion rotation is q v q^-1 in the form v + w t + u x t, t = 2 u x v.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <vector>

#include "../include/avbd.h"

namespace cpuref {

struct V3 { float x, y, z; };
static inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
static inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
static inline V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
static inline V3 mulv(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline V3& operator+=(V3& a, V3 b) { a = a + b; return a; }
static inline V3& operator-=(V3& a, V3 b) { a = a - b; return a; }
static inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline float len2(V3 a) { return dot(a, a); }
static inline float length(V3 a) { return std::sqrt(dot(a, a)); }
static inline V3 normalize(V3 a) { return a / length(a); }
static inline float comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
static inline float& compr(V3& a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
static inline V3 absv(V3 a) { return v3(std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)); }
static inline float clampf(float x, float lo, float hi) { return std::min(std::max(x, lo), hi); }
static inline V3 clamp3(V3 x, V3 lo, V3 hi) {
    return v3(clampf(x.x, lo.x, hi.x), clampf(x.y, lo.y, hi.y), clampf(x.z, lo.z, hi.z));
}
static inline V3 min3(V3 a, V3 b) { return v3(std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)); }

struct Q { V3 v; float w; };   // (imag, real)
static inline Q qmul(Q a, Q b) {
    return Q{a.v * b.w + b.v * a.w + cross(a.v, b.v), a.w * b.w - dot(a.v, b.v)};
}
static inline Q qconj(Q q) { return Q{-q.v, q.w}; }
static inline Q qinv(Q q) { float n = q.w * q.w + dot(q.v, q.v); return Q{(-q.v) / n, q.w / n}; }
static inline Q qnorm(Q q) { float n = std::sqrt(q.w * q.w + dot(q.v, q.v)); return Q{q.v / n, q.w / n}; }
static inline V3 qrot(Q q, V3 v) { V3 t = cross(q.v, v) * 2.0f; return v + t * q.w + cross(q.v, t); }
// Math.swift:68-79
static inline V3 quat_sub(Q a, Q b) { Q d = qmul(a, qinv(b)); return (d.w < 0.0f ? -d.v : d.v) * 2.0f; }
static inline Q quat_add(Q q, V3 w) {
    Q dq = qmul(Q{w, 0.0f}, q);
    return qnorm(Q{q.v + dq.v * 0.5f, q.w + 0.5f * dq.w});
}
static inline V3 xform(V3 p, Q q, V3 v) { return qrot(q, v) + p; }

struct M3 { V3 r0, r1, r2; };
static inline M3 mzero() { return M3{v3(0, 0, 0), v3(0, 0, 0), v3(0, 0, 0)}; }
static inline M3 mdiag(V3 d) { return M3{v3(d.x, 0, 0), v3(0, d.y, 0), v3(0, 0, d.z)}; }
static inline M3 mident() { return mdiag(v3(1, 1, 1)); }
static inline V3 row(const M3& m, int i) { return i == 0 ? m.r0 : (i == 1 ? m.r1 : m.r2); }
static inline V3 col(const M3& m, int i) { return v3(comp(m.r0, i), comp(m.r1, i), comp(m.r2, i)); }
static inline M3 mT(const M3& m) { return M3{col(m, 0), col(m, 1), col(m, 2)}; }
static inline V3 mmulv(const M3& m, V3 v) { return v3(dot(m.r0, v), dot(m.r1, v), dot(m.r2, v)); }
static inline M3 mmul(const M3& a, const M3& b) {
    V3 c0 = col(b, 0), c1 = col(b, 1), c2 = col(b, 2);
    return M3{v3(dot(a.r0, c0), dot(a.r0, c1), dot(a.r0, c2)), v3(dot(a.r1, c0), dot(a.r1, c1), dot(a.r1, c2)),
              v3(dot(a.r2, c0), dot(a.r2, c1), dot(a.r2, c2))};
}
static inline M3 madd(const M3& a, const M3& b) { return M3{a.r0 + b.r0, a.r1 + b.r1, a.r2 + b.r2}; }
static inline M3 mscale(const M3& a, float s) { return M3{a.r0 * s, a.r1 * s, a.r2 * s}; }
static inline M3 mneg(const M3& a) { return M3{-a.r0, -a.r1, -a.r2}; }
static inline M3 mskew(V3 r) { return M3{v3(0, -r.z, r.y), v3(r.z, 0, -r.x), v3(-r.y, r.x, 0)}; }
static inline M3 mdiagonalized(const M3& m) { return mdiag(v3(length(col(m, 0)), length(col(m, 1)), length(col(m, 2)))); }
static inline M3 outer_rows(V3 a, V3 b) { return M3{b * a.x, b * a.y, b * a.z}; }
// worldInertiaRows (Math.swift:86-95): sum_i I_i c_i c_i^T
static inline M3 world_inertia(Q q, V3 I) {
    V3 c0 = qrot(q, v3(1, 0, 0)), c1 = qrot(q, v3(0, 1, 0)), c2 = qrot(q, v3(0, 0, 1));
    return madd(madd(mscale(outer_rows(c0, c0), I.x), mscale(outer_rows(c1, c1), I.y)), mscale(outer_rows(c2, c2), I.z));
}
// orthonormalBasis (Math.swift:58-63)
static inline void ortho_basis(V3 n, V3& t1, V3& t2) {
    t1 = std::fabs(n.x) > std::fabs(n.z) ? v3(-n.y, n.x, 0) : v3(0, -n.z, n.y);
    t1 = normalize(t1);
    t2 = cross(n, t1);
}

// Unpreconditioned 6x6 LDL^T (Math.swift:163-226).
static void solve6x6(const M3& aLin, const M3& aAng, const M3& aCross, V3 bLin, V3 bAng, V3& xLin, V3& xAng) {
    const float A11 = aLin.r0.x;
    const float A21 = aLin.r1.x, A22 = aLin.r1.y;
    const float A31 = aLin.r2.x, A32 = aLin.r2.y, A33 = aLin.r2.z;
    const float A41 = aCross.r0.x, A42 = aCross.r0.y, A43 = aCross.r0.z, A44 = aAng.r0.x;
    const float A51 = aCross.r1.x, A52 = aCross.r1.y, A53 = aCross.r1.z, A54 = aAng.r1.x, A55 = aAng.r1.y;
    const float A61 = aCross.r2.x, A62 = aCross.r2.y, A63 = aCross.r2.z, A64 = aAng.r2.x, A65 = aAng.r2.y,
                A66 = aAng.r2.z;
    const float L21 = A21 / A11, L31 = A31 / A11, L41 = A41 / A11, L51 = A51 / A11, L61 = A61 / A11;
    const float D1 = A11;
    const float D2 = A22 - L21 * L21 * D1;
    const float L32 = (A32 - L21 * L31 * D1) / D2;
    const float L42 = (A42 - L21 * L41 * D1) / D2;
    const float L52 = (A52 - L21 * L51 * D1) / D2;
    const float L62 = (A62 - L21 * L61 * D1) / D2;
    const float D3 = A33 - (L31 * L31 * D1 + L32 * L32 * D2);
    const float L43 = (A43 - L31 * L41 * D1 - L32 * L42 * D2) / D3;
    const float L53 = (A53 - L31 * L51 * D1 - L32 * L52 * D2) / D3;
    const float L63 = (A63 - L31 * L61 * D1 - L32 * L62 * D2) / D3;
    const float D4 = A44 - (L41 * L41 * D1 + L42 * L42 * D2 + L43 * L43 * D3);
    const float L54 = (A54 - L41 * L51 * D1 - L42 * L52 * D2 - L43 * L53 * D3) / D4;
    const float L64 = (A64 - L41 * L61 * D1 - L42 * L62 * D2 - L43 * L63 * D3) / D4;
    const float D5 = A55 - (L51 * L51 * D1 + L52 * L52 * D2 + L53 * L53 * D3 + L54 * L54 * D4);
    const float L65 = (A65 - L51 * L61 * D1 - L52 * L62 * D2 - L53 * L63 * D3 - L54 * L64 * D4) / D5;
    const float D6 = A66 - (L61 * L61 * D1 + L62 * L62 * D2 + L63 * L63 * D3 + L64 * L64 * D4 + L65 * L65 * D5);
    const float y1 = bLin.x;
    const float y2 = bLin.y - L21 * y1;
    const float y3 = bLin.z - L31 * y1 - L32 * y2;
    const float y4 = bAng.x - L41 * y1 - L42 * y2 - L43 * y3;
    const float y5 = bAng.y - L51 * y1 - L52 * y2 - L53 * y3 - L54 * y4;
    const float y6 = bAng.z - L61 * y1 - L62 * y2 - L63 * y3 - L64 * y4 - L65 * y5;
    const float z1 = y1 / D1, z2 = y2 / D2, z3 = y3 / D3, z4 = y4 / D4, z5 = y5 / D5, z6 = y6 / D6;
    xAng.z = z6;
    xAng.y = z5 - L65 * xAng.z;
    xAng.x = z4 - L54 * xAng.y - L64 * xAng.z;
    xLin.z = z3 - L43 * xAng.x - L53 * xAng.y - L63 * xAng.z;
    xLin.y = z2 - L32 * xLin.z - L42 * xAng.x - L52 * xAng.y - L62 * xAng.z;
    xLin.x = z1 - L21 * xLin.y - L31 * xLin.z - L41 * xAng.x - L51 * xAng.y - L61 * xAng.z;
}

const float PENALTY_MIN = 1.0f, PENALTY_MAX = 1.0e10f, PENALTY_MAX_T = 1.0e6f, STICK_THRESH = 0.00001f;
const float FINF = std::numeric_limits<float>::infinity();

static float combine_friction(float a, float b, uint32_t mode) {
    if (mode == 1u) return a * b;
    if (mode == 2u) return std::min(a, b);
    if (mode == 3u) return std::max(a, b);
    if (mode == 4u) return 0.5f * (a + b);
    return std::sqrt(std::max(a * b, 0.0f));
}

struct Solver;
struct Force;

struct Rigid {
    V3 positionLin, initialLin, inertialLin, velocityLin, velocityAng, prevVelocityLin, size, moment;
    Q positionAng, initialAng, inertialAng;
    float mass, friction, dynamicFriction, gravityScale, radius;
    uint32_t shape;
    bool isParticle = false;
    std::vector<Force*> forces;
};

struct Force {
    Rigid* a = nullptr;   // null = world
    Rigid* b = nullptr;
    bool alive = true;
    virtual ~Force() {}
    virtual bool initialize(Solver&) { return true; }
    virtual void update_primal(Solver&, Rigid*, M3&, M3&, M3&, V3&, V3&) {}
    virtual void update_dual(Solver&) {}
};

struct Contact {
    int32_t featureKey = 0;
    V3 rA{0, 0, 0}, rB{0, 0, 0}, C0{0, 0, 0}, penalty{0, 0, 0}, lambda{0, 0, 0};
    bool stick = false;
};

struct Solver {
    float dt = 1.0f / 60.0f, gravity = -10.0f, collisionMargin = 0.01f, alpha = 0.99f, betaLin = 5000.0f,
          betaAng = 100.0f, gamma = 0.999f, lambdaMax = 1.0e6f;
    int iterations = 10;
    uint32_t frictionCombineMode = 0;
    float rigidLinearDamping = 0.0f, rigidAngularDamping = 0.0f;
    std::vector<std::unique_ptr<Rigid>> bodies;
    std::vector<Force*> forces;
    std::vector<std::unique_ptr<Force>> owned;
    std::vector<avbd_spinner_desc> spinners;

    void add_force(Force* f) {
        owned.emplace_back(f);
        forces.push_back(f);
        if (f->a) f->a->forces.push_back(f);
        if (f->b) f->b->forces.push_back(f);
    }
    void drop_from_bodies(Force* f) {
        for (Rigid* r : {f->a, f->b})
            if (r) r->forces.erase(std::remove(r->forces.begin(), r->forces.end(), f), r->forces.end());
    }
    bool constrained(Rigid* a, Rigid* b) const {
        for (Force* f : a->forces)
            if ((f->a == a && f->b == b) || (f->a == b && f->b == a)) return true;
        return false;
    }
    void step();
    float max_constraint_error() const;
};

// ---------------------------------------------------------------- joints
static M3 geom_stiff(int k, V3 v) {            // CPUForces.swift:6-12
    M3 m = mdiag(v3(-comp(v, k), -comp(v, k), -comp(v, k)));
    compr(m.r0, k) += v.x;
    compr(m.r1, k) += v.y;
    compr(m.r2, k) += v.z;
    return m;
}

struct Joint : Force {
    V3 rA, rB, C0Lin{0, 0, 0}, C0Ang{0, 0, 0}, penaltyLin{0, 0, 0}, penaltyAng{0, 0, 0}, lambdaLin{0, 0, 0},
        lambdaAng{0, 0, 0};
    float stiffnessLin, stiffnessAng, fracture, torqueArm;
    bool broken = false, fractureLinear = false, hasHinge = false;
    Q restRel;
    V3 hingeAxis{0, 0, 0};

    V3 currentCLin() const {
        V3 pA = a ? xform(a->positionLin, a->positionAng, rA) : rA;
        return pA - xform(b->positionLin, b->positionAng, rB);
    }
    V3 currentCAng() const {
        Q qA = a ? a->positionAng : Q{v3(0, 0, 0), 1.0f};
        if (hasHinge) {
            V3 aB = qrot(b->positionAng, hingeAxis);
            V3 aA = qrot(qnorm(qmul(qA, restRel)), hingeAxis);
            return cross(aA, aB) * torqueArm;
        }
        return quat_sub(qnorm(qmul(qA, restRel)), b->positionAng) * torqueArm;
    }
    bool initialize(Solver& S) override {
        C0Lin = currentCLin();
        C0Ang = currentCAng();
        lambdaLin = lambdaLin * (S.alpha * S.gamma);
        lambdaAng = lambdaAng * (S.alpha * S.gamma);
        penaltyLin = clamp3(penaltyLin * S.gamma, v3(PENALTY_MIN, PENALTY_MIN, PENALTY_MIN),
                            v3(PENALTY_MAX, PENALTY_MAX, PENALTY_MAX));
        penaltyAng = clamp3(penaltyAng * S.gamma, v3(PENALTY_MIN, PENALTY_MIN, PENALTY_MIN),
                            v3(PENALTY_MAX, PENALTY_MAX, PENALTY_MAX));
        penaltyLin = min3(penaltyLin, v3(stiffnessLin, stiffnessLin, stiffnessLin));
        penaltyAng = min3(penaltyAng, v3(stiffnessAng, stiffnessAng, stiffnessAng));
        return !broken;
    }
    void update_primal(Solver& S, Rigid* body, M3& lhsLin, M3& lhsAng, M3& lhsCross, V3& rhsLin,
                       V3& rhsAng) override {
        const bool isA = body == a;
        if (len2(penaltyLin) > 0.0f) {
            V3 C = currentCLin();
            if (std::isinf(stiffnessLin)) C -= C0Lin * S.alpha;
            V3 F = mulv(penaltyLin, C) + lambdaLin;
            M3 jLin = isA ? mident() : mneg(mident());
            M3 jAng = isA ? mskew(-qrot(a->positionAng, rA)) : mskew(qrot(b->positionAng, rB));
            M3 jLinT = mT(jLin), jAngT = mT(jAng);
            M3 K = mdiag(penaltyLin);
            M3 jAngTk = mmul(jAngT, K);
            lhsLin = madd(lhsLin, mmul(mmul(jLinT, K), jLin));
            lhsAng = madd(lhsAng, mmul(jAngTk, jAng));
            lhsCross = madd(lhsCross, mmul(jAngTk, jLin));
            V3 r = isA ? qrot(a->positionAng, rA) : -qrot(b->positionAng, rB);
            M3 H = mscale(geom_stiff(0, r), F.x);
            H = madd(H, mscale(geom_stiff(1, r), F.y));
            H = madd(H, mscale(geom_stiff(2, r), F.z));
            lhsAng = madd(lhsAng, mdiagonalized(H));
            rhsLin += mmulv(jLinT, F);
            rhsAng += mmulv(jAngT, F);
        }
        if (len2(penaltyAng) > 0.0f) {
            V3 C = currentCAng();
            if (std::isinf(stiffnessAng)) C -= C0Ang * S.alpha;
            V3 F = mulv(penaltyAng, C) + lambdaAng;
            float s = (isA ? 1.0f : -1.0f) * torqueArm;
            if (hasHinge) s = -s;
            lhsAng = madd(lhsAng, mdiag(penaltyAng * (s * s)));
            rhsAng += F * s;
        }
    }
    void update_dual(Solver& S) override {
        if (len2(penaltyLin) > 0.0f) {
            V3 C = currentCLin();
            if (std::isinf(stiffnessLin)) {
                C -= C0Lin * S.alpha;
                lambdaLin = mulv(penaltyLin, C) + lambdaLin;
            }
            float cap = std::min(stiffnessLin, PENALTY_MAX);
            penaltyLin = min3(penaltyLin + absv(C) * S.betaLin, v3(cap, cap, cap));
        }
        if (len2(penaltyAng) > 0.0f) {
            V3 C = currentCAng();
            if (std::isinf(stiffnessAng)) {
                C -= C0Ang * S.alpha;
                lambdaAng = mulv(penaltyAng, C) + lambdaAng;
            }
            float cap = std::min(stiffnessAng, PENALTY_MAX);
            penaltyAng = min3(penaltyAng + absv(C) * S.betaAng, v3(cap, cap, cap));
        }
        float lin2 = fractureLinear ? len2(lambdaLin) : 0.0f;
        if (len2(lambdaAng) + lin2 > fracture * fracture) {
            penaltyLin = penaltyAng = lambdaLin = lambdaAng = v3(0, 0, 0);
            broken = true;
        }
    }
};

struct Spring : Force {
    V3 rA, rB;
    float rest, stiffness, lambda = 0.0f, penalty = 0.0f, C0 = 0.0f;
    bool hard = false;
    bool initialize(Solver& S) override {
        if (!hard) return true;
        V3 pA = xform(a->positionLin, a->positionAng, rA), pB = xform(b->positionLin, b->positionAng, rB);
        C0 = length(pA - pB) - rest;
        lambda *= S.alpha * S.gamma;
        penalty = std::min(clampf(penalty * S.gamma, PENALTY_MIN, PENALTY_MAX), stiffness);
        return true;
    }
    void update_dual(Solver& S) override {
        if (!hard) return;
        V3 pA = xform(a->positionLin, a->positionAng, rA), pB = xform(b->positionLin, b->positionAng, rB);
        float C = length(pA - pB) - rest - C0 * S.alpha;
        lambda = clampf(penalty * C + lambda, -S.lambdaMax, S.lambdaMax);
        penalty = std::min(penalty + std::fabs(C) * S.betaLin, std::min(stiffness, PENALTY_MAX));
    }
    void update_primal(Solver& S, Rigid* body, M3& lhsLin, M3& lhsAng, M3& lhsCross, V3& rhsLin,
                       V3& rhsAng) override {
        V3 pA = xform(a->positionLin, a->positionAng, rA), pB = xform(b->positionLin, b->positionAng, rB);
        V3 d = pA - pB;
        float dLen = length(d);
        if (dLen <= 1e-6f) return;
        V3 n = d / dLen;
        float k = stiffness, f;
        if (hard) { k = penalty; f = penalty * (dLen - rest - C0 * S.alpha) + lambda; }
        else f = stiffness * (dLen - rest);
        const bool isA = body == a;
        V3 rWorld = isA ? qrot(a->positionAng, rA) : qrot(b->positionAng, rB);
        V3 jLin = isA ? n : -n;
        V3 jAng = isA ? cross(rWorld, n) : -cross(rWorld, n);
        lhsLin = madd(lhsLin, mscale(outer_rows(jLin, jLin), k));
        lhsAng = madd(lhsAng, mscale(outer_rows(jAng, jAng), k));
        lhsCross = madd(lhsCross, mscale(outer_rows(jAng, jLin), k));
        rhsLin += jLin * f;
        rhsAng += jAng * f;
    }
};

// ---------------------------------------------------------------- collision
const int MAX_CONTACTS = 8, MAX_POLY = 16;
const float SAT_EPS = 1.0e-6f, PLANE_EPS = 1.0e-5f, MERGE_SQ = 1.0e-6f;
enum { AX_FACE_A = 0, AX_FACE_B = 1, AX_EDGE = 2 };

struct OBB {
    V3 center, half, ax[3];
    explicit OBB(const Rigid& r) {
        center = r.positionLin;
        half = r.size * 0.5f;
        ax[0] = qrot(r.positionAng, v3(1, 0, 0));
        ax[1] = qrot(r.positionAng, v3(0, 1, 0));
        ax[2] = qrot(r.positionAng, v3(0, 0, 1));
    }
};
struct SatAxis { int type = AX_FACE_A, ia = -1, ib = -1; float sep = -std::numeric_limits<float>::max(); V3 n{0, 0, 0}; bool valid = false; };

static V3 support_point(const OBB& b, V3 dir) {
    float sx = dot(dir, b.ax[0]) >= 0.0f ? 1.0f : -1.0f;
    float sy = dot(dir, b.ax[1]) >= 0.0f ? 1.0f : -1.0f;
    float sz = dot(dir, b.ax[2]) >= 0.0f ? 1.0f : -1.0f;
    return b.center + b.ax[0] * (b.half.x * sx) + b.ax[1] * (b.half.y * sy) + b.ax[2] * (b.half.z * sz);
}
static void face_axes(const OBB& b, int i, V3& u, V3& v, float& eu, float& ev) {
    if (i == 0) { u = b.ax[1]; v = b.ax[2]; eu = b.half.y; ev = b.half.z; }
    else if (i == 1) { u = b.ax[0]; v = b.ax[2]; eu = b.half.x; ev = b.half.z; }
    else { u = b.ax[0]; v = b.ax[1]; eu = b.half.x; ev = b.half.y; }
}
static bool test_axis(const OBB& A, const OBB& B, V3 delta, V3 axis, int type, int ia, int ib, SatAxis& best) {
    float lsq = len2(axis);
    if (lsq < SAT_EPS) return true;
    V3 n = axis / std::sqrt(lsq);
    if (dot(n, delta) < 0.0f) n = -n;
    float dist = std::fabs(dot(delta, n));
    float rA = A.half.x * std::fabs(dot(n, A.ax[0])) + A.half.y * std::fabs(dot(n, A.ax[1])) +
               A.half.z * std::fabs(dot(n, A.ax[2]));
    float rB = B.half.x * std::fabs(dot(n, B.ax[0])) + B.half.y * std::fabs(dot(n, B.ax[1])) +
               B.half.z * std::fabs(dot(n, B.ax[2]));
    float sep = dist - (rA + rB);
    if (sep > 0.0f) return false;
    if (!best.valid || sep > best.sep) { best.valid = true; best.type = type; best.ia = ia; best.ib = ib; best.sep = sep; best.n = n; }
    return true;
}
static std::vector<V3> clip_poly(const std::vector<V3>& in, V3 pn, float off) {
    std::vector<V3> out;
    if (in.empty()) return out;
    V3 a = in.back();
    float da = dot(pn, a) - off;
    for (V3 b : in) {
        float db = dot(pn, b) - off;
        bool aIn = da <= PLANE_EPS, bIn = db <= PLANE_EPS;
        if (aIn != bIn) {
            float t = 0.0f, denom = da - db;
            if (std::fabs(denom) > SAT_EPS) t = clampf(da / denom, 0.0f, 1.0f);
            if ((int)out.size() < MAX_POLY) out.push_back(a + (b - a) * t);
        }
        if (bIn && (int)out.size() < MAX_POLY) out.push_back(b);
        a = b;
        da = db;
    }
    return out;
}
static void closest_seg(V3 p0, V3 p1, V3 q0, V3 q1, V3& c0, V3& c1) {
    V3 d1 = p1 - p0, d2 = q1 - q0, r = p0 - q0;
    float a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r), s = 0.0f, t = 0.0f;
    if (a <= SAT_EPS && e <= SAT_EPS) { c0 = p0; c1 = q0; return; }
    if (a <= SAT_EPS) {
        t = clampf(f / e, 0.0f, 1.0f);
    } else {
        float c = dot(d1, r);
        if (e <= SAT_EPS) {
            s = clampf(-c / a, 0.0f, 1.0f);
        } else {
            float b = dot(d1, d2), denom = a * e - b * b;
            if (std::fabs(denom) > SAT_EPS) s = clampf((b * f - c * e) / denom, 0.0f, 1.0f);
            t = (b * s + f) / e;
            if (t < 0.0f) { t = 0.0f; s = clampf(-c / a, 0.0f, 1.0f); }
            else if (t > 1.0f) { t = 1.0f; s = clampf((b - c) / a, 0.0f, 1.0f); }
        }
    }
    c0 = p0 + d1 * s;
    c1 = q0 + d2 * t;
}
static void support_edge(const OBB& b, int axis, V3 dir, V3& e0, V3& e1) {
    int a1 = (axis + 1) % 3, a2 = (axis + 2) % 3;
    float s1 = dot(dir, b.ax[a1]) >= 0.0f ? 1.0f : -1.0f;
    float s2 = dot(dir, b.ax[a2]) >= 0.0f ? 1.0f : -1.0f;
    V3 c = b.center + b.ax[a1] * (comp(b.half, a1) * s1) + b.ax[a2] * (comp(b.half, a2) * s2);
    e0 = c - b.ax[axis] * comp(b.half, axis);
    e1 = c + b.ax[axis] * comp(b.half, axis);
}
static void add_contact(const Rigid& A, const Rigid& B, std::vector<Contact>& cs, std::vector<V3>& mids, V3 xA, V3 xB,
                        int32_t key) {
    V3 mid = (xA + xB) * 0.5f;
    for (V3 m : mids)
        if (len2(mid - m) < MERGE_SQ) return;
    if ((int)cs.size() >= MAX_CONTACTS) return;
    Contact c;
    c.featureKey = key;
    c.rA = qrot(qconj(A.positionAng), xA - A.positionLin);
    c.rB = qrot(qconj(B.positionAng), xB - B.positionLin);
    cs.push_back(c);
    mids.push_back(mid);
}
static void face_manifold(const Rigid& bA, const Rigid& bB, const OBB& A, const OBB& B, bool refIsA, int refAxis,
                          V3 nAB, std::vector<Contact>& cs) {
    const OBB& R = refIsA ? A : B;
    const OBB& I = refIsA ? B : A;
    V3 refOut = refIsA ? nAB : -nAB;
    float sR = dot(refOut, R.ax[refAxis]) >= 0.0f ? 1.0f : -1.0f;
    V3 refN = R.ax[refAxis] * sR;
    V3 refC = R.center + refN * comp(R.half, refAxis);
    V3 rU, rV;
    float rEU, rEV;
    face_axes(R, refAxis, rU, rV, rEU, rEV);
    int incAxis = 0;
    float bestD = -std::numeric_limits<float>::max();
    for (int i = 0; i < 3; i++) {
        float d = std::fabs(dot(I.ax[i], refN));
        if (d > bestD) { bestD = d; incAxis = i; }
    }
    float sI = dot(I.ax[incAxis], refN) > 0.0f ? -1.0f : 1.0f;
    V3 incN = I.ax[incAxis] * sI;
    V3 incC = I.center + incN * comp(I.half, incAxis);
    V3 iU, iV;
    float iEU, iEV;
    face_axes(I, incAxis, iU, iV, iEU, iEV);
    std::vector<V3> poly = {incC + iU * iEU + iV * iEV, incC - iU * iEU + iV * iEV, incC - iU * iEU - iV * iEV,
                            incC + iU * iEU - iV * iEV};
    poly = clip_poly(poly, rU, dot(rU, refC) + rEU);
    if (poly.empty()) return;
    poly = clip_poly(poly, -rU, dot(-rU, refC) + rEU);
    if (poly.empty()) return;
    poly = clip_poly(poly, rV, dot(rV, refC) + rEV);
    if (poly.empty()) return;
    poly = clip_poly(poly, -rV, dot(-rV, refC) + rEV);
    if (poly.empty()) return;
    std::vector<V3> mids;
    int32_t prefix = (int32_t)((refIsA ? AX_FACE_A : AX_FACE_B) << 24);
    prefix |= (int32_t)((refAxis & 0xFF) << 16);
    prefix |= (int32_t)((incAxis & 0xFF) << 8);
    for (size_t i = 0; i < poly.size() && (int)cs.size() < MAX_CONTACTS; i++) {
        V3 p = poly[i];
        float distance = dot(p - refC, refN);
        if (distance > PLANE_EPS) continue;
        V3 pr = p - refN * distance;
        add_contact(bA, bB, cs, mids, refIsA ? pr : p, refIsA ? p : pr, prefix | (int32_t)(i & 0xFF));
    }
    if (cs.empty()) add_contact(bA, bB, cs, mids, support_point(A, nAB), support_point(B, -nAB), prefix);
}
static void edge_contact(const Rigid& bA, const Rigid& bB, const OBB& A, const OBB& B, int axA, int axB, V3 nAB,
                         std::vector<Contact>& cs) {
    V3 a0, a1, b0, b1, xA, xB;
    support_edge(A, axA, nAB, a0, a1);
    support_edge(B, axB, -nAB, b0, b1);
    closest_seg(a0, a1, b0, b1, xA, xB);
    std::vector<V3> mids;
    int32_t key = (int32_t)(AX_EDGE << 24) | (int32_t)((axA & 0xFF) << 8) | (int32_t)(axB & 0xFF);
    add_contact(bA, bB, cs, mids, xA, xB, key);
    if (cs.empty()) add_contact(bA, bB, cs, mids, support_point(A, nAB), support_point(B, -nAB), key);
}
static int collide_box_box(const Rigid& bA, const Rigid& bB, std::vector<Contact>& cs, V3 basis[3]) {
    OBB A(bA), B(bB);
    V3 delta = B.center - A.center;
    SatAxis bf, be;
    for (int i = 0; i < 3; i++) if (!test_axis(A, B, delta, A.ax[i], AX_FACE_A, i, -1, bf)) return 0;
    for (int i = 0; i < 3; i++) if (!test_axis(A, B, delta, B.ax[i], AX_FACE_B, -1, i, bf)) return 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            if (!test_axis(A, B, delta, cross(A.ax[i], B.ax[j]), AX_EDGE, i, j, be)) return 0;
    if (!bf.valid) return 0;
    SatAxis best = bf;
    if (be.valid && 0.95f * be.sep > bf.sep + 0.01f) best = be;
    basis[0] = -best.n;
    ortho_basis(basis[0], basis[1], basis[2]);
    cs.clear();
    if (best.type == AX_EDGE) edge_contact(bA, bB, A, B, best.ia, best.ib, best.n, cs);
    else if (best.type == AX_FACE_A) face_manifold(bA, bB, A, B, true, best.ia, best.n, cs);
    else face_manifold(bA, bB, A, B, false, best.ib, best.n, cs);
    return (int)cs.size();
}
static int collide_sphere_sphere(const Rigid& a, const Rigid& b, float margin, std::vector<Contact>& cs, V3 basis[3]) {
    cs.clear();
    float rA = a.size.x / 2.0f, rB = b.size.x / 2.0f;
    V3 d = a.positionLin - b.positionLin;
    float dist = length(d);
    if (dist > rA + rB + margin) return 0;
    V3 n = dist > 1e-9f ? d / dist : v3(0, 0, 1);
    basis[0] = n;
    ortho_basis(n, basis[1], basis[2]);
    Contact c;
    V3 xA = a.positionLin - n * rA, xB = b.positionLin + n * rB;
    c.rA = xA - a.positionLin;
    c.rB = xB - b.positionLin;
    cs.push_back(c);
    return 1;
}
static int collide_sphere_box(const Rigid& sphere, const Rigid& box, bool sphereIsA, float margin,
                              std::vector<Contact>& cs, V3 basis[3]) {
    cs.clear();
    float r = sphere.size.x / 2.0f;
    V3 half = box.size * 0.5f;
    V3 local = qrot(qconj(box.positionAng), sphere.positionLin - box.positionLin);
    V3 clamped = clamp3(local, -half, half);
    V3 nLocal, qLocal;
    if (clamped.x == local.x && clamped.y == local.y && clamped.z == local.z) {
        V3 pen = half - absv(local);
        int axis = 0;
        if (pen.y < comp(pen, axis)) axis = 1;
        if (pen.z < comp(pen, axis)) axis = 2;
        V3 n = v3(0, 0, 0);
        compr(n, axis) = comp(local, axis) >= 0.0f ? 1.0f : -1.0f;
        nLocal = n;
        qLocal = local;
        compr(qLocal, axis) = comp(n, axis) * comp(half, axis);
    } else {
        V3 d = local - clamped;
        float dist = length(d);
        if (dist > r + margin) return 0;
        nLocal = d / std::max(dist, 1e-9f);
        qLocal = clamped;
    }
    V3 nW = qrot(box.positionAng, nLocal);
    V3 qW = xform(box.positionLin, box.positionAng, qLocal);
    V3 xS = sphere.positionLin - nW * r;
    V3 n = sphereIsA ? nW : -nW;
    basis[0] = n;
    ortho_basis(n, basis[1], basis[2]);
    const Rigid& A = sphereIsA ? sphere : box;
    const Rigid& B = sphereIsA ? box : sphere;
    V3 xA = sphereIsA ? xS : qW, xB = sphereIsA ? qW : xS;
    Contact c;
    c.rA = A.shape == AVBD_SHAPE_SPHERE ? xA - A.positionLin : qrot(qconj(A.positionAng), xA - A.positionLin);
    c.rB = B.shape == AVBD_SHAPE_SPHERE ? xB - B.positionLin : qrot(qconj(B.positionAng), xB - B.positionLin);
    cs.push_back(c);
    return 1;
}

// ---------------------------------------------------------------- manifold
struct Manifold : Force {
    std::vector<Contact> contacts;
    V3 basis[3] = {v3(0, 0, 0), v3(0, 0, 0), v3(0, 0, 0)};
    float staticFriction = 0.0f, dynamicFriction = 0.0f;

    V3 anchor_world(const Rigid* r, V3 off) const {
        return r->shape != AVBD_SHAPE_BOX ? r->positionLin + off : xform(r->positionLin, r->positionAng, off);
    }
    V3 anchor_offset(const Rigid* r, V3 off) const { return r->shape != AVBD_SHAPE_BOX ? off : qrot(r->positionAng, off); }
    float penetration(const Solver& S, size_t i) const {
        return dot(basis[0], anchor_world(a, contacts[i].rA) - anchor_world(b, contacts[i].rB)) + S.collisionMargin;
    }
    bool initialize(Solver& S) override {
        staticFriction = combine_friction(a->friction, b->friction, S.frictionCombineMode);
        dynamicFriction = combine_friction(a->dynamicFriction, b->dynamicFriction, S.frictionCombineMode);
        std::vector<Contact> fresh;
        int count = 0;
        const uint32_t sa = a->shape, sb = b->shape;
        if (sa == AVBD_SHAPE_SPHERE && sb == AVBD_SHAPE_SPHERE) count = collide_sphere_sphere(*a, *b, S.collisionMargin, fresh, basis);
        else if (sa == AVBD_SHAPE_SPHERE && sb == AVBD_SHAPE_BOX) count = collide_sphere_box(*a, *b, true, S.collisionMargin, fresh, basis);
        else if (sa == AVBD_SHAPE_BOX && sb == AVBD_SHAPE_SPHERE) count = collide_sphere_box(*b, *a, false, S.collisionMargin, fresh, basis);
        else count = collide_box_box(*a, *b, fresh, basis);
        const bool anySphere = sa != AVBD_SHAPE_BOX || sb != AVBD_SHAPE_BOX;
        for (int i = 0; i < count; i++) {
            for (const Contact& old : contacts) {
                if (old.featureKey != fresh[i].featureKey) continue;
                V3 nA = fresh[i].rA, nB = fresh[i].rB;
                fresh[i] = old;
                if (!old.stick || anySphere) { fresh[i].rA = nA; fresh[i].rB = nB; }
                break;
            }
        }
        contacts = fresh;
        V3 wA = v3(0, 0, 0), wB = v3(0, 0, 0);
        for (const auto& sp : S.spinners) {
            if (S.bodies[sp.body].get() == a) wA = v3(sp.axis[0], sp.axis[1], sp.axis[2]) * sp.omega;
            if (S.bodies[sp.body].get() == b) wB = v3(sp.axis[0], sp.axis[1], sp.axis[2]) * sp.omega;
        }
        for (Contact& c : contacts) {
            V3 xA = anchor_world(a, c.rA), xB = anchor_world(b, c.rB), d = xA - xB;
            c.C0 = v3(dot(basis[0], d) + S.collisionMargin, dot(basis[1], d), dot(basis[2], d));
            V3 sA = cross(wA, xA - a->positionLin) * S.dt, sB = cross(wB, xB - b->positionLin) * S.dt;
            V3 rel = (sB - sA) / std::max(1.0f - S.alpha, 0.01f);
            c.C0.y -= dot(basis[1], rel);
            c.C0.z -= dot(basis[2], rel);
            c.lambda = c.lambda * (S.alpha * S.gamma);
            float minMass = std::numeric_limits<float>::infinity();
            if (a->mass > 0.0f) minMass = std::min(minMass, a->mass);
            if (b->mass > 0.0f) minMass = std::min(minMass, b->mass);
            if (std::isinf(minMass)) minMass = 0.0f;
            float kFloor = std::min(PENALTY_MAX, std::max(PENALTY_MIN, minMass / std::max(S.dt * S.dt, 1e-12f)));
            V3 pmin = v3(kFloor, std::min(kFloor, PENALTY_MAX_T), std::min(kFloor, PENALTY_MAX_T));
            c.penalty = clamp3(c.penalty * S.gamma, pmin, v3(PENALTY_MAX, PENALTY_MAX_T, PENALTY_MAX_T));
        }
        return !contacts.empty();
    }
    void force_c(const Solver& S, size_t i, float al, V3 dALin, V3 dAAng, V3 dBLin, V3 dBAng, V3 rAW, V3 rBW, V3& F,
                 V3& C, float& fscale, float& bounds) const {
        const Contact& c = contacts[i];
        V3 j0 = basis[0], j1 = basis[1], j2 = basis[2];
        C = c.C0 * (1.0f - al);
        C += v3(dot(j0, dALin), dot(j1, dALin), dot(j2, dALin));
        C -= v3(dot(j0, dBLin), dot(j1, dBLin), dot(j2, dBLin));
        C += v3(dot(cross(rAW, j0), dAAng), dot(cross(rAW, j1), dAAng), dot(cross(rAW, j2), dAAng));
        C += v3(dot(cross(rBW, -j0), dBAng), dot(cross(rBW, -j1), dBAng), dot(cross(rBW, -j2), dBAng));
        F = mulv(c.penalty, C) + c.lambda;
        F.x = std::min(F.x, 0.0f);
        float staticB = std::fabs(F.x) * staticFriction, dynB = std::fabs(F.x) * dynamicFriction;
        fscale = std::sqrt(F.y * F.y + F.z * F.z);
        if (fscale > staticB && fscale > 0.0f) {
            F.y *= dynB / fscale;
            F.z *= dynB / fscale;
        }
        bounds = staticB;
        (void)S;
    }
    void update_primal(Solver& S, Rigid* body, M3& lhsLin, M3& lhsAng, M3& lhsCross, V3& rhsLin,
                       V3& rhsAng) override {
        V3 dALin = a->positionLin - a->initialLin, dAAng = quat_sub(a->positionAng, a->initialAng);
        V3 dBLin = b->positionLin - b->initialLin, dBAng = quat_sub(b->positionAng, b->initialAng);
        const bool isA = body == a;
        for (size_t i = 0; i < contacts.size(); i++) {
            V3 rAW = anchor_offset(a, contacts[i].rA), rBW = anchor_offset(b, contacts[i].rB), F, C;
            float fs, bd;
            force_c(S, i, S.alpha, dALin, dAAng, dBLin, dBAng, rAW, rBW, F, C, fs, bd);
            float s = isA ? 1.0f : -1.0f;
            M3 jLin{basis[0] * s, basis[1] * s, basis[2] * s};
            V3 rW = isA ? rAW : rBW;
            M3 jAng{cross(rW, jLin.r0), cross(rW, jLin.r1), cross(rW, jLin.r2)};
            M3 K = mdiag(contacts[i].penalty);
            M3 jLinT = mT(jLin), jAngT = mT(jAng), jAngTk = mmul(jAngT, K);
            lhsLin = madd(lhsLin, mmul(mmul(jLinT, K), jLin));
            lhsAng = madd(lhsAng, mmul(jAngTk, jAng));
            lhsCross = madd(lhsCross, mmul(jAngTk, jLin));
            rhsLin += mmulv(jLinT, F);
            rhsAng += mmulv(jAngT, F);
        }
    }
    void update_dual(Solver& S) override {
        V3 dALin = a->positionLin - a->initialLin, dAAng = quat_sub(a->positionAng, a->initialAng);
        V3 dBLin = b->positionLin - b->initialLin, dBAng = quat_sub(b->positionAng, b->initialAng);
        for (size_t i = 0; i < contacts.size(); i++) {
            V3 rAW = anchor_offset(a, contacts[i].rA), rBW = anchor_offset(b, contacts[i].rB), F, C;
            float fs, bd;
            force_c(S, i, S.alpha, dALin, dAAng, dBLin, dBAng, rAW, rBW, F, C, fs, bd);
            V3 Fb = F;
            Fb.x = std::max(Fb.x, -S.lambdaMax);
            contacts[i].lambda = Fb;
            if (F.x < 0.0f) contacts[i].penalty.x = std::min(contacts[i].penalty.x + S.betaLin * std::fabs(C.x), PENALTY_MAX);
            if (fs <= bd) {
                contacts[i].penalty.y = std::min(contacts[i].penalty.y + S.betaLin * std::fabs(C.y), PENALTY_MAX_T);
                contacts[i].penalty.z = std::min(contacts[i].penalty.z + S.betaLin * std::fabs(C.z), PENALTY_MAX_T);
                contacts[i].stick = std::sqrt(C.y * C.y + C.z * C.z) < STICK_THRESH;
            }
        }
    }
};

// ---------------------------------------------------------------- step
void Solver::step() {
    for (const auto& sp : spinners) {
        Rigid* body = bodies[sp.body].get();
        float half = 0.5f * sp.omega * dt;
        V3 axis = normalize(v3(sp.axis[0], sp.axis[1], sp.axis[2]));
        Q dq{axis * std::sin(half), std::cos(half)};
        body->positionAng = qnorm(qmul(dq, body->positionAng));
    }
    // O(n^2) sphere broadphase (CPUSolver.swift:218-228)
    for (size_t i = 0; i < bodies.size(); i++) {
        for (size_t j = i + 1; j < bodies.size(); j++) {
            Rigid* a = bodies[i].get();
            Rigid* b = bodies[j].get();
            V3 dp = a->positionLin - b->positionLin;
            float r = a->radius + b->radius;
            if (dot(dp, dp) <= r * r && !constrained(a, b)) {
                Manifold* m = new Manifold();
                m->a = a;
                m->b = b;
                add_force(m);
            }
        }
    }
    std::vector<Force*> keep;
    keep.reserve(forces.size());
    for (Force* f : forces) {
        if (f->initialize(*this)) keep.push_back(f);
        else drop_from_bodies(f);
    }
    forces.swap(keep);
    const float g = gravity;
    for (auto& bp : bodies) {
        Rigid& b = *bp;
        b.inertialLin = b.positionLin + b.velocityLin * dt;
        if (b.mass > 0.0f) b.inertialLin += v3(0, 0, g * b.gravityScale) * (dt * dt);
        b.inertialAng = quat_add(b.positionAng, b.velocityAng * dt);
        V3 accel = (b.velocityLin - b.prevVelocityLin) / dt;
        float accelExt = accel.z * (g < 0.0f ? -1.0f : (g > 0.0f ? 1.0f : 0.0f));
        float w = clampf(accelExt / std::fabs(g), 0.0f, 1.0f);
        if (!std::isfinite(w)) w = 0.0f;
        b.initialLin = b.positionLin;
        b.initialAng = b.positionAng;
        if (b.mass > 0.0f) {
            b.positionLin += b.velocityLin * dt + v3(0, 0, g * b.gravityScale) * (w * dt * dt);
            b.positionAng = quat_add(b.positionAng, b.velocityAng * dt);
        }
    }
    for (int it = 0; it < iterations; it++) {
        for (auto& bp : bodies) {
            Rigid& b = *bp;
            if (!(b.mass > 0.0f)) continue;
            M3 lhsLin = mdiag(v3(b.mass / (dt * dt), b.mass / (dt * dt), b.mass / (dt * dt)));
            M3 inertia = mscale(world_inertia(b.positionAng, b.moment), 1.0f / (dt * dt));
            M3 lhsAng = inertia, lhsCross = mzero();
            V3 rhsLin = (b.positionLin - b.inertialLin) * (b.mass / (dt * dt));
            V3 rhsAng = mmulv(inertia, quat_sub(b.positionAng, b.inertialAng));
            for (Force* f : b.forces) f->update_primal(*this, &b, lhsLin, lhsAng, lhsCross, rhsLin, rhsAng);
            V3 dxLin{0, 0, 0}, dxAng{0, 0, 0};
            if (b.isParticle) { lhsAng = mident(); lhsCross = mzero(); rhsAng = v3(0, 0, 0); }
            solve6x6(lhsLin, lhsAng, lhsCross, -rhsLin, -rhsAng, dxLin, dxAng);
            b.positionLin += dxLin;
            b.positionAng = quat_add(b.positionAng, dxAng);
        }
        for (Force* f : forces) f->update_dual(*this);
    }
    for (auto& bp : bodies) {
        Rigid& b = *bp;
        b.prevVelocityLin = b.velocityLin;
        if (b.mass > 0.0f) {
            b.velocityLin = (b.positionLin - b.initialLin) / dt;
            b.velocityAng = quat_sub(b.positionAng, b.initialAng) / dt;
            if (!b.isParticle) {
                b.velocityLin = b.velocityLin * std::exp(-rigidLinearDamping * dt);
                b.velocityAng = b.velocityAng * std::exp(-rigidAngularDamping * dt);
            }
        }
    }
}

float Solver::max_constraint_error() const {
    float err = 0.0f;
    for (Force* f : forces) {
        if (Joint* j = dynamic_cast<Joint*>(f)) {
            if (j->stiffnessLin == 0.0f && j->stiffnessAng == 0.0f) continue;
            err = std::max(err, length(j->currentCLin()));
        } else if (Manifold* m = dynamic_cast<Manifold*>(f)) {
            for (size_t i = 0; i < m->contacts.size(); i++) err = std::max(err, std::max(0.0f, -m->penetration(*this, i)));
        }
    }
    return err;
}

// CPURigid.init (CPUSolver.swift:40-98) for boxes and spheres
static Rigid make_body(const avbd_body_desc& d) {
    Rigid r{};
    r.size = v3(d.size[0], d.size[1], d.size[2]);
    r.friction = d.friction;
    r.dynamicFriction = d.dynamic_friction;
    r.gravityScale = d.gravity_scale;
    r.positionLin = v3(d.position[0], d.position[1], d.position[2]);
    r.positionAng = Q{v3(d.rotation[0], d.rotation[1], d.rotation[2]), d.rotation[3]};
    r.initialAng = r.inertialAng = Q{v3(0, 0, 0), 1.0f};
    r.velocityLin = r.prevVelocityLin = v3(d.velocity[0], d.velocity[1], d.velocity[2]);
    r.velocityAng = v3(0, 0, 0);
    r.shape = d.shape;
    r.isParticle = d.is_particle != 0;
    if (d.shape == AVBD_SHAPE_SPHERE) {
        float rr = r.size.x / 2.0f;
        float m = d.density > 0.0f ? 4.0f / 3.0f * (float)M_PI * rr * rr * rr * d.density : 0.0f;
        r.mass = m;
        r.moment = v3(0.4f * m * rr * rr, 0.4f * m * rr * rr, 0.4f * m * rr * rr);
        r.radius = rr;
    } else {
        const V3 s = r.size;
        float m = s.x * s.y * s.z * d.density;
        r.mass = d.density > 0.0f ? m : 0.0f;
        r.moment = v3((s.y * s.y + s.z * s.z) / 12.0f * m, (s.x * s.x + s.z * s.z) / 12.0f * m,
                      (s.x * s.x + s.y * s.y) / 12.0f * m);
        r.radius = length(s * 0.5f);
    }
    if (d.has_explicit_mass) {
        r.mass = d.mass;
        r.moment = v3(d.diagonal_inertia[0], d.diagonal_inertia[1], d.diagonal_inertia[2]);
    }
    return r;
}

}  // namespace cpuref

using cpuref::Solver;

extern "C" {

// PhysicsScene.makeCPUSolver (CPU/PhysicsScene+CPUSolver.swift:5-62).
// Returns 0, or AVBD_ERR_UNSUPPORTED for scenes the CPU solver has no
// counterpart for here (tets, triangles, tori, capsules).
int cpu_solver_create(const avbd_scene_desc* s, void** out) {
    using namespace cpuref;
    if (!s || !out) return AVBD_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (s->num_tets || s->num_tris) return AVBD_ERR_UNSUPPORTED;
    for (uint32_t i = 0; i < s->num_bodies; i++)
        if (s->bodies[i].shape != AVBD_SHAPE_BOX && s->bodies[i].shape != AVBD_SHAPE_SPHERE) return AVBD_ERR_UNSUPPORTED;
    Solver* S = new Solver();
    const avbd_settings& st = s->settings;
    S->dt = st.dt; S->gravity = st.gravity; S->iterations = st.iterations; S->alpha = st.alpha;
    S->betaLin = st.beta_lin; S->betaAng = st.beta_ang; S->gamma = st.gamma; S->lambdaMax = st.lambda_max;
    S->collisionMargin = std::max(st.collision_margin, 0.0f); S->frictionCombineMode = st.friction_combine_mode;
    S->rigidLinearDamping = st.rigid_linear_damping; S->rigidAngularDamping = st.rigid_angular_damping;
    for (uint32_t i = 0; i < s->num_bodies; i++) S->bodies.emplace_back(new Rigid(make_body(s->bodies[i])));
    for (uint32_t i = 0; i < s->num_joints; i++) {
        const avbd_joint_desc& d = s->joints[i];
        Joint* j = new Joint();
        j->a = d.body_a >= 0 ? S->bodies[d.body_a].get() : nullptr;
        j->b = S->bodies[d.body_b].get();
        j->rA = v3(d.r_a[0], d.r_a[1], d.r_a[2]);
        j->rB = v3(d.r_b[0], d.r_b[1], d.r_b[2]);
        j->stiffnessLin = d.stiffness_lin;
        j->stiffnessAng = d.stiffness_ang;
        j->fracture = d.fracture;
        j->fractureLinear = d.fracture_linear != 0;
        V3 sa = j->a ? j->a->size : v3(0, 0, 0);
        j->torqueArm = len2(sa + j->b->size);
        if (j->stiffnessLin > 0.0f && std::isfinite(j->stiffnessLin)) {
            float p = std::min(j->stiffnessLin, 1e9f);
            j->penaltyLin = v3(p, p, p);
        }
        if (j->stiffnessAng > 0.0f && std::isfinite(j->stiffnessAng)) {
            float p = std::min(j->stiffnessAng, 1e9f);
            j->penaltyAng = v3(p, p, p);
        }
        Q qA0 = j->a ? j->a->positionAng : Q{v3(0, 0, 0), 1.0f};
        j->restRel = qnorm(qmul(qinv(qA0), j->b->positionAng));
        j->hasHinge = d.has_hinge != 0;
        j->hingeAxis = v3(d.hinge_axis[0], d.hinge_axis[1], d.hinge_axis[2]);
        S->add_force(j);
    }
    for (uint32_t i = 0; i < s->num_springs; i++) {
        const avbd_spring_desc& d = s->springs[i];
        Spring* sp = new Spring();
        sp->a = S->bodies[d.body_a].get();
        sp->b = S->bodies[d.body_b].get();
        sp->rA = v3(d.r_a[0], d.r_a[1], d.r_a[2]);
        sp->rB = v3(d.r_b[0], d.r_b[1], d.r_b[2]);
        sp->stiffness = d.stiffness;
        if (d.rest < 0.0f) {
            V3 pA = xform(sp->a->positionLin, sp->a->positionAng, sp->rA);
            V3 pB = xform(sp->b->positionLin, sp->b->positionAng, sp->rB);
            sp->rest = length(pA - pB);
        } else {
            sp->rest = d.rest;
        }
        sp->hard = d.hard != 0;
        S->add_force(sp);
    }
    for (uint32_t i = 0; i < s->num_spinners; i++) S->spinners.push_back(s->spinners[i]);
    *out = S;
    return AVBD_OK;
}

void cpu_solver_destroy(void* h) { delete static_cast<Solver*>(h); }

int cpu_solver_step(void* h, uint32_t frames) {
    Solver* S = static_cast<Solver*>(h);
    for (uint32_t f = 0; f < frames; f++) S->step();
    return AVBD_OK;
}

int cpu_solver_get_body_states(void* h, uint32_t n, avbd_body_state* out) {
    Solver* S = static_cast<Solver*>(h);
    if (n > S->bodies.size()) return AVBD_ERR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < n; i++) {
        const cpuref::Rigid& b = *S->bodies[i];
        avbd_body_state& o = out[i];
        o.position[0] = b.positionLin.x; o.position[1] = b.positionLin.y; o.position[2] = b.positionLin.z;
        o.rotation[0] = b.positionAng.v.x; o.rotation[1] = b.positionAng.v.y; o.rotation[2] = b.positionAng.v.z;
        o.rotation[3] = b.positionAng.w;
        o.velocity[0] = b.velocityLin.x; o.velocity[1] = b.velocityLin.y; o.velocity[2] = b.velocityLin.z;
        o.angular_velocity[0] = b.velocityAng.x; o.angular_velocity[1] = b.velocityAng.y;
        o.angular_velocity[2] = b.velocityAng.z;
    }
    return AVBD_OK;
}

float cpu_solver_max_constraint_error(void* h) { return static_cast<Solver*>(h)->max_constraint_error(); }

uint32_t cpu_solver_num_forces(void* h) { return (uint32_t)static_cast<Solver*>(h)->forces.size(); }

}  // extern "C"
