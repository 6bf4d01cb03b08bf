// narrowphase.cu — contact manifolds per candidate pair and the collider-
// pair-keyed persistence map.
//
// Follows Shaders/30_narrowphase.metal:17-263 (box SAT helpers),
// :978-1136 (sphere/sphere, sphere/box), :1138-1321 (box/box) and
// Shaders/20_broadphase.metal:547-608 (persistence map).  One thread per
// pair; each thread warm-starts its contacts from last frame's manifold of
// the same collider pair (map lookup + feature key or proximity match).
#include "dmath.cuh"
#include "kernels.h"

namespace avbd {

namespace {
constexpr float SAT_EPS = 1.0e-6f;
constexpr float PLANE_EPS = 1.0e-5f;
constexpr float MERGE_DIST_SQ = 1.0e-6f;
constexpr int NP_MAX_POLY = 16;

struct Box { float3 center, half, ax0, ax1, ax2; };
struct AxisBest { int type, ia, ib; float sep; float3 n; bool valid; };
struct Hit { float3 xA, xB; uint32_t feature; };

__device__ __forceinline__ float3 box_axis(const Box& b, int i) { return i == 0 ? b.ax0 : (i == 1 ? b.ax1 : b.ax2); }
__device__ __forceinline__ float box_half(const Box& b, int i) { return comp(b.half, i); }

__device__ __forceinline__ float spec_cap(float ra, float rb, float margin) {
    const float r = mn(fabsf(ra), fabsf(rb));
    return mn(0.25f, mx(4.0f * margin, 3.0f * r));
}
__device__ __forceinline__ float detect_margin(float3 n, float3 relVel, const Params& P, float ra, float rb) {
    const float approach = mx(0.0f, -dot(relVel, n));
    const float allowed = mn(approach * P.dt, spec_cap(ra, rb, P.collisionMargin));
    return P.collisionMargin + allowed;
}
__device__ bool test_axis(const Box& A, const Box& B, float3 delta, float3 axis, int type, int ia, int ib,
                          float3 relVel, float cap, const Params& P, AxisBest& best) {
    const float lenSq = dot(axis, axis);
    if (lenSq < SAT_EPS) return true;
    float3 n = axis * rsq(lenSq);
    if (dot(n, delta) < 0.0f) n = -n;
    const float dist = fabsf(dot(delta, n));
    const float rA = A.half.x * fabsf(dot(n, A.ax0)) + A.half.y * fabsf(dot(n, A.ax1)) + A.half.z * fabsf(dot(n, A.ax2));
    const float rB = B.half.x * fabsf(dot(n, B.ax0)) + B.half.y * fabsf(dot(n, B.ax1)) + B.half.z * fabsf(dot(n, B.ax2));
    const float sep = dist - (rA + rB);
    const float approach = mx(0.0f, -dot(relVel, n));
    const float allowed = mn(approach * P.dt, cap);
    if (sep > allowed) return false;
    if (!best.valid || sep > best.sep) { best.valid = true; best.type = type; best.ia = ia; best.ib = ib; best.sep = sep; best.n = n; }
    return true;
}
__device__ float3 support(const Box& b, float3 dir) {
    const float sx = dot(dir, b.ax0) >= 0.0f ? 1.0f : -1.0f;
    const float sy = dot(dir, b.ax1) >= 0.0f ? 1.0f : -1.0f;
    const float sz = dot(dir, b.ax2) >= 0.0f ? 1.0f : -1.0f;
    return b.center + b.ax0 * (b.half.x * sx) + b.ax1 * (b.half.y * sy) + b.ax2 * (b.half.z * sz);
}
__device__ void face_axes(const Box& b, int i, float3& u, float3& v, float& eu, float& ev) {
    if (i == 0) { u = b.ax1; v = b.ax2; eu = b.half.y; ev = b.half.z; }
    else if (i == 1) { u = b.ax0; v = b.ax2; eu = b.half.x; ev = b.half.z; }
    else { u = b.ax0; v = b.ax1; eu = b.half.x; ev = b.half.y; }
}
__device__ int clip_poly(const float3* in, int n, float3 nrm, float off, float3* out) {
    if (n <= 0) return 0;
    int m = 0;
    float3 a = in[n - 1];
    float da = dot(nrm, a) - off;
    for (int i = 0; i < n; i++) {
        const float3 b = in[i];
        const float db = dot(nrm, b) - off;
        const bool aIn = da <= PLANE_EPS, bIn = db <= PLANE_EPS;
        if (aIn != bIn) {
            float t = 0.0f;
            const float den = da - db;
            if (fabsf(den) > SAT_EPS) t = clampf(da / den, 0.0f, 1.0f);
            if (m < NP_MAX_POLY) out[m++] = a + (b - a) * t;
        }
        if (bIn && m < NP_MAX_POLY) out[m++] = b;
        a = b;
        da = db;
    }
    return m;
}
__device__ void support_edge(const Box& b, int axis, float3 dir, float3& eA, float3& eB) {
    const int a1 = (axis + 1) % 3, a2 = (axis + 2) % 3;
    const float s1 = dot(dir, box_axis(b, a1)) >= 0.0f ? 1.0f : -1.0f;
    const float s2 = dot(dir, box_axis(b, a2)) >= 0.0f ? 1.0f : -1.0f;
    const float3 c = b.center + box_axis(b, a1) * (box_half(b, a1) * s1) + box_axis(b, a2) * (box_half(b, a2) * s2);
    eA = c - box_axis(b, axis) * box_half(b, axis);
    eB = c + box_axis(b, axis) * box_half(b, axis);
}
__device__ void closest_seg_seg(float3 p0, float3 p1, float3 q0, float3 q1, float3& c0, float3& c1) {
    const float3 d1 = p1 - p0, d2 = q1 - q0, r = p0 - q0;
    const float a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    float s = 0.0f, t = 0.0f;
    if (a <= SAT_EPS && e <= SAT_EPS) { c0 = p0; c1 = q0; return; }
    if (a <= SAT_EPS) {
        t = clampf(f / e, 0.0f, 1.0f);
    } else {
        const float c = dot(d1, r);
        if (e <= SAT_EPS) {
            s = clampf(-c / a, 0.0f, 1.0f);
        } else {
            const float b = dot(d1, d2);
            const float den = a * e - b * b;
            if (fabsf(den) > SAT_EPS) s = clampf((b * f - c * e) / den, 0.0f, 1.0f);
            t = (b * s + f) / e;
            if (t < 0.0f) { t = 0.0f; s = clampf(-c / a, 0.0f, 1.0f); }
            else if (t > 1.0f) { t = 1.0f; s = clampf((b - c) / a, 0.0f, 1.0f); }
        }
    }
    c0 = p0 + d1 * s;
    c1 = q0 + d2 * t;
}
__device__ bool add_contact(Hit* cs, int& count, float3* mids, float3 xA, float3 xB, uint32_t feature) {
    const float3 mid = (xA + xB) * 0.5f;
    for (int i = 0; i < count; i++) if (dist2(mid, mids[i]) < MERGE_DIST_SQ) return false;
    if (count >= MAX_CONTACTS) return false;
    cs[count].xA = xA; cs[count].xB = xB; cs[count].feature = feature;
    mids[count] = mid;
    count++;
    return true;
}
__device__ __forceinline__ void spin_shift(float4 wA, float4 wB, float3 rAoff, float3 rBoff, float3 t1, float3 t2,
                                           float dt, float alpha, float& sx, float& sy) {
    const float3 sA = wA.w != 0.0f ? cross(xyz(wA), rAoff) * dt : s3(0);
    const float3 sB = wB.w != 0.0f ? cross(xyz(wB), rBoff) * dt : s3(0);
    const float3 rel = sB - sA;
    const float k = 1.0f / mx(1.0f - alpha, 0.01f);
    sx = dot(t1, rel) * k;
    sy = dot(t2, rel) * k;
}
__device__ __forceinline__ float3 penalty_floor(const DevPtrs& d, const Params& P, uint32_t ia, uint32_t ib) {
    const float mA = d.posLin[ia].w, mB = d.posLin[ib].w;
    const float minMass = mn(mA > 0.0f ? mA : 3.402823466e38f, mB > 0.0f ? mB : 3.402823466e38f);
    if (minMass == 3.402823466e38f) return s3(PENALTY_MIN);
    const float k = mn(PENALTY_MAX, mx(PENALTY_MIN, minMass / mx(P.dt * P.dt, 1e-12f)));
    return mk3(k, mn(k, PENALTY_MAX_T), mn(k, PENALTY_MAX_T));
}
__device__ int map_find(const DevPtrs& d, const Params& P, uint32_t a, uint32_t b) {
    uint32_t h = pair_map_hash(a, b, P.mapCapacity);
    for (uint32_t probe = 0; probe < P.mapCapacity; probe++) {
        const uint32_t ka = d.mapKeyA[h];
        if (ka == 0) return -1;
        if (ka == a + 1 && d.mapKeyB[h] == b) return (int)d.mapVal[h];
        h = (h + 1) & (P.mapCapacity - 1u);
    }
    return -1;
}
__device__ __forceinline__ void write_contact(ManifoldGPU& m, int i, float3 rA, uint32_t feature, float3 rB,
                                              float stick, float3 C0, float3 lambda, float3 penalty) {
    m.contacts[i].rA = tof4(rA, __uint_as_float(feature));
    m.contacts[i].rB = tof4(rB, stick);
    m.contacts[i].C0 = tof4(C0, 0.0f);
    m.contacts[i].lambda = tof4(lambda, 0.0f);
    m.contacts[i].penalty = tof4(penalty, 0.0f);
}

// One candidate pair as np_collide forms it (30_narrowphase.metal:396-428):
// owning bodies, collider centres and rotations, contact-point velocities.
struct NPair {
    uint32_t ia, ib, ba, bb;
    float4 bodyPA, bodyPB, qBodyA, qBodyB, qA, qB, cshA, cshB;
    float3 vA, vB;
    Box A, B;
};

// Contacts matched to last frame's by feature key, anchors in body frames
// (box/box and convex-hull/box, 30_narrowphase.metal:490-545 and :1280-1321).
__device__ void emit_feature_manifold(const Params& P, const DevPtrs& d, const NPair& p, ManifoldGPU& outM,
                                      const Hit* contacts, int count, float3 nrm) {
    float3 t1, t2;
    orthonormal(nrm, t1, t2);
    const float2 frA = d.colFriction[p.ia], frB = d.colFriction[p.ib];
    const float sf = combine_friction(frA.x, frB.x, P.frictionCombineMode);
    const float df = combine_friction(frA.y, frB.y, P.frictionCombineMode);
    const int prev = map_find(d, P, p.ia, p.ib);
    outM.header = u4{p.ba, p.bb, (uint32_t)count, 1u};
    outM.basisN = tof4(nrm, df);
    outM.basisT1 = tof4(t1, sf);
    const float warm = P.alpha * P.gamma;
    const float4 qAc = q_conj(p.qBodyA), qBc = q_conj(p.qBodyB);
    for (int i = 0; i < count; i++) {
        float3 rA = q_rotate(qAc, contacts[i].xA - xyz(p.bodyPA));
        float3 rB = q_rotate(qBc, contacts[i].xB - xyz(p.bodyPB));
        float3 lambda = s3(0), penalty = s3(0);
        float stick = 0.0f;
        if (prev >= 0) {
            const ManifoldGPU& pm = d.prevManifolds[prev];
            for (uint32_t j = 0; j < pm.header.z; j++) {
                if (__float_as_uint(pm.contacts[j].rA.w) == contacts[i].feature) {
                    lambda = xyz(pm.contacts[j].lambda);
                    penalty = xyz(pm.contacts[j].penalty);
                    stick = pm.contacts[j].rB.w;
                    if (stick != 0.0f) { rA = xyz(pm.contacts[j].rA); rB = xyz(pm.contacts[j].rB); }
                    break;
                }
            }
        }
        const float3 xAw = xform(xyz(p.bodyPA), p.qBodyA, rA);
        const float3 xBw = xform(xyz(p.bodyPB), p.qBodyB, rB);
        const float3 dd = xAw - xBw;
        float3 C0 = mk3(dot(nrm, dd) + P.collisionMargin, dot(t1, dd), dot(t2, dd));
        float sx, sy;
        spin_shift(d.spinVel[p.ba], d.spinVel[p.bb], xAw - xyz(p.bodyPA), xBw - xyz(p.bodyPB), t1, t2, P.dt, P.alpha, sx, sy);
        C0.y -= sx;
        C0.z -= sy;
        lambda *= warm;
        penalty = clamp3(penalty * P.gamma, penalty_floor(d, P, p.ba, p.bb), mk3(PENALTY_MAX, PENALTY_MAX_T, PENALTY_MAX_T));
        write_contact(outM, i, rA, contacts[i].feature, rB, stick, C0, lambda, penalty);
    }
}

// Which previous anchors a round contact keeps while it sticks: spheres keep
// them unless a world-space round anchor belongs to a rigid body (:1088-1100),
// capsules only between two material-anchored colliders (:711-724), tori
// never (:944-962).
enum { STICK_SPHERE = 0, STICK_CAPSULE = 1, STICK_NONE = 2 };

// Contacts on round shapes, matched to last frame's by anchor proximity with
// the tangential dual carried into the new basis (sphere, capsule, torus:
// 30_narrowphase.metal:668-745, :910-975, :1058-1136).
__device__ void emit_round_manifold(const Params& P, const DevPtrs& d, const NPair& p, ManifoldGPU& outM,
                                    const Hit* contacts, int count, float3 nrm, float matchDist, int stickRule) {
    float3 t1, t2;
    orthonormal(nrm, t1, t2);
    const float2 frA = d.colFriction[p.ia], frB = d.colFriction[p.ib];
    const float sf = combine_friction(frA.x, frB.x, P.frictionCombineMode);
    const float df = combine_friction(frA.y, frB.y, P.frictionCombineMode);
    const int prev = map_find(d, P, p.ia, p.ib);
    const bool roundA = (d.colShapeType[p.ia] & COLLIDER_WORLD_ROUND_ANCHOR) != 0;
    const bool roundB = (d.colShapeType[p.ib] & COLLIDER_WORLD_ROUND_ANCHOR) != 0;
    outM.header = u4{p.ba, p.bb, (uint32_t)count, 1u | (roundA ? 2u : 0u) | (roundB ? 4u : 0u)};
    outM.basisN = tof4(nrm, df);
    outM.basisT1 = tof4(t1, sf);
    const float warm = P.alpha * P.gamma;
    const float4 qAc = q_conj(p.qBodyA), qBc = q_conj(p.qBodyB);
    bool keepAnchors;
    if (stickRule == STICK_SPHERE) keepAnchors = (p.cshA.w < 0.0f || !roundA) && (p.cshB.w < 0.0f || !roundB);
    else if (stickRule == STICK_CAPSULE) keepAnchors = !roundA && !roundB;
    else keepAnchors = false;
    for (int i = 0; i < count; i++) {
        float3 rA_ = roundA ? contacts[i].xA - xyz(p.bodyPA) : q_rotate(qAc, contacts[i].xA - xyz(p.bodyPA));
        float3 rB_ = roundB ? contacts[i].xB - xyz(p.bodyPB) : q_rotate(qBc, contacts[i].xB - xyz(p.bodyPB));
        float3 lambda = s3(0), penalty = s3(0);
        float stick = 0.0f;
        if (prev >= 0) {
            const ManifoldGPU& pm = d.prevManifolds[prev];
            const uint32_t pn = pm.header.z;
            float bestD = matchDist;
            int bestJ = -1;
            for (uint32_t j = 0; j < pn; j++) {
                const float dj = dist3(xyz(pm.contacts[j].rA), rA_);
                if (dj < bestD) { bestD = dj; bestJ = (int)j; }
            }
            if (bestJ >= 0) {
                lambda = xyz(pm.contacts[bestJ].lambda);
                penalty = xyz(pm.contacts[bestJ].penalty);
                const float3 t1o = xyz(pm.basisT1);
                const float3 t2o = cross(xyz(pm.basisN), t1o);
                const float3 lt = t1o * lambda.y + t2o * lambda.z;
                lambda.y = dot(t1, lt);
                lambda.z = dot(t2, lt);
                if (keepAnchors) {
                    stick = pm.contacts[bestJ].rB.w;
                    if (stick != 0.0f) { rA_ = xyz(pm.contacts[bestJ].rA); rB_ = xyz(pm.contacts[bestJ].rB); }
                }
            }
        }
        // tori measure the gap between the hit points themselves
        // (30_narrowphase.metal:925-958); capsules and spheres between the
        // points their stored anchors give back (:727-731, :1115-1119)
        const bool fromHits = stickRule == STICK_NONE;
        const float3 xAw = fromHits ? contacts[i].xA
                                    : (roundA ? xyz(p.bodyPA) + rA_ : xform(xyz(p.bodyPA), p.qBodyA, rA_));
        const float3 xBw = fromHits ? contacts[i].xB
                                    : (roundB ? xyz(p.bodyPB) + rB_ : xform(xyz(p.bodyPB), p.qBodyB, rB_));
        const float3 dd = xAw - xBw;
        float3 C0 = mk3(dot(nrm, dd) + P.collisionMargin, dot(t1, dd), dot(t2, dd));
        float sx, sy;
        spin_shift(d.spinVel[p.ba], d.spinVel[p.bb], xAw - xyz(p.bodyPA), xBw - xyz(p.bodyPB), t1, t2, P.dt, P.alpha, sx, sy);
        C0.y -= sx;
        C0.z -= sy;
        lambda *= warm;
        penalty = clamp3(penalty * P.gamma, penalty_floor(d, P, p.ba, p.bb), mk3(PENALTY_MAX, PENALTY_MAX_T, PENALTY_MAX_T));
        write_contact(outM, i, rA_, contacts[i].feature, rB_, stick, C0, lambda, penalty);
    }
}

// Index of the smallest component, first on ties (the face a point inside a
// box leaves through).
__device__ __forceinline__ int min_axis(float3 v) {
    int a = 0;
    if (v.y < comp(v, a)) a = 1;
    if (v.z < comp(v, a)) a = 2;
    return a;
}

// Closest point of segment ab to p (30_narrowphase.metal:286-290).
__device__ __forceinline__ float3 closest_on_segment(float3 p, float3 a, float3 b) {
    const float3 ab = b - a;
    const float t = clampf(dot(p - a, ab) / mx(dot(ab, ab), 1e-12f), 0.0f, 1.0f);
    return a + ab * t;
}

// ---- convex hull vs box (30_narrowphase.metal:189-246, :430-545)
struct HullCand { float3 xHull, xBox, boxToHull; float sep; uint32_t feature; };

// One hull vertex against the box: inside, it leaves through the nearest
// face; outside, the clamped point is a candidate within the velocity-aware
// detection margin.
__device__ bool hull_vertex_box(float3 vw, uint32_t vid, const Box& box, float4 qBox, float3 relHullBox,
                                float hullR, float boxR, const Params& P, HullCand& out) {
    const float3 local = q_rotate(q_conj(qBox), vw - box.center);
    const float3 h = box.half;
    const float3 cl = clamp3(local, -h, h);
    float3 nL, bL;
    float sep;
    const bool inside = local.x >= -h.x && local.y >= -h.y && local.z >= -h.z &&
                        local.x <= h.x && local.y <= h.y && local.z <= h.z;
    if (inside) {
        const float3 clr = h - abs3(local);
        const int axis = min_axis(clr);
        nL = s3(0);
        setcomp(nL, axis, comp(local, axis) >= 0.0f ? 1.0f : -1.0f);
        bL = local;
        setcomp(bL, axis, comp(nL, axis) * comp(h, axis));
        sep = -comp(clr, axis);
    } else {
        const float3 dl = local - cl;
        const float dist = len3(dl);
        if (dist < 1e-8f) return false;
        nL = dl / dist;
        const float det = detect_margin(q_rotate(qBox, nL), relHullBox, P, hullR, boxR);
        if (dist > det) return false;
        bL = cl;
        sep = dist;
    }
    out.xHull = vw;
    out.xBox = q_rotate(qBox, bL) + box.center;
    out.boxToHull = q_rotate(qBox, nL);
    out.sep = sep;
    out.feature = (4u << 24) | (vid & 0x00FFFFFFu);
    return true;
}

__device__ __noinline__ void narrow_hull(const Params& P, const DevPtrs& d, const NPair& p, ManifoldGPU& outM,
                                         uint32_t stA, uint32_t stB) {
    const bool hIsA = stA == 4;
    // convex-vs-box only; other pairs with a hull produce no contact
    if ((stA == 4 && stB == 4) || (hIsA ? stB : stA) != 0) { outM.header = u4{p.ba, p.bb, 0, 0}; return; }
    const uint32_t ih = hIsA ? p.ia : p.ib;
    const float4 qH = hIsA ? p.qA : p.qB;
    const float3 pH = hIsA ? p.A.center : p.B.center;
    const Box& box = hIsA ? p.B : p.A;
    const float4 qBox = hIsA ? p.qB : p.qA;
    const float3 rel = hIsA ? (p.vA - p.vB) : (p.vB - p.vA);
    const float hullR = fabsf(d.colShape[ih].w);
    const float boxR = fabsf(d.colShape[hIsA ? p.ib : p.ia].w);
    const uint2 range = d.colHullRange[ih];
    HullCand best;
    bool have = false;
    for (uint32_t v = 0; v < range.y; v++) {
        const float3 vw = pH + q_rotate(qH, xyz(d.hullVerts[range.x + v]));
        HullCand c;
        if (!hull_vertex_box(vw, v, box, qBox, rel, hullR, boxR, P, c)) continue;
        if (!have || c.sep < best.sep - 1e-8f || (fabsf(c.sep - best.sep) <= 1e-8f && c.feature < best.feature)) {
            best = c;
            have = true;
        }
    }
    if (!have) { outM.header = u4{p.ba, p.bb, 0, 0}; return; }
    // greedy: the deepest vertex, then vertices of the same face spread
    // widest across the contact plane
    HullCand chosen[MAX_CONTACTS];
    int count = 1;
    chosen[0] = best;
    const float band = 0.75f * P.collisionMargin;
    while (count < MAX_CONTACTS) {
        HullCand next;
        bool haveNext = false;
        float bestSpread = -1.0f;
        for (uint32_t v = 0; v < range.y; v++) {
            const float3 vw = pH + q_rotate(qH, xyz(d.hullVerts[range.x + v]));
            HullCand c;
            if (!hull_vertex_box(vw, v, box, qBox, rel, hullR, boxR, P, c)) continue;
            if (c.sep > best.sep + band || dot(c.boxToHull, best.boxToHull) < 0.98f) continue;
            bool dup = false;
            float minSpread = 3.402823466e38f;
            for (int j = 0; j < count; j++) {
                if (c.feature == chosen[j].feature) { dup = true; break; }
                float3 dd = c.xHull - chosen[j].xHull;
                dd -= best.boxToHull * dot(best.boxToHull, dd);
                minSpread = mn(minSpread, dot(dd, dd));
            }
            if (dup) continue;
            if (!haveNext || minSpread > bestSpread + 1e-10f ||
                (fabsf(minSpread - bestSpread) <= 1e-10f && c.feature < next.feature)) {
                next = c;
                bestSpread = minSpread;
                haveNext = true;
            }
        }
        if (!haveNext || bestSpread < MERGE_DIST_SQ) break;
        chosen[count++] = next;
    }
    Hit contacts[MAX_CONTACTS];
    for (int i = 0; i < count; i++) {
        contacts[i].xA = hIsA ? chosen[i].xHull : chosen[i].xBox;
        contacts[i].xB = hIsA ? chosen[i].xBox : chosen[i].xHull;
        contacts[i].feature = chosen[i].feature;
    }
    emit_feature_manifold(P, d, p, outM, contacts, count, hIsA ? best.boxToHull : -best.boxToHull);
}

// ---- capsule vs sphere / capsule / box (30_narrowphase.metal:547-745)
__device__ __noinline__ void narrow_capsule(const Params& P, const DevPtrs& d, const NPair& p, ManifoldGPU& outM,
                                            uint32_t stA, uint32_t stB) {
    const bool cIsA = stA == 3;
    const uint32_t ic = cIsA ? p.ia : p.ib, io = cIsA ? p.ib : p.ia;
    const float4 qC = cIsA ? p.qA : p.qB, qO = cIsA ? p.qB : p.qA;
    const float3 pC = cIsA ? p.A.center : p.B.center, pO = cIsA ? p.B.center : p.A.center;
    const float4 shC = d.colShape[ic], shO = d.colShape[io];
    const float half_ = shC.x * 0.5f, rc = shC.y;
    const float3 axC = q_rotate(qC, mk3(0, 0, 1));
    const float3 c0 = pC - axC * half_, c1 = pC + axC * half_;
    const uint32_t other = cIsA ? stB : stA;
    const float3 relCO = cIsA ? (p.vB - p.vA) : (p.vA - p.vB);
    Hit hits[3];
    int nh = 0;
    float3 nCO = mk3(0, 0, 1);  // capsule -> other
    if (other == 1) {
        const float rs = shO.x * 0.5f;
        const float3 q = closest_on_segment(pO, c0, c1);
        const float3 dd = pO - q;
        const float dist = len3(dd);
        const float3 nT = dist > 1e-6f ? dd / dist : mk3(0, 0, 1);
        const float dm = detect_margin(nT, relCO, P, shC.w, shO.w);
        if (dist <= rc + rs + dm) {
            nCO = nT;
            hits[0].xA = q + nCO * rc;
            hits[0].xB = pO - nCO * rs;
            hits[0].feature = 0;
            nh = 1;
        }
    } else if (other == 3) {
        const float halfO = shO.x * 0.5f, ro = shO.y;
        const float3 axO = q_rotate(qO, mk3(0, 0, 1));
        const float3 o0 = pO - axO * halfO, o1 = pO + axO * halfO;
        float3 qa, qb;
        closest_seg_seg(c0, c1, o0, o1, qa, qb);
        const float3 dd = qb - qa;
        const float dist = len3(dd);
        const float3 nT = dist > 1e-6f ? dd / dist : mk3(0, 0, 1);
        const float dm = detect_margin(nT, relCO, P, shC.w, shO.w);
        if (dist <= rc + ro + dm) {
            nCO = nT;
            hits[0].xA = qa + nCO * rc;
            hits[0].xB = qb - nCO * ro;
            hits[0].feature = 0;
            nh = 1;
        }
    } else {
        // capsule - box: alternate box clamp and segment projection from
        // three seeds along the axis
        const float4 qOc = q_conj(qO);
        const float3 halfO = xyz(shO) * 0.5f;
        float3 nAccum = s3(0);
        for (int seed = 0; seed < 3 && nh < 3; seed++) {
            const float t = (float)seed * 0.5f;
            float3 q = c0 + (c1 - c0) * t;
            float3 bw = q;
            for (int it = 0; it < 5; it++) {
                const float3 lb = clamp3(q_rotate(qOc, q - pO), -halfO, halfO);
                bw = q_rotate(qO, lb) + pO;
                q = closest_on_segment(bw, c0, c1);
            }
            const float3 dd = bw - q;
            const float dist = len3(dd);
            float3 n;
            if (dist < 1e-6f) {
                const float3 lb = q_rotate(qOc, q - pO);
                const float3 pen = halfO - abs3(lb);
                const int axis = min_axis(pen);
                float3 nl = s3(0);
                setcomp(nl, axis, comp(lb, axis) >= 0.0f ? 1.0f : -1.0f);
                n = -q_rotate(qO, nl);
                bw = q - n * comp(pen, axis);
            } else {
                n = dd / dist;
                const float dm = detect_margin(n, relCO, P, shC.w, shO.w);
                if (dist - rc > dm) continue;
            }
            bool dup = false;
            for (int h = 0; h < nh; h++)
                if (dist3(hits[h].xA, q + n * rc) < 0.4f * rc + 0.05f) { dup = true; break; }
            if (dup) continue;
            hits[nh].xA = q + n * rc;
            hits[nh].xB = bw;
            hits[nh].feature = (uint32_t)seed;
            nAccum += n;
            nh++;
        }
        if (nh > 0) nCO = nrm3(nAccum);
    }
    if (nh == 0) { outM.header = u4{p.ba, p.bb, 0, 0}; return; }
    Hit contacts[3];
    for (int i = 0; i < nh; i++) {
        contacts[i].xA = cIsA ? hits[i].xA : hits[i].xB;
        contacts[i].xB = cIsA ? hits[i].xB : hits[i].xA;
        contacts[i].feature = hits[i].feature;
    }
    emit_round_manifold(P, d, p, outM, contacts, nh, cIsA ? -nCO : nCO, 0.6f * (shC.y + 0.2f), STICK_CAPSULE);
}

// ---- torus vs sphere / box / capsule / torus (30_narrowphase.metal:292-340, :747-975)
struct Torus { float3 center, axis, u, v; float R, r; };

__device__ Torus torus_frame(float3 pos, float4 q, float R, float r) {
    Torus t;
    t.center = pos;
    t.axis = q_rotate(q, mk3(0, 0, 1));
    t.u = fabsf(t.axis.x) > fabsf(t.axis.z) ? mk3(-t.axis.y, t.axis.x, 0.0f) : mk3(0.0f, -t.axis.z, t.axis.y);
    t.u = nrm3(t.u);
    t.v = cross(t.axis, t.u);
    t.R = R;
    t.r = r;
    return t;
}

// Nearest point of the spine circle.
__device__ float3 torus_spine(const Torus& t, float3 p) {
    float3 dd = p - t.center;
    dd -= t.axis * dot(t.axis, dd);
    const float l = len3(dd);
    return l < 1e-6f ? t.center + t.u * t.R : t.center + dd / l * t.R;
}

// cos and sin of the 32 spine sample angles float(i) / 32 * 2 * pi (each the
// correctly rounded value at that float angle).
__constant__ float kSpineCos[32] = {
    1.0f, 0.980785251f, 0.923879504f, 0.831469595f, 0.707106769f, 0.555570185f, 0.382683426f, 0.195090234f,
    -4.37113883e-08f, -0.195090324f, -0.382683516f, -0.555570364f, -0.707106769f, -0.831469655f, -0.923879623f,
    -0.98078531f, -1.0f, -0.980785251f, -0.923879504f, -0.831469536f, -0.70710665f, -0.555570006f, -0.382683128f,
    -0.195090383f, 1.19248806e-08f, 0.195090413f, 0.382683605f, 0.555570424f, 0.707107008f, 0.831469595f,
    0.923879564f, 0.98078531f};
__constant__ float kSpineSin[32] = {
    0.0f, 0.195090324f, 0.382683456f, 0.555570245f, 0.707106769f, 0.831469655f, 0.923879504f, 0.98078531f,
    1.0f, 0.980785251f, 0.923879504f, 0.831469536f, 0.707106769f, 0.555570185f, 0.382683277f, 0.195090309f,
    -8.74227766e-08f, -0.195090488f, -0.382683426f, -0.555570304f, -0.707106888f, -0.831469774f, -0.923879683f,
    -0.980785251f, -1.0f, -0.980785251f, -0.923879445f, -0.831469476f, -0.707106531f, -0.555570304f,
    -0.382683426f, -0.195090234f};

struct TorusHit { float3 xT, xO, n; float sep; uint32_t feature; };

__device__ __noinline__ void narrow_torus(const Params& P, const DevPtrs& d, const NPair& p, ManifoldGPU& outM,
                                          uint32_t stA, uint32_t stB) {
    const bool tIsA = stA == 2;
    const uint32_t it = tIsA ? p.ia : p.ib, io = tIsA ? p.ib : p.ia;
    const float4 qT = tIsA ? p.qA : p.qB, qO = tIsA ? p.qB : p.qA;
    const float3 pT = tIsA ? p.A.center : p.B.center, pO = tIsA ? p.B.center : p.A.center;
    const float4 shT = d.colShape[it], shO = d.colShape[io];
    const Torus T = torus_frame(pT, qT, shT.x, shT.y);
    const uint32_t other = tIsA ? stB : stA;
    // catches fast approaches before deep penetration
    const float detectM = mx(P.collisionMargin, 0.8f * T.r);
    TorusHit hits[4];
    int nHits = 0;
    if (other == 1) {
        const float rs = shO.x * 0.5f;
        const float3 spine = torus_spine(T, pO);
        const float3 dd = pO - spine;
        const float dist = len3(dd);
        if (dist <= T.r + rs + detectM) {
            const float3 n = dist > 1e-6f ? dd / dist : mk3(0, 0, 1);  // torus -> sphere
            hits[0].xT = spine + n * T.r;
            hits[0].xO = pO - n * rs;
            hits[0].n = -n;
            hits[0].sep = dist - T.r - rs;
            hits[0].feature = 0;
            nHits = 1;
        }
    } else {
        // sample the spine; each sample has an exact closest point on the
        // other shape; refine the deepest angularly spread samples by two
        // alternating projections
        constexpr int NSAMP = 32;
        const bool isBox = other == 0, isCap = other == 3;
        Torus T2{};
        const float4 qOc = q_conj(qO);
        const float3 halfO = xyz(shO) * 0.5f;
        float otherR = 0.0f;
        float3 cs0 = s3(0), cs1 = s3(0);
        if (isCap) {
            const float chalf = shO.x * 0.5f;
            const float3 axO = q_rotate(qO, mk3(0, 0, 1));
            cs0 = pO - axO * chalf;
            cs1 = pO + axO * chalf;
            otherR = shO.y;
        } else if (!isBox) {
            T2 = torus_frame(pO, qO, shO.x, shO.y);
            otherR = T2.r;
        }
        auto closest_other = [&](float3 q) {
            if (isBox) return q_rotate(qO, clamp3(q_rotate(qOc, q - pO), -halfO, halfO)) + pO;
            if (isCap) return closest_on_segment(q, cs0, cs1);
            return torus_spine(T2, q);
        };
        float dists[NSAMP];
        float3 closest[NSAMP];
#pragma unroll 1
        for (int i = 0; i < NSAMP; i++) {
            const float3 q = T.center + (T.u * kSpineCos[i] + T.v * kSpineSin[i]) * T.R;
            const float3 b = closest_other(q);
            closest[i] = b;
            dists[i] = dist3(q, b);
        }
        uint32_t used = 0;
        for (int pick = 0; pick < 4; pick++) {
            int best = -1;
            float bd = 3.402823466e38f;
#pragma unroll 1
            for (int i = 0; i < NSAMP; i++) {
                if ((used >> i) & 1u) continue;
                if (dists[i] < bd) { bd = dists[i]; best = i; }
            }
            if (best < 0) break;
            if (bd - T.r - otherR > detectM) break;
            for (int k = -3; k <= 3; k++) used |= 1u << ((best + k + NSAMP) % NSAMP);  // 45 degrees
            float3 q = T.center + (T.u * kSpineCos[best] + T.v * kSpineSin[best]) * T.R;
            float3 b = closest[best];
            for (int it2 = 0; it2 < 2; it2++) {
                q = torus_spine(T, b);
                b = closest_other(q);
            }
            const float3 dd = q - b;
            const float dist = len3(dd);
            float3 n;
            float3 xO_ = b;
            if (dist < 1e-6f) {
                if (isBox) {
                    // spine inside the box: leave through the nearest face
                    const float3 lb = q_rotate(qOc, q - pO);
                    const float3 pen = halfO - abs3(lb);
                    const int axis = min_axis(pen);
                    float3 nl = s3(0);
                    setcomp(nl, axis, comp(lb, axis) >= 0.0f ? 1.0f : -1.0f);
                    n = q_rotate(qO, nl);
                    xO_ = q + n * comp(pen, axis);
                } else if (isCap) {
                    n = nrm3(cross(T.axis, nrm3(cs1 - cs0)) + mk3(1e-4f, 0, 0));
                } else {
                    n = nrm3(cross(T.axis, T2.axis) + mk3(1e-4f, 0, 0));
                }
            } else {
                if (dist - T.r - otherR > detectM) continue;
                n = dd / dist;  // other -> torus
            }
            hits[nHits].xT = q - n * T.r;
            hits[nHits].xO = xO_ + (isBox ? s3(0) : n * otherR);
            hits[nHits].n = n;
            hits[nHits].sep = dist - T.r - otherR;
            hits[nHits].feature = (uint32_t)best;
            nHits++;
        }
    }
    if (nHits == 0) { outM.header = u4{p.ba, p.bb, 0, 0}; return; }
    // the deepest contact's normal defines the basis
    int deep = 0;
    float minSep = 3.402823466e38f;
    for (int h = 0; h < nHits; h++)
        if (hits[h].sep < minSep) { minSep = hits[h].sep; deep = h; }
    const float3 nT = hits[deep].n;  // other -> torus
    Hit contacts[4];
    for (int i = 0; i < nHits; i++) {
        contacts[i].xA = tIsA ? hits[i].xT : hits[i].xO;
        contacts[i].xB = tIsA ? hits[i].xO : hits[i].xT;
        contacts[i].feature = hits[i].feature;
    }
    emit_round_manifold(P, d, p, outM, contacts, nHits, tIsA ? nT : -nT, 1.1f * shT.x, STICK_NONE);
}
}  // namespace

// ROUND = false: box and sphere pairs; ROUND = true: pairs with a torus,
// capsule or convex hull (a second pass, launched only for scenes that have
// such colliders, so that the common pass keeps its register budget).
template <bool ROUND>
__device__ void narrow_one(const Params& P, const DevPtrs& d, uint32_t gid) {
    const uint2 pr = d.pairs[gid];
    NPair p;
    p.ia = pr.x;
    p.ib = pr.y;
    const uint32_t ia = p.ia, ib = p.ib;
    p.ba = d.colOwner[ia];
    p.bb = d.colOwner[ib];
    const uint32_t ba = p.ba, bb = p.bb;
    p.bodyPA = d.posLin[ba];
    p.bodyPB = d.posLin[bb];
    p.qBodyA = d.posAng[ba];
    p.qBodyB = d.posAng[bb];
    const float3 centerA = xyz(p.bodyPA) + q_rotate(p.qBodyA, xyz(d.colLocalPos[ia]));
    const float3 centerB = xyz(p.bodyPB) + q_rotate(p.qBodyB, xyz(d.colLocalPos[ib]));
    p.qA = q_mul(p.qBodyA, d.colLocalRot[ia]);
    p.qB = q_mul(p.qBodyB, d.colLocalRot[ib]);
    p.vA = xyz(d.velLin[ba]) + cross(xyz(d.velAng[ba]), centerA - xyz(p.bodyPA));
    p.vB = xyz(d.velLin[bb]) + cross(xyz(d.velAng[bb]), centerB - xyz(p.bodyPB));
    const float3 vA = p.vA, vB = p.vB;
    const float3 relVel = vB - vA;
    p.cshA = d.colShape[ia];
    p.cshB = d.colShape[ib];
    const float4 cshA = p.cshA, cshB = p.cshB;
    Box& A = p.A;
    Box& B = p.B;
    A.center = centerA; A.half = xyz(cshA) * 0.5f;
    A.ax0 = q_rotate(p.qA, mk3(1, 0, 0)); A.ax1 = q_rotate(p.qA, mk3(0, 1, 0)); A.ax2 = q_rotate(p.qA, mk3(0, 0, 1));
    B.center = centerB; B.half = xyz(cshB) * 0.5f;
    B.ax0 = q_rotate(p.qB, mk3(1, 0, 0)); B.ax1 = q_rotate(p.qB, mk3(0, 1, 0)); B.ax2 = q_rotate(p.qB, mk3(0, 0, 1));
    const float3 delta = B.center - A.center;
    ManifoldGPU& outM = d.manifolds[gid];
    outM.colliderPair = u4{ia, ib, 0, 0};
    // shape dispatch (0 box, 1 sphere, 2 torus, 3 capsule, 4 convex hull)
    const uint32_t stA = d.colShapeType[ia] & SHAPE_KIND_MASK, stB = d.colShapeType[ib] & SHAPE_KIND_MASK;
    if (stA >= 2 || stB >= 2) {
        if (!ROUND) return;  // written by the round-shape pass
        if (stA == 4 || stB == 4) narrow_hull(P, d, p, outM, stA, stB);
        else if ((stA == 3 || stB == 3) && stA != 2 && stB != 2) narrow_capsule(P, d, p, outM, stA, stB);
        else narrow_torus(P, d, p, outM, stA, stB);
        return;
    }
    if (ROUND) return;
    const bool sphA = stA == 1, sphB = stB == 1;
    Hit contacts[MAX_CONTACTS];
    int count = 0;
    float3 nrm;

    if (sphA || sphB) {
        const float rA = cshA.x * 0.5f, rB = cshB.x * 0.5f;
        if (sphA && sphB) {
            const float3 dd = A.center - B.center;
            const float dist = len3(dd);
            const float3 nT = dist > 1e-9f ? dd / dist : mk3(0, 0, 1);
            const float dm = detect_margin(nT, vA - vB, P, rA, rB);
            if (dist > rA + rB + dm) { outM.header = u4{ba, bb, 0, 0}; return; }
            nrm = nT;
            contacts[0].xA = A.center - nrm * rA;
            contacts[0].xB = B.center + nrm * rB;
            contacts[0].feature = 0;
            count = 1;
        } else {
            const bool sIsA = sphA;
            const float r = sIsA ? rA : rB;
            const Box& box = sIsA ? B : A;
            const float4 qBox = sIsA ? p.qB : p.qA;
            const float3 sc = sIsA ? A.center : B.center;
            const float3 local = q_rotate(q_conj(qBox), sc - box.center);
            const float3 h = box.half;
            const float3 cl = clamp3(local, -h, h);
            float3 nLocal, qLocal;
            if (cl.x == local.x && cl.y == local.y && cl.z == local.z) {
                const float3 pen = h - abs3(local);
                const int axis = min_axis(pen);
                float3 n = s3(0);
                setcomp(n, axis, comp(local, axis) >= 0.0f ? 1.0f : -1.0f);
                nLocal = n;
                qLocal = local;
                setcomp(qLocal, axis, comp(n, axis) * comp(h, axis));
            } else {
                const float3 dd = local - cl;
                const float dist = len3(dd);
                const float3 nLT = dd / mx(dist, 1e-9f);
                const float3 nWT = q_rotate(qBox, nLT);
                const float3 vS = sIsA ? vA : vB, vBx = sIsA ? vB : vA;
                const float dm = detect_margin(nWT, vS - vBx, P, r, sIsA ? cshB.w : cshA.w);
                if (dist > r + dm) { outM.header = u4{ba, bb, 0, 0}; return; }
                nLocal = nLT;
                qLocal = cl;
            }
            const float3 nW = q_rotate(qBox, nLocal);
            const float3 qW = q_rotate(qBox, qLocal) + box.center;
            const float3 xS = sc - nW * r;
            nrm = sIsA ? nW : -nW;
            contacts[0].xA = sIsA ? xS : qW;
            contacts[0].xB = sIsA ? qW : xS;
            contacts[0].feature = 0;
            count = 1;
        }
        emit_round_manifold(P, d, p, outM, contacts, count, nrm, 0.5f * mx(rA, rB), STICK_SPHERE);
        return;
    }

    // box - box SAT with reference-face clipping or an edge-edge contact
    AxisBest bestFace{0, 0, 0, -3.402823466e38f, s3(0), false};
    AxisBest bestEdge{0, 0, 0, -3.402823466e38f, s3(0), false};
    const float cap = spec_cap(cshA.w, cshB.w, P.collisionMargin);
    bool separated = false;
    for (int i = 0; i < 3 && !separated; i++)
        if (!test_axis(A, B, delta, box_axis(A, i), 0, i, -1, relVel, cap, P, bestFace)) separated = true;
    for (int i = 0; i < 3 && !separated; i++)
        if (!test_axis(A, B, delta, box_axis(B, i), 1, -1, i, relVel, cap, P, bestFace)) separated = true;
    for (int i = 0; i < 3 && !separated; i++)
        for (int j = 0; j < 3 && !separated; j++)
            if (!test_axis(A, B, delta, cross(box_axis(A, i), box_axis(B, j)), 2, i, j, relVel, cap, P, bestEdge))
                separated = true;
    if (separated || !bestFace.valid) { outM.header = u4{ba, bb, 0, 0}; return; }
    AxisBest best = bestFace;
    if (bestEdge.valid && 0.95f * bestEdge.sep > bestFace.sep + 0.01f) best = bestEdge;
    float3 mids[MAX_CONTACTS];
    if (best.type == 2) {
        float3 a0, a1, b0, b1, xA, xB;
        support_edge(A, best.ia, best.n, a0, a1);
        support_edge(B, best.ib, -best.n, b0, b1);
        closest_seg_seg(a0, a1, b0, b1, xA, xB);
        const uint32_t feature = (2u << 24) | ((uint32_t)(best.ia & 0xFF) << 8) | (uint32_t)(best.ib & 0xFF);
        add_contact(contacts, count, mids, xA, xB, feature);
        if (count == 0) add_contact(contacts, count, mids, support(A, best.n), support(B, -best.n), feature);
    } else {
        const bool refIsA = best.type == 0;
        const int refAxis = refIsA ? best.ia : best.ib;
        const Box& ref = refIsA ? A : B;
        const Box& inc = refIsA ? B : A;
        const float3 refOut = refIsA ? best.n : -best.n;
        const float signR = dot(refOut, box_axis(ref, refAxis)) >= 0.0f ? 1.0f : -1.0f;
        const float3 refN = box_axis(ref, refAxis) * signR;
        const float3 refC = ref.center + refN * box_half(ref, refAxis);
        float3 refU, refV;
        float refEU, refEV;
        face_axes(ref, refAxis, refU, refV, refEU, refEV);
        int incAxis = 0;
        float bestD = -3.402823466e38f;
        for (int i = 0; i < 3; i++) {
            const float dd = fabsf(dot(box_axis(inc, i), refN));
            if (dd > bestD) { bestD = dd; incAxis = i; }
        }
        const float signI = dot(box_axis(inc, incAxis), refN) > 0.0f ? -1.0f : 1.0f;
        const float3 incN = box_axis(inc, incAxis) * signI;
        const float3 incC = inc.center + incN * box_half(inc, incAxis);
        float3 incU, incV;
        float incEU, incEV;
        face_axes(inc, incAxis, incU, incV, incEU, incEV);
        float3 p0[NP_MAX_POLY], p1[NP_MAX_POLY];
        p0[0] = incC + incU * incEU + incV * incEV;
        p0[1] = incC - incU * incEU + incV * incEV;
        p0[2] = incC - incU * incEU - incV * incEV;
        p0[3] = incC + incU * incEU - incV * incEV;
        int n = 4;
        n = clip_poly(p0, n, refU, dot(refU, refC) + refEU, p1);
        n = clip_poly(p1, n, -refU, dot(-refU, refC) + refEU, p0);
        n = clip_poly(p0, n, refV, dot(refV, refC) + refEV, p1);
        n = clip_poly(p1, n, -refV, dot(-refV, refC) + refEV, p0);
        uint32_t prefix = (refIsA ? 0u : 1u) << 24;
        prefix |= (uint32_t)(refAxis & 0xFF) << 16;
        prefix |= (uint32_t)(incAxis & 0xFF) << 8;
        const float slop = PLANE_EPS + mx(0.0f, best.sep);
        for (int i = 0; i < n && count < MAX_CONTACTS; i++) {
            const float3 pInc = p0[i];
            const float dd = dot(pInc - refC, refN);
            if (dd > slop) continue;
            const float3 pRef = pInc - refN * dd;
            add_contact(contacts, count, mids, refIsA ? pRef : pInc, refIsA ? pInc : pRef, prefix | (uint32_t)(i & 0xFF));
        }
        if (count == 0) add_contact(contacts, count, mids, support(A, best.n), support(B, -best.n), prefix);
    }
    emit_feature_manifold(P, d, p, outM, contacts, count, -best.n);
}

template <bool ROUND>
__global__ void k_narrowphase(const Params P, const DevPtrs d) {
    const uint32_t n = d.counters->numPairs;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x)
        narrow_one<ROUND>(P, d, g);
}

// Insert this frame's active manifolds (queried by next frame's narrowphase).
__global__ void k_map_insert(const Params P, const DevPtrs d) {
    const uint32_t n = d.counters->numPairs;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        const ManifoldGPU& m = d.manifolds[g];
        if (m.header.z == 0) continue;
        const uint32_t a = m.colliderPair.x, b = m.colliderPair.y;
        uint32_t h = pair_map_hash(a, b, P.mapCapacity);
        for (uint32_t probe = 0; probe < P.mapCapacity; probe++) {
            if (atomicCAS(&d.mapKeyA[h], 0u, a + 1) == 0u) {
                d.mapKeyB[h] = b;
                d.mapVal[h] = g;
                break;
            }
            h = (h + 1) & (P.mapCapacity - 1u);
        }
    }
}

static uint32_t stride_blocks(uint32_t upper, int threads) {
    const uint32_t need = (upper + threads - 1) / threads;
    const uint32_t cap = 148u * 8u;
    return need == 0 ? 1u : (need < cap ? need : cap);
}

void launch_narrowphase(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    k_narrowphase<false><<<stride_blocks(z.maxPairs, 128), 128, 0, st>>>(P, d);
    if (P.roundShapes) k_narrowphase<true><<<stride_blocks(z.maxPairs, 128), 128, 0, st>>>(P, d);
}

void launch_map_rebuild(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    cudaMemsetAsync(d.mapKeyA, 0, sizeof(uint32_t) * P.mapCapacity, st);
    k_map_insert<<<stride_blocks(z.maxPairs, 128), 128, 0, st>>>(P, d);
}

}  // namespace avbd
