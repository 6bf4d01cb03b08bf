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
}  // namespace

__device__ void narrow_one(const Params& P, const DevPtrs& d, uint32_t gid) {
    const uint2 pr = d.pairs[gid];
    const uint32_t ia = pr.x, ib = pr.y;
    const uint32_t ba = d.colOwner[ia], bb = d.colOwner[ib];
    const float4 bodyPA = d.posLin[ba], bodyPB = d.posLin[bb];
    const float4 qBodyA = d.posAng[ba], qBodyB = d.posAng[bb];
    const float3 centerA = xyz(bodyPA) + q_rotate(qBodyA, xyz(d.colLocalPos[ia]));
    const float3 centerB = xyz(bodyPB) + q_rotate(qBodyB, xyz(d.colLocalPos[ib]));
    const float4 qA = q_mul(qBodyA, d.colLocalRot[ia]);
    const float4 qB = q_mul(qBodyB, d.colLocalRot[ib]);
    const float3 vA = xyz(d.velLin[ba]) + cross(xyz(d.velAng[ba]), centerA - xyz(bodyPA));
    const float3 vB = xyz(d.velLin[bb]) + cross(xyz(d.velAng[bb]), centerB - xyz(bodyPB));
    const float3 relVel = vB - vA;
    const float4 cshA = d.colShape[ia], cshB = d.colShape[ib];
    Box A, B;
    A.center = centerA; A.half = xyz(cshA) * 0.5f;
    A.ax0 = q_rotate(qA, mk3(1, 0, 0)); A.ax1 = q_rotate(qA, mk3(0, 1, 0)); A.ax2 = q_rotate(qA, mk3(0, 0, 1));
    B.center = centerB; B.half = xyz(cshB) * 0.5f;
    B.ax0 = q_rotate(qB, mk3(1, 0, 0)); B.ax1 = q_rotate(qB, mk3(0, 1, 0)); B.ax2 = q_rotate(qB, mk3(0, 0, 1));
    const float3 delta = B.center - A.center;
    ManifoldGPU& outM = d.manifolds[gid];
    outM.colliderPair = u4{ia, ib, 0, 0};
    const uint32_t stA = d.colShapeType[ia] & SHAPE_KIND_MASK, stB = d.colShapeType[ib] & SHAPE_KIND_MASK;
    const bool sphA = stA == 1, sphB = stB == 1;
    if (stA >= 2 || stB >= 2) { outM.header = u4{ba, bb, 0, 0}; return; }
    const float warm = P.alpha * P.gamma;
    const float2 frA = d.colFriction[ia], frB = d.colFriction[ib];
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
            const float4 qBox = sIsA ? qB : qA;
            const float3 sc = sIsA ? A.center : B.center;
            const float3 local = q_rotate(q_conj(qBox), sc - box.center);
            const float3 h = box.half;
            const float3 cl = clamp3(local, -h, h);
            float3 nLocal, qLocal;
            if (cl.x == local.x && cl.y == local.y && cl.z == local.z) {
                const float3 pen = h - abs3(local);
                int axis = 0;
                if (pen.y < comp(pen, axis)) axis = 1;
                if (pen.z < comp(pen, axis)) axis = 2;
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
        float3 t1, t2;
        orthonormal(nrm, t1, t2);
        const float sf = combine_friction(frA.x, frB.x, P.frictionCombineMode);
        const float df = combine_friction(frA.y, frB.y, P.frictionCombineMode);
        const int prev = map_find(d, P, ia, ib);
        const bool roundA = (d.colShapeType[ia] & COLLIDER_WORLD_ROUND_ANCHOR) != 0;
        const bool roundB = (d.colShapeType[ib] & COLLIDER_WORLD_ROUND_ANCHOR) != 0;
        outM.header = u4{ba, bb, (uint32_t)count, 1u | (roundA ? 2u : 0u) | (roundB ? 4u : 0u)};
        outM.basisN = tof4(nrm, df);
        outM.basisT1 = tof4(t1, sf);
        const float4 qAc = q_conj(qBodyA), qBc = q_conj(qBodyB);
        for (int i = 0; i < count; i++) {
            float3 rA_ = roundA ? contacts[i].xA - xyz(bodyPA) : q_rotate(qAc, contacts[i].xA - xyz(bodyPA));
            float3 rB_ = roundB ? contacts[i].xB - xyz(bodyPB) : q_rotate(qBc, contacts[i].xB - xyz(bodyPB));
            float3 lambda = s3(0), penalty = s3(0);
            float stick = 0.0f;
            if (prev >= 0) {
                const ManifoldGPU& pm = d.prevManifolds[prev];
                const uint32_t pn = pm.header.z;
                float bestD = 0.5f * mx(rA, rB);
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
                    const bool partA = cshA.w < 0.0f, partB = cshB.w < 0.0f;
                    if ((partA || !roundA) && (partB || !roundB)) {
                        stick = pm.contacts[bestJ].rB.w;
                        if (stick != 0.0f) { rA_ = xyz(pm.contacts[bestJ].rA); rB_ = xyz(pm.contacts[bestJ].rB); }
                    }
                }
            }
            const float3 xAw = roundA ? xyz(bodyPA) + rA_ : xform(xyz(bodyPA), qBodyA, rA_);
            const float3 xBw = roundB ? xyz(bodyPB) + rB_ : xform(xyz(bodyPB), qBodyB, rB_);
            const float3 dd = xAw - xBw;
            float3 C0 = mk3(dot(nrm, dd) + P.collisionMargin, dot(t1, dd), dot(t2, dd));
            float sx, sy;
            spin_shift(d.spinVel[ba], d.spinVel[bb], xAw - xyz(bodyPA), xBw - xyz(bodyPB), t1, t2, P.dt, P.alpha, sx, sy);
            C0.y -= sx;
            C0.z -= sy;
            lambda *= warm;
            penalty = clamp3(penalty * P.gamma, penalty_floor(d, P, ba, bb), mk3(PENALTY_MAX, PENALTY_MAX_T, PENALTY_MAX_T));
            write_contact(outM, i, rA_, contacts[i].feature, rB_, stick, C0, lambda, penalty);
        }
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
    nrm = -best.n;
    float3 t1, t2;
    orthonormal(nrm, t1, t2);
    const float sf = combine_friction(frA.x, frB.x, P.frictionCombineMode);
    const float df = combine_friction(frA.y, frB.y, P.frictionCombineMode);
    const int prev = map_find(d, P, ia, ib);
    outM.header = u4{ba, bb, (uint32_t)count, 1u};
    outM.basisN = tof4(nrm, df);
    outM.basisT1 = tof4(t1, sf);
    const float4 qAc = q_conj(qBodyA), qBc = q_conj(qBodyB);
    for (int i = 0; i < count; i++) {
        float3 rA = q_rotate(qAc, contacts[i].xA - xyz(bodyPA));
        float3 rB = q_rotate(qBc, contacts[i].xB - xyz(bodyPB));
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
        const float3 xAw = xform(xyz(bodyPA), qBodyA, rA);
        const float3 xBw = xform(xyz(bodyPB), qBodyB, rB);
        const float3 dd = xAw - xBw;
        float3 C0 = mk3(dot(nrm, dd) + P.collisionMargin, dot(t1, dd), dot(t2, dd));
        float sx, sy;
        spin_shift(d.spinVel[ba], d.spinVel[bb], xAw - xyz(bodyPA), xBw - xyz(bodyPB), t1, t2, P.dt, P.alpha, sx, sy);
        C0.y -= sx;
        C0.z -= sy;
        lambda *= warm;
        penalty = clamp3(penalty * P.gamma, penalty_floor(d, P, ba, bb), mk3(PENALTY_MAX, PENALTY_MAX_T, PENALTY_MAX_T));
        write_contact(outM, i, rA, contacts[i].feature, rB, stick, C0, lambda, penalty);
    }
}

__global__ void k_narrowphase(const Params P, const DevPtrs d) {
    const uint32_t n = d.counters->numPairs;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x)
        narrow_one(P, d, g);
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
    k_narrowphase<<<stride_blocks(z.maxPairs, 128), 128, 0, st>>>(P, d);
}

void launch_map_rebuild(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    cudaMemsetAsync(d.mapKeyA, 0, sizeof(uint32_t) * P.mapCapacity, st);
    k_map_insert<<<stride_blocks(z.maxPairs, 128), 128, 0, st>>>(P, d);
}

}  // namespace avbd
