// solver.cu — warm start, per-frame adjacency, dynamic coloring, the
// per-color block-descent primal, the augmented-Lagrangian dual, BDF1
// finalize and the constraint-error diagnostic.
//
// Follows Shaders/40_solver.metal: warm start :546-722, adjacency :27-243,
// coloring :250-540, force stamps :741-1152 and :1155-1230, the 8-lane
// primal_particles_split :1544-1684, dual :1729-1906, finalize :2108-2147,
// diag_error :2189-2229.
//
// The primal gives every body of the current color a group of 8 consecutive
// lanes.  Lane l stamps adjacency entries l, l+8, l+16, ... of the body; the
// lanes then sum their 6x6 systems with an xor butterfly (offsets 4, 2, 1)
// and lane 0 solves.  The static part of the adjacency (joints, springs,
// tets) is built once at upload; only contact entries are rebuilt per frame.
#include <utility>

#include "dmath.cuh"
#include "kernels.h"
#include "pdl.cuh"

namespace avbd {

constexpr float FLT_BIG = 3.402823466e38f;

// failure kinds (mirrors AVBD_FAIL_* of include/avbd.h)
constexpr uint32_t AVBD_FAIL_RIGID_PAIR_CAPACITY_ = 2;
constexpr uint32_t AVBD_FAIL_UNRESOLVED_COLORING_ = 5;

__device__ __forceinline__ bool body_dynamic(const DevPtrs& d, uint32_t b) {
    return b != WORLD_BODY && d.posLin[b].w > 0.0f;
}

static uint32_t stride_blocks(uint32_t upper, int threads) {
    const uint32_t need = (upper + threads - 1) / threads;
    const uint32_t cap = 148u * 8u;
    return need == 0 ? 1u : (need < cap ? need : cap);
}

// ---------------------------------------------------------------------------
// Warm start (40_solver.metal:546-722)
// ---------------------------------------------------------------------------
__global__ void k_warmstart_constraints(const Params P, const DevPtrs d, uint32_t nJ, uint32_t nS) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nJ + nS) return;
    if (t >= nJ) {
        SpringGPU& sp = d.springs[d.hardSprings[t - nJ]];
        const uint32_t a = sp.header.x, b = sp.header.y;
        const float3 pA = xform(xyz(d.posLin[a]), d.posAng[a], xyz(sp.rA));
        const float3 pB = xform(xyz(d.posLin[b]), d.posAng[b], xyz(sp.rB));
        sp.dual.z = 0.5f * mx(len3(pA - pB) - sp.rB.w, 0.0f);
        float warm = P.alpha * P.gamma;
        if (P.rodDecayPow > 0.0f) {
            const float3 dd = pA - pB;
            const float3 dPrev = dd - (xyz(d.velLin[a]) - xyz(d.velLin[b])) * P.dt;
            const float dl = len3(dd), dpl = len3(dPrev);
            if (dl > 1e-7f && dpl > 1e-7f) {
                const float ct = clampf(dot(dd / dl, dPrev / dpl), 0.0f, 1.0f);
                warm *= powf(ct, P.rodDecayPow);
            }
        }
        sp.dual.x *= warm;
        sp.dual.y = mn(clampf(sp.dual.y * P.gamma, PENALTY_MIN, PENALTY_MAX), sp.rA.w);
        return;
    }
    JointGPU& j = d.joints[d.activeJoints[t]];
    if (j.header.z != 0) return;
    const uint32_t a = j.header.x, b = j.header.y;
    const float3 pA = a == WORLD_BODY ? xyz(j.rA) : xform(xyz(d.posLin[a]), d.posAng[a], xyz(j.rA));
    const float3 pB = xform(xyz(d.posLin[b]), d.posAng[b], xyz(j.rB));
    const float4 qA = a == WORLD_BODY ? make_float4(0, 0, 0, 1) : d.posAng[a];
    const float4 qB = d.posAng[b];
    const float torqueArm = j.C0Lin.w;
    j.C0Lin = tof4(pA - pB, torqueArm);
    const float3 axis = xyz(j.hingeAxis);
    const float4 restRel = tof(j.restRel);
    float3 c0a;
    if (j.hingeAxis.w != 0.0f) {
        const float3 aB = q_rotate(qB, axis);
        const float3 aA = q_rotate(q_mul(qA, restRel), axis);
        c0a = cross(aA, aB) * torqueArm;
        if (j.dynamics.x > 0.0f) {
            const float twist = twist_angle(q_mul(qA, restRel), qB, axis);
            const float3 omegaA = a == WORLD_BODY ? s3(0) : xyz(d.velAng[a]);
            const float twistRate = dot(xyz(d.velAng[b]) - omegaA, aB);
            j.dynamics.y = twist + P.dt * twistRate;
        }
    } else {
        c0a = q_sub(q_mul(qA, restRel), qB) * torqueArm;
    }
    j.C0Ang = tof4(c0a, j.C0Ang.w);
    if (j.motor.y > 0.0f) {
        j.motor.z = 0.0f;
        j.dynamics.z = 0.0f;
        const uint32_t mode = j.header.w & MOTOR_MODE_MASK;
        if (mode == MOTOR_EXPLICIT || mode == MOTOR_VELOCITY) {
            const float4 qAr = a == WORLD_BODY ? restRel : q_mul(d.posAng[a], restRel);
            const float twist = twist_angle(qAr, qB, axis);
            const float3 axisW = q_rotate(qB, axis);
            const float3 omegaA = a == WORLD_BODY ? s3(0) : xyz(d.velAng[a]);
            const float twistRate = dot(xyz(d.velAng[b]) - omegaA, axisW);
            if (mode == MOTOR_VELOCITY)
                j.dynamics.z = clampf(j.limits.z * (j.motor.x - twistRate), -j.motor.y, j.motor.y);
            else
                j.dynamics.z = clampf(j.motor.w * (j.motor.x - twist) - j.limits.z * twistRate, -j.motor.y, j.motor.y);
        }
    }
    const float warm = P.alpha * P.gamma;
    j.lambdaLin.x *= warm; j.lambdaLin.y *= warm; j.lambdaLin.z *= warm;
    j.lambdaAng.x *= warm; j.lambdaAng.y *= warm; j.lambdaAng.z *= warm;
    float3 pl = clamp3(xyz(j.penaltyLin) * P.gamma, s3(PENALTY_MIN), s3(PENALTY_MAX));
    float3 pa = clamp3(xyz(j.penaltyAng) * P.gamma, s3(PENALTY_MIN), s3(PENALTY_MAX));
    pl = mn3(pl, s3(j.rA.w));
    pa = mn3(pa, s3(j.rB.w));
    j.penaltyLin = tof4(pl, j.penaltyLin.w);
    j.penaltyAng = tof4(pa, j.penaltyAng.w);
}

__global__ void k_warmstart_bodies(const Params P, const DevPtrs d) {
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= P.numBodies) return;
    const float4 pl = d.posLin[gid], pa = d.posAng[gid];
    const float mass = pl.w, dt = P.dt;
    const float3 vl = xyz(d.velLin[gid]), va = xyz(d.velAng[gid]);
    float3 inertial = xyz(pl) + vl * dt;
    const float bodyGravity = P.gravity * d.gravityScale[gid];
    if (mass > 0.0f) inertial += mk3(0, 0, bodyGravity) * (dt * dt);
    d.inertLin[gid] = mk4(inertial, 0.0f);
    d.inertAng[gid] = q_addw(pa, va * dt);
    const float3 accel = (vl - xyz(d.prevVelLin[gid])) / dt;
    const float gsign = P.gravity < 0.0f ? -1.0f : (P.gravity > 0.0f ? 1.0f : 0.0f);
    float w = clampf(accel.z * gsign / fabsf(P.gravity), 0.0f, 1.0f);
    if (!isfinite(w)) w = 0.0f;
    d.initLin[gid] = mk4(xyz(pl), 0.0f);
    d.initAng[gid] = pa;
    // the committed collision-query pose of every surface vertex, pins included
    if ((P.cloth || P.ogc) && P.surfaceTruncationMode != 0u && d.shape[gid].w < 0.0f)
        d.ogcPrev[gid] = mk4(xyz(pl), 0.0f);
    if (mass > 0.0f) {
        float3 guess = xyz(pl) + vl * dt + mk3(0, 0, bodyGravity) * (w * dt * dt);
        // Isotropic OGC: the warm start stays within the particle's bound
        // (40_solver.metal:700-717).  Without element contacts (P.ogc == 0)
        // every bound is "far" and this is a no-op.
        if (P.ogc && d.shape[gid].w < 0.0f) {
            const float d2 = __uint_as_float(d.ogcBounds[gid]);
            if (d2 < 1e37f) {
                const float bv = mx(0.45f * sqrtf(d2), -0.2f * d.shape[gid].w);
                const float3 tot = guess - xyz(pl);
                const float t2 = dot(tot, tot);
                if (t2 > bv * bv) guess = xyz(pl) + tot * (bv * rsq(t2));
            }
        }
        d.posLin[gid] = mk4(guess, mass);
        d.posAng[gid] = q_addw(pa, va * dt);
    }
}

void launch_warmstart(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    const uint32_t n = z.numActiveJoints + z.numHardSprings;
    if (n) k_warmstart_constraints<<<(n + 127) / 128, 128, 0, st>>>(P, d, z.numActiveJoints, z.numHardSprings);
    k_warmstart_bodies<<<(P.numBodies + 127) / 128, 128, 0, st>>>(P, d);
}

// ---------------------------------------------------------------------------
// Per-frame contact adjacency: count, scan, scatter, sort per body.
// ---------------------------------------------------------------------------
// Items: this frame's manifolds, then (cloth scenes) its element contacts.
template <bool SCATTER>
__global__ void k_adj_dyn(const Params P, const DevPtrs d) {
    const uint32_t nm = d.counters->numPairs;
    const uint32_t ns = (P.cloth || P.ogc) ? d.counters->numSoft : 0u;
    auto put = [&](uint32_t b, uint32_t e) {
        if (!body_dynamic(d, b)) return;
        if (SCATTER) d.dynList[atomicAdd(&d.dynCursor[b], 1u)] = e;
        else atomicAdd(&d.dynCount[b], 1u);
    };
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nm + ns; i += gridDim.x * blockDim.x) {
        if (i < nm) {
            const u4 h = d.manifolds[i].header;
            if (h.z == 0) continue;
            const uint32_t e = (FK_MANIFOLD << ADJ_KIND_SHIFT) | i;
            put(h.x, e);
            put(h.y, e);
        } else {
            const uint32_t k = i - nm;
            const u4 ids = d.soft[k].ids;
            const uint32_t e = (FK_SOFT << ADJ_KIND_SHIFT) | k;
            put(ids.x, e);
            put(ids.y, e);
            put(ids.z, e);
            put(ids.w, e);
        }
    }
}
constexpr uint32_t kLongSegment = 2048;   // entries a block sorts in shared memory

__global__ void k_adj_dyn_sort(const DevPtrs d, uint32_t nb) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    uint32_t* l = d.dynList + d.dynStart[b];
    const uint32_t n = d.dynCount[b];
    if (n <= 32) {
        for (uint32_t i = 1; i < n; i++) {
            const uint32_t v = l[i];
            uint32_t j = i;
            while (j > 0 && l[j - 1] > v) { l[j] = l[j - 1]; j--; }
            l[j] = v;
        }
    } else if (n <= kLongSegment) {
        // left to k_adj_long_sort (one block per segment)
        d.dynSplit[b] = 0xFFFFFFFFu;
        d.adjLongQueue[atomicAdd(&d.counters->adjLong, 1u)] = b;
        return;
    } else {
        // heapsort: bodies under a pile (a box on a cloth) carry hundreds of
        // entries; the entries are distinct, so the order is unique
        auto sift = [&](uint32_t root, uint32_t end) {
            while (2 * root + 1 < end) {
                uint32_t c = 2 * root + 1;
                if (c + 1 < end && l[c] < l[c + 1]) c++;
                if (l[root] >= l[c]) return;
                const uint32_t t = l[root]; l[root] = l[c]; l[c] = t;
                root = c;
            }
        };
        for (uint32_t i = n / 2; i-- > 0;) sift(i, n);
        for (uint32_t end = n - 1; end > 0; end--) {
            const uint32_t t = l[0]; l[0] = l[end]; l[end] = t;
            sift(0, end);
        }
    }
    uint32_t m = 0;
    while (m < n && (l[m] >> ADJ_KIND_SHIFT) == FK_MANIFOLD) m++;
    d.dynSplit[b] = m;
}

// Segments of 33..2048 entries: one block loads the segment into shared
// memory, sorts it with a bitonic network (padded with 0xFFFFFFFF), writes
// it back and marks the manifold run.  Entries are distinct, so the result
// equals the serial sort.
__global__ void __launch_bounds__(256) k_adj_long_sort(const DevPtrs d) {
    __shared__ uint32_t buf[kLongSegment];
    const uint32_t count = d.counters->adjLong;
    for (uint32_t q = blockIdx.x; q < count; q += gridDim.x) {
        const uint32_t b = d.adjLongQueue[q];
        uint32_t* l = d.dynList + d.dynStart[b];
        const uint32_t n = d.dynCount[b];
        uint32_t m = 64;
        while (m < n) m <<= 1;
        for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) buf[i] = i < n ? l[i] : 0xFFFFFFFFu;
        __syncthreads();
        for (uint32_t k = 2; k <= m; k <<= 1)
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
                    const uint32_t p = i ^ j;
                    if (p > i) {
                        const uint32_t x = buf[i], y = buf[p];
                        const bool up = (i & k) == 0;
                        if ((x > y) == up) { buf[i] = y; buf[p] = x; }
                    }
                }
                __syncthreads();
            }
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) l[i] = buf[i];
        // manifold entries lead the sorted segment
        uint32_t man = 0;
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) man += (buf[i] >> ADJ_KIND_SHIFT) == FK_MANIFOLD ? 1u : 0u;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) man += __shfl_xor_sync(0xffffffffu, man, o);
        __shared__ uint32_t warpMan[8];
        if ((threadIdx.x & 31u) == 0) warpMan[threadIdx.x >> 5] = man;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t t = 0;
            for (uint32_t w = 0; w < (blockDim.x >> 5); w++) t += warpMan[w];
            d.dynSplit[b] = t;
        }
        __syncthreads();
    }
}

void launch_adjacency(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    cudaMemsetAsync(d.dynCount, 0, sizeof(uint32_t) * P.numBodies, st);
    const uint32_t items = z.maxPairs + ((P.cloth || P.ogc) ? z.maxSoft : 0u);
    k_adj_dyn<false><<<stride_blocks(items, 128), 128, 0, st>>>(P, d);
    launch_exclusive_scan(d.dynCount, d.dynStart, P.numBodies, d.scanScratch, st);
    cudaMemcpyAsync(d.dynCursor, d.dynStart, sizeof(uint32_t) * P.numBodies, cudaMemcpyDeviceToDevice, st);
    k_adj_dyn<true><<<stride_blocks(items, 128), 128, 0, st>>>(P, d);
    k_adj_dyn_sort<<<(P.numBodies + 127) / 128, 128, 0, st>>>(d, P.numBodies);
    k_adj_long_sort<<<148, 256, 0, st>>>(d);
}

// The five runs in ascending (kind << 28 | index) order: static pre
// (joints, springs), this frame's manifolds, static tets, this frame's
// element contacts, static membranes and bends.
struct AdjView {
    const uint32_t* pre; uint32_t nPre;
    const uint32_t* dyn; uint32_t nMan, nDyn;
    const uint32_t* post; uint32_t nTet, nPost, postBase;
    __device__ __forceinline__ uint32_t count() const { return nPre + nDyn + nPost; }
    __device__ __forceinline__ uint32_t at(uint32_t k) const {
        if (k < nPre) return pre[k];
        k -= nPre;
        if (k < nMan) return dyn[k];
        k -= nMan;
        if (k < nTet) return post[k];
        k -= nTet;
        if (k < nDyn - nMan) return dyn[nMan + k];
        return post[nTet + k - (nDyn - nMan)];
    }
};
// The view from the body's static segment (set at upload) and this frame's
// contact segment.
__device__ __forceinline__ AdjView adj_view_from(const DevPtrs& d, uint32_t b, uint4 s, uint32_t nTet) {
    AdjView v;
    v.pre = d.preList + s.x; v.nPre = s.y;
    v.dyn = d.dynList + d.dynStart[b]; v.nDyn = d.dynCount[b]; v.nMan = d.dynSplit[b];
    v.post = d.postList + s.z; v.nPost = s.w; v.nTet = nTet; v.postBase = s.z;
    return v;
}
__device__ __forceinline__ AdjView adj_view(const DevPtrs& d, uint32_t b) {
    const uint4 s = d.staticSeg[b];
    AdjView v;
    v.pre = d.preList + s.x; v.nPre = s.y;
    v.dyn = d.dynList + d.dynStart[b]; v.nDyn = d.dynCount[b]; v.nMan = d.dynSplit[b];
    v.post = d.postList + s.z; v.nPost = s.w; v.nTet = d.postTets[b]; v.postBase = s.z;
    return v;
}

// ---------------------------------------------------------------------------
// Dynamic coloring for rigid-only scenes (40_solver.metal:250-540)
// ---------------------------------------------------------------------------
__device__ void neighbor_colors(const DevPtrs& d, uint32_t entry, uint32_t self, uint32_t myColor,
                                const uint32_t* colorsIn, uint32_t& maskLo, uint32_t& maskHi,
                                uint32_t& allLo, uint32_t& allHi, bool& conflict) {
    const uint32_t kind = entry >> ADJ_KIND_SHIFT, idx = entry & ADJ_INDEX_MASK;
    uint32_t nbs[3];
    uint32_t n = 0;
    if (kind == FK_TET) {
        const u4 ids = d.tets[idx].ids;
        if (ids.x != self && n < 3) nbs[n++] = ids.x;
        if (ids.y != self && n < 3) nbs[n++] = ids.y;
        if (ids.z != self && n < 3) nbs[n++] = ids.z;
        if (ids.w != self && n < 3) nbs[n++] = ids.w;
    } else {
        uint32_t a, b;
        if (kind == FK_JOINT) { a = d.joints[idx].header.x; b = d.joints[idx].header.y; }
        else if (kind == FK_SPRING) { a = d.springs[idx].header.x; b = d.springs[idx].header.y; }
        else { a = d.manifolds[idx].header.x; b = d.manifolds[idx].header.y; }
        nbs[0] = a == self ? b : a;
        n = 1;
    }
    for (uint32_t k = 0; k < n; k++) {
        const uint32_t nb = nbs[k];
        if (nb == WORLD_BODY || d.posLin[nb].w <= 0.0f) continue;
        const uint32_t c = colorsIn[nb];
        const uint32_t lo = c < 32 ? (1u << c) : 0u;
        const uint32_t hi = (c >= 32 && c < 64) ? (1u << (c - 32)) : 0u;
        allLo |= lo; allHi |= hi;
        if (nb < self) { maskLo |= lo; maskHi |= hi; if (c == myColor) conflict = true; }
    }
}

__device__ __forceinline__ void scan_neighbors(const DevPtrs& d, uint32_t b, uint32_t my, const uint32_t* colors,
                                               uint32_t& mLo, uint32_t& mHi, uint32_t& aLo, uint32_t& aHi,
                                               bool& conflict) {
    const AdjView v = adj_view(d, b);
    const uint32_t n = v.count();
    for (uint32_t k = 0; k < n; k++) neighbor_colors(d, v.at(k), b, my, colors, mLo, mHi, aLo, aHi, conflict);
}

__device__ __forceinline__ uint32_t ctz32(uint32_t x) { return (uint32_t)(__ffs((int)x) - 1); }

__global__ void k_color_iterate(const Params P, const DevPtrs d, const uint32_t* src, uint32_t* dst, uint32_t pass) {
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= P.numBodies) return;
    if (pass > 0 && d.counters->changed[pass - 1] == 0u) return;
    if (d.posLin[gid].w <= 0.0f) { dst[gid] = 0; return; }
    const uint32_t my = src[gid];
    uint32_t mLo = 0, mHi = 0, aLo = 0, aHi = 0;
    bool conflict = false;
    scan_neighbors(d, gid, my, src, mLo, mHi, aLo, aHi, conflict);
    if (conflict) {
        const uint32_t freeLo = ~mLo;
        uint32_t nc;
        if (freeLo != 0) nc = ctz32(freeLo);
        else { const uint32_t freeHi = ~mHi; nc = freeHi != 0 ? 32 + ctz32(freeHi) : (MAX_COLORS - 1); }
        dst[gid] = nc < (uint32_t)(MAX_COLORS - 1) ? nc : (uint32_t)(MAX_COLORS - 1);
        atomicOr(&d.counters->changed[pass], 1u);
    } else {
        const uint32_t freeLo = ~aLo;
        const uint32_t best = freeLo != 0 ? ctz32(freeLo) : (~aHi != 0 ? 32 + ctz32(~aHi) : my);
        dst[gid] = best < my ? best : my;
        if (best < my) atomicOr(&d.counters->changed[pass], 1u);
    }
}

// Serial greedy completion when the bounded parallel phase has not settled.
__global__ void k_color_repair(const Params P, const DevPtrs d, uint32_t* colors, uint32_t finalPass) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    if (d.counters->changed[finalPass] == 0u) return;
    for (uint32_t self = 0; self < P.numBodies; self++) {
        if (d.posLin[self].w <= 0.0f) { colors[self] = 0; continue; }
        uint32_t mLo = 0, mHi = 0, aLo = 0, aHi = 0;
        bool conflict = false;
        scan_neighbors(d, self, colors[self], colors, mLo, mHi, aLo, aHi, conflict);
        const uint32_t freeLo = ~mLo;
        if (freeLo != 0) colors[self] = ctz32(freeLo);
        else { const uint32_t freeHi = ~mHi; colors[self] = freeHi != 0 ? 32 + ctz32(freeHi) : (MAX_COLORS - 1); }
    }
}

__global__ void k_color_validate_count(const Params P, const DevPtrs d, const uint32_t* colors) {
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= P.numBodies || d.posLin[gid].w <= 0.0f) return;
    uint32_t mLo = 0, mHi = 0, aLo = 0, aHi = 0;
    bool conflict = false;
    scan_neighbors(d, gid, colors[gid], colors, mLo, mHi, aLo, aHi, conflict);
    if (conflict) atomicAdd(&d.counters->colorConflicts, 1u);
    d.bodySlot[gid] = atomicAdd(&d.counters->colorCount[colors[gid]], 1u);
}

__global__ void k_color_scan(const DevPtrs d) {
    if (threadIdx.x != 0) return;
    uint32_t run = 0, used = 0;
    for (int c = 0; c < MAX_COLORS; c++) {
        d.counters->colorStart[c] = run;
        const uint32_t n = d.counters->colorCount[c];
        run += n;
        if (n > 0) used = c + 1;
    }
    d.counters->colorStart[MAX_COLORS] = run;
    d.counters->colorStart[MAX_COLORS + 1] = used;
    d.counters->usedColors = used;
}

__global__ void k_color_scatter(const Params P, const DevPtrs d, const uint32_t* colors) {
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= P.numBodies || d.posLin[gid].w <= 0.0f) return;
    d.colorList[d.counters->colorStart[colors[gid]] + d.bodySlot[gid]] = gid;
}

void launch_dynamic_coloring(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    const int T = 128;
    const uint32_t blocks = (P.numBodies + T - 1) / T;
    const int passes = 20;
    for (int pass = 0; pass < passes; pass++) {
        const uint32_t* src = (pass & 1) ? d.colorsB : d.colorsA;
        uint32_t* dst = (pass & 1) ? d.colorsA : d.colorsB;
        k_color_iterate<<<blocks, T, 0, st>>>(P, d, src, dst, (uint32_t)pass);
    }
    k_color_repair<<<1, 1, 0, st>>>(P, d, d.colorsA, passes - 1);
    k_color_validate_count<<<blocks, T, 0, st>>>(P, d, d.colorsA);
    k_color_scan<<<1, 32, 0, st>>>(d);
    k_color_scatter<<<blocks, T, 0, st>>>(P, d, d.colorsA);
}

// ---------------------------------------------------------------------------
// Force stamps (40_solver.metal:733-1230)
// ---------------------------------------------------------------------------
struct Accum { M3 lhsLin, lhsAng, lhsCross; float3 rhsLin, rhsAng; };

__device__ __forceinline__ M3 geom_stiff_ball_socket(int k, float3 v) {
    M3 m = m3_diag(s3(-comp(v, k)));
    if (k == 0) { m.r0.x += v.x; m.r1.x += v.y; m.r2.x += v.z; }
    else if (k == 1) { m.r0.y += v.x; m.r1.y += v.y; m.r2.y += v.z; }
    else { m.r0.z += v.x; m.r1.z += v.y; m.r2.z += v.z; }
    return m;
}

__device__ void stamp_joint(const Params& P, const DevPtrs& d, const JointGPU& j, uint32_t self, Accum& acc) {
    const uint32_t a = j.header.x, b = j.header.y;
    const bool isA = self == a;
    const float torqueArm = j.C0Lin.w;
    const float3 penLin = xyz(j.penaltyLin);
    const float4 qBb = d.posAng[b];
    if (dot(penLin, penLin) > 0.0f) {
        const float3 pA = a == WORLD_BODY ? xyz(j.rA) : xform(xyz(d.posLin[a]), d.posAng[a], xyz(j.rA));
        const float3 pB = xform(xyz(d.posLin[b]), qBb, xyz(j.rB));
        float3 C = pA - pB;
        if (j.header.w & 1) C -= xyz(j.C0Lin) * P.alpha;
        const float3 F = penLin * C + xyz(j.lambdaLin);
        const float jsign = isA ? 1.0f : -1.0f;
        const float3 rW = isA ? q_rotate(d.posAng[a], xyz(j.rA)) : q_rotate(qBb, xyz(j.rB));
        const M3 jAng = m3_skew(-jsign * rW);
        const M3 jAngT = m3_transpose(jAng);
        const M3 K = m3_diag(penLin);
        const M3 jAngTk = m3_mulm(jAngT, K);
        acc.lhsLin = m3_add(acc.lhsLin, K);
        acc.lhsAng = m3_add(acc.lhsAng, m3_mulm(jAngTk, jAng));
        acc.lhsCross = m3_add(acc.lhsCross, m3_scale(jAngTk, jsign));
        const float3 r = jsign * rW;
        const M3 H = m3_add(m3_add(m3_scale(geom_stiff_ball_socket(0, r), F.x),
                                   m3_scale(geom_stiff_ball_socket(1, r), F.y)),
                            m3_scale(geom_stiff_ball_socket(2, r), F.z));
        acc.lhsAng = m3_add(acc.lhsAng, m3_diagonalize(H));
        acc.rhsLin += jsign * F;
        acc.rhsAng += m3_mul(jAngT, F);
    }
    const float3 penAng = xyz(j.penaltyAng);
    if (dot(penAng, penAng) > 0.0f) {
        const float4 qA = a == WORLD_BODY ? make_float4(0, 0, 0, 1) : d.posAng[a];
        const float4 restRel = tof(j.restRel);
        float3 C = q_sub(q_mul(qA, restRel), qBb) * torqueArm;
        const float s = (isA ? 1.0f : -1.0f) * torqueArm;
        if (j.hingeAxis.w != 0.0f) {
            const float3 axis = xyz(j.hingeAxis);
            const float3 aB = q_rotate(qBb, axis);
            const float3 aA = q_rotate(q_mul(qA, restRel), axis);
            C = cross(aA, aB) * torqueArm;
            if (j.header.w & 2) C -= xyz(j.C0Ang) * P.alpha;
            const float3 F = penAng * C + xyz(j.lambdaAng);
            const float alignment = dot(aA, aB);
            M3 J = isA ? m3_add(m3_outer(aA, aB), m3_scale(m3_identity(), -alignment))
                       : m3_add(m3_scale(m3_identity(), alignment), m3_scale(m3_outer(aB, aA), -1.0f));
            J = m3_scale(J, torqueArm);
            const M3 JT = m3_transpose(J);
            const M3 K = m3_diag(penAng);
            acc.lhsAng = m3_add(acc.lhsAng, m3_mulm(m3_mulm(JT, K), J));
            acc.rhsAng += m3_mul(JT, F);
            if (j.motor.y > 0.0f || j.limits.x < j.limits.y) {
                const float twist = twist_angle(q_mul(qA, restRel), qBb, axis);
                if (j.dynamics.x > 0.0f) {
                    const float Ca = wrap_pi(twist - j.dynamics.y);
                    const float ka = j.dynamics.x / mx(P.dt * P.dt, 1e-12f);
                    const float sm = (self == a) ? -1.0f : 1.0f;
                    acc.lhsAng = m3_add(acc.lhsAng, m3_scale(m3_outer(aB, aB), ka));
                    acc.rhsAng += aB * (ka * Ca * sm);
                }
                if (j.limits.x < j.limits.y) {
                    const float over = mx(twist - j.limits.y, 0.0f) + mn(twist - j.limits.x, 0.0f);
                    if (over != 0.0f) {
                        const float kL = 4.0e4f;
                        const float FL = clampf(kL * over, -3000.0f, 3000.0f);
                        const float sm = (self == a) ? -1.0f : 1.0f;
                        acc.lhsAng = m3_add(acc.lhsAng, m3_scale(m3_outer(aB, aB), kL));
                        acc.rhsAng += aB * (FL * sm);
                    }
                }
                if (j.motor.y > 0.0f) {
                    const float sm = (self == a) ? -1.0f : 1.0f;
                    const uint32_t mode = j.header.w & MOTOR_MODE_MASK;
                    if (mode == MOTOR_EXPLICIT || mode == MOTOR_VELOCITY) {
                        acc.rhsAng += aB * (-j.dynamics.z * sm);
                    } else {
                        const float Cm = wrap_pi(twist - j.motor.x);
                        const float4 qA0 = a == WORLD_BODY ? make_float4(0, 0, 0, 1) : d.initAng[a];
                        const float twist0 = twist_angle(q_mul(qA0, restRel), d.initAng[b], axis);
                        const float dTwist = wrap_pi(twist - twist0);
                        const float cD = j.limits.z / mx(P.dt, 1e-6f);
                        const float raw = j.motor.w * Cm + cD * dTwist;
                        const float effort = clampf(raw, -j.motor.y, j.motor.y);
                        if (fabsf(raw) < j.motor.y)
                            acc.lhsAng = m3_add(acc.lhsAng, m3_scale(m3_outer(aB, aB), j.motor.w + cD));
                        acc.rhsAng += aB * (effort * sm);
                    }
                }
            }
        } else {
            if (j.header.w & 2) C -= xyz(j.C0Ang) * P.alpha;
            const float3 F = penAng * C + xyz(j.lambdaAng);
            acc.lhsAng = m3_add(acc.lhsAng, m3_diag(penAng * (s * s)));
            acc.rhsAng += F * s;
        }
    }
}

__device__ void stamp_spring(const Params& P, const DevPtrs& d, const SpringGPU& sp, uint32_t self, Accum& acc) {
    const uint32_t a = sp.header.x, b = sp.header.y;
    float stiffness = sp.rA.w;
    const float rest = sp.rB.w;
    const float3 pA = xform(xyz(d.posLin[a]), d.posAng[a], xyz(sp.rA));
    const float3 pB = xform(xyz(d.posLin[b]), d.posAng[b], xyz(sp.rB));
    const float3 dd = pA - pB;
    const float dLen = len3(dd);
    if (dLen <= 1.0e-6f) return;
    const float3 n = dd / dLen;
    float f;
    if (sp.header.z != 0) {
        const float C = dLen - rest - sp.dual.z * P.alpha;
        stiffness = sp.dual.y;
        f = stiffness * C + sp.dual.x;
        if (f <= 0.0f) return;
    } else {
        f = stiffness * (dLen - rest);
    }
    const bool isA = self == a;
    const float3 rW = isA ? q_rotate(d.posAng[a], xyz(sp.rA)) : q_rotate(d.posAng[b], xyz(sp.rB));
    const float3 jLin = isA ? n : -n;
    const float3 jAng = isA ? cross(rW, n) : -cross(rW, n);
    acc.lhsLin = m3_add(acc.lhsLin, m3_scale(m3_outer(jLin, jLin), stiffness));
    acc.lhsAng = m3_add(acc.lhsAng, m3_scale(m3_outer(jAng, jAng), stiffness));
    acc.lhsCross = m3_add(acc.lhsCross, m3_scale(m3_outer(jAng, jLin), stiffness));
    acc.rhsLin += jLin * f;
    acc.rhsAng += jAng * f;
    const float ft = mx(f, 0.0f) / dLen;
    if (ft > 0.0f) acc.lhsLin = m3_add(acc.lhsLin, m3_add(m3_diag(s3(ft)), m3_scale(m3_outer(n, n), -ft)));
}

// Stable Neo-Hookean tet, VBD per-vertex Hessian (40_solver.metal:966-1020).
__device__ void stamp_tet(const DevPtrs& d, const TetGPU& t, uint32_t self, Accum& acc) {
    const float3 x0 = xyz(d.posLin[t.ids.x]), x1 = xyz(d.posLin[t.ids.y]);
    const float3 x2 = xyz(d.posLin[t.ids.z]), x3 = xyz(d.posLin[t.ids.w]);
    const float muV = t.r1.w, lamV = t.r2.w;
    const float alphaT = 1.0f + muV / mx(lamV, 1e-9f);
    const float3 d0 = x1 - x0, d1 = x2 - x0, d2 = x3 - x0;
    const float3 m0 = xyz(t.r0), m1 = xyz(t.r1), m2 = xyz(t.r2);
    const float3 f0 = d0 * m0.x + d1 * m1.x + d2 * m2.x;
    const float3 f1 = d0 * m0.y + d1 * m1.y + d2 * m2.y;
    const float3 f2 = d0 * m0.z + d1 * m1.z + d2 * m2.z;
    const float J = dot(f0, cross(f1, f2));
    const float3 j0 = cross(f1, f2), j1 = cross(f2, f0), j2 = cross(f0, f1);
    const float s2 = lamV * (J - alphaT);
    const float3 p0 = muV * f0 + s2 * j0;
    const float3 p1 = muV * f1 + s2 * j1;
    const float3 p2 = muV * f2 + s2 * j2;
    float3 w;
    if (self == t.ids.y) w = m0;
    else if (self == t.ids.z) w = m1;
    else if (self == t.ids.w) w = m2;
    else w = -mk3(m0.x + m1.x + m2.x, m0.y + m1.y + m2.y, m0.z + m1.z + m2.z);
    const float3 grad = p0 * w.x + p1 * w.y + p2 * w.z;
    const float3 g = j0 * w.x + j1 * w.y + j2 * w.z;
    acc.rhsLin += grad;
    acc.lhsLin = m3_add(acc.lhsLin, m3_diag(s3(muV * dot(w, w))));
    acc.lhsLin = m3_add(acc.lhsLin, m3_scale(m3_outer(g, g), lamV));
}

// Linearised contact constraint and its cone-projected force.
__device__ __forceinline__ float3 contact_force(const ContactGPU& c, float3 nrm, float3 t1, float3 t2,
                                                float dynF, float statF, float alpha,
                                                float3 dqALin, float3 dqAAng, float3 dqBLin, float3 dqBAng,
                                                float3 rAW, float3 rBW, float3& Cout, float& fs, float& bounds) {
    float3 C = xyz(c.C0) * (1.0f - alpha);
    C += mk3(dot(nrm, dqALin), dot(t1, dqALin), dot(t2, dqALin));
    C -= mk3(dot(nrm, dqBLin), dot(t1, dqBLin), dot(t2, dqBLin));
    C += mk3(dot(cross(rAW, nrm), dqAAng), dot(cross(rAW, t1), dqAAng), dot(cross(rAW, t2), dqAAng));
    C -= mk3(dot(cross(rBW, nrm), dqBAng), dot(cross(rBW, t1), dqBAng), dot(cross(rBW, t2), dqBAng));
    float3 F = xyz(c.penalty) * C + xyz(c.lambda);
    F.x = mn(F.x, 0.0f);
    bounds = fabsf(F.x) * statF;
    fs = sqrtf(F.y * F.y + F.z * F.z);
    if (fs > bounds && fs > 0.0f) {
        const float db = fabsf(F.x) * dynF;
        const float sc = db / fs;
        F.y *= sc;
        F.z *= sc;
    }
    Cout = C;
    return F;
}

// What one contact point (or one rigid element-contact slot) adds to a
// body's 6x6 system: each accumulator component takes exactly one add per
// point, so a point's increment can be formed anywhere and added later in
// the original order with the same result.
struct PointInc { M3 lhsLin, lhsAng, lhsCross; float3 rhsLin, rhsAng; };
__device__ __forceinline__ void add_inc(Accum& acc, const PointInc& x) {
    acc.lhsLin = m3_add(acc.lhsLin, x.lhsLin);
    acc.lhsAng = m3_add(acc.lhsAng, x.lhsAng);
    acc.lhsCross = m3_add(acc.lhsCross, x.lhsCross);
    acc.rhsLin += x.rhsLin;
    acc.rhsAng += x.rhsAng;
}
// Jacobian-weighted increment of a contact frame with world lever rW.
__device__ __forceinline__ PointInc point_inc(const M3& jLin, float3 rW, const M3& K, float3 F) {
    const M3 jAng = M3{cross(rW, jLin.r0), cross(rW, jLin.r1), cross(rW, jLin.r2)};
    const M3 jLinT = m3_transpose(jLin), jAngT = m3_transpose(jAng);
    const M3 jAngTk = m3_mulm(jAngT, K);
    PointInc x;
    x.lhsLin = m3_mulm(m3_mulm(jLinT, K), jLin);
    x.lhsAng = m3_mulm(jAngTk, jAng);
    x.lhsCross = m3_mulm(jAngTk, jLin);
    x.rhsLin = m3_mul(jLinT, F);
    x.rhsAng = m3_mul(jAngT, F);
    return x;
}

// Pose data of a manifold's two bodies shared by its contact points.
struct ManifoldCtx {
    float4 qa, qb;
    float3 dqALin, dqAAng, dqBLin, dqBAng, nrm, t1, t2;
    float dynF, statF;
    bool isA, sphA, sphB;
};
__device__ __forceinline__ ManifoldCtx manifold_ctx(const DevPtrs& d, const ManifoldGPU& m, uint32_t self) {
    const u4 h = m.header;
    const uint32_t a = h.x, b = h.y;
    ManifoldCtx x;
    x.isA = self == a;
    x.sphA = (h.w & 2u) != 0;
    x.sphB = (h.w & 4u) != 0;
    x.qa = d.posAng[a];
    x.qb = d.posAng[b];
    x.dqALin = xyz(d.posLin[a]) - xyz(d.initLin[a]);
    x.dqAAng = q_sub(x.qa, d.initAng[a]);
    x.dqBLin = xyz(d.posLin[b]) - xyz(d.initLin[b]);
    x.dqBAng = q_sub(x.qb, d.initAng[b]);
    x.nrm = xyz(m.basisN);
    x.t1 = xyz(m.basisT1);
    x.t2 = cross(x.nrm, x.t1);
    x.dynF = m.basisN.w;
    x.statF = m.basisT1.w;
    return x;
}
// Increment of contact point i of a manifold.
__device__ __forceinline__ PointInc manifold_point_inc(const Params& P, const ManifoldCtx& x, const ContactGPU& c) {
    const float3 rAW = x.sphA ? xyz(c.rA) : q_rotate(x.qa, xyz(c.rA));
    const float3 rBW = x.sphB ? xyz(c.rB) : q_rotate(x.qb, xyz(c.rB));
    float3 C;
    float fs, bnd;
    const float3 F = contact_force(c, x.nrm, x.t1, x.t2, x.dynF, x.statF, P.alpha, x.dqALin, x.dqAAng, x.dqBLin,
                                   x.dqBAng, rAW, rBW, C, fs, bnd);
    const float s = x.isA ? 1.0f : -1.0f;
    const M3 jLin = M3{x.nrm * s, x.t1 * s, x.t2 * s};
    return point_inc(jLin, x.isA ? rAW : rBW, m3_diag(xyz(c.penalty)), F);
}

__device__ void stamp_manifold(const Params& P, const DevPtrs& d, const ManifoldGPU& m, uint32_t self, Accum& acc) {
    const uint32_t n = m.header.z;
    const ManifoldCtx x = manifold_ctx(d, m, self);
    for (uint32_t i = 0; i < n; i++) add_inc(acc, manifold_point_inc(P, x, m.contacts[i]));
}

// StVK membrane, Gauss-Newton Hessian (40_solver.metal:1088-1134).
__device__ void stamp_membrane(const DevPtrs& d, const MembraneGPU& mb, uint32_t self, Accum& acc) {
    const float3 x0 = xyz(d.posLin[mb.ids.x]), x1 = xyz(d.posLin[mb.ids.y]), x2 = xyz(d.posLin[mb.ids.z]);
    const float muA = mb.mat.x, lamA = mb.mat.y;
    const float3 d0 = x1 - x0, d1 = x2 - x0;
    const float a = mb.dm.x, b = mb.dm.y, c = mb.dm.z, dd = mb.dm.w;
    const float3 f1 = d0 * a + d1 * b;
    const float3 f2 = d0 * c + d1 * dd;
    const float E11 = 0.5f * (dot(f1, f1) - 1.0f);
    const float E22 = 0.5f * (dot(f2, f2) - 1.0f);
    const float E12 = 0.5f * dot(f1, f2);
    const float trE = E11 + E22;
    const float S11 = 2.0f * muA * E11 + lamA * trE;
    const float S22 = 2.0f * muA * E22 + lamA * trE;
    const float S12 = 2.0f * muA * E12;
    const float3 p1 = f1 * S11 + f2 * S12;
    const float3 p2 = f1 * S12 + f2 * S22;
    float wx, wy;
    if (self == mb.ids.y) { wx = a; wy = c; }
    else if (self == mb.ids.z) { wx = b; wy = dd; }
    else { wx = -a - b; wy = -c - dd; }
    acc.rhsLin += p1 * wx + p2 * wy;
    const float3 g11 = f1 * wx, g22 = f2 * wy;
    const float3 g12 = (f2 * wx + f1 * wy) * 0.5f;
    const float3 gtr = g11 + g22;
    acc.lhsLin = m3_add(acc.lhsLin, m3_scale(m3_outer(g11, g11), 2.0f * muA));
    acc.lhsLin = m3_add(acc.lhsLin, m3_scale(m3_outer(g22, g22), 2.0f * muA));
    acc.lhsLin = m3_add(acc.lhsLin, m3_scale(m3_outer(g12, g12), 4.0f * muA));
    acc.lhsLin = m3_add(acc.lhsLin, m3_scale(m3_outer(gtr, gtr), lamA));
}

// Quadratic (Bergou) bending, rank-1 isotropic Hessian (40_solver.metal:1136-1153).
__device__ void stamp_bend(const DevPtrs& d, const BendGPU& bd, uint32_t self, Accum& acc) {
    const float sc = bd.mat.x;
    const float3 m = xyz(d.posLin[bd.ids.x]) * bd.K.x + xyz(d.posLin[bd.ids.y]) * bd.K.y +
                     xyz(d.posLin[bd.ids.z]) * bd.K.z + xyz(d.posLin[bd.ids.w]) * bd.K.w;
    float k;
    if (self == bd.ids.x) k = bd.K.x;
    else if (self == bd.ids.y) k = bd.K.y;
    else if (self == bd.ids.z) k = bd.K.z;
    else k = bd.K.w;
    acc.rhsLin += m * (sc * k);
    acc.lhsLin = m3_add(acc.lhsLin, m3_diag(s3(sc * k * k)));
}

// Element-contact constraint over the 4-slot stencil (40_solver.metal:1236-1263).
__device__ float3 soft_c(const Params& P, const DevPtrs& d, const SoftContactGPU& sc, float3& n, float3& t1,
                         float3& t2, float3& rAW, bool& rigidA) {
    const uint32_t flags = __float_as_uint(sc.anchorA.w);
    rigidA = (flags & SCF_RIGID_A) != 0;
    const bool roundA = (flags & SCF_ROUND_A) != 0;
    n = xyz(sc.normal);
    orthonormal(n, t1, t2);
    rAW = s3(0);
    float3 C = xyz(sc.C0) * (1.0f - P.alpha);
    const uint32_t ids[4] = {sc.ids.x, sc.ids.y, sc.ids.z, sc.ids.w};
    const float ws[4] = {sc.weights.x, sc.weights.y, sc.weights.z, sc.weights.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const uint32_t b = ids[k];
        if (b == WORLD_BODY) continue;
        const float w = ws[k];
        const float3 dq = xyz(d.posLin[b]) - xyz(d.initLin[b]);
        C += mk3(dot(n, dq), dot(t1, dq), dot(t2, dq)) * w;
        if (k == 0 && rigidA) {
            const float4 q = d.posAng[b];
            rAW = roundA ? xyz(sc.anchorA) : q_rotate(q, xyz(sc.anchorA));
            const float3 dqa = q_sub(q, d.initAng[b]);
            C += mk3(dot(cross(rAW, n), dqa), dot(cross(rAW, t1), dqa), dot(cross(rAW, t2), dqa)) * w;
        }
    }
    return C;
}

// softContactForce with the two-stage barrier (40_solver.metal:1265-1359):
// the force, the normal stiffness and the frame of an element contact, and
// which of its four slots `self` is (-1: none) with that slot's weight.
struct SoftForce { float3 n, t1, t2, rAW, F; float kN, w; int slot; bool rigidA; };
__device__ __forceinline__ SoftForce soft_force(const Params& P, const DevPtrs& d, const SoftContactGPU& sc,
                                                uint32_t self) {
    SoftForce r;
    const float3 C = soft_c(P, d, sc, r.n, r.t1, r.t2, r.rAW, r.rigidA);
    float3 F = xyz(sc.penalty) * C + xyz(sc.lambda);
    float kN = sc.penalty.x;
    const float rT = sc.anchorA.x;
    const uint32_t kindB = (__float_as_uint(sc.anchorA.w) >> SCF_KIND_SHIFT) & 3u;
    if (rT > 0.0f && kindB != SC_RT && C.x < -0.5f * rT) {
        const float dsep = mx(C.x + rT, 0.02f * rT);
        const float kp = 0.25f * rT * rT * sc.penalty.x;
        F.x = -kp / dsep + sc.lambda.x;
        kN = kp / (dsep * dsep);
    }
    F.x = mn(F.x, 0.0f);
    const float bounds = fabsf(F.x) * sc.normal.w;
    const float fs = sqrtf(F.y * F.y + F.z * F.z);
    if (fs > bounds && fs > 0.0f) {
        const float q = bounds / fs;
        F.y *= q;
        F.z *= q;
    }
    r.F = F;
    r.kN = kN;
    r.slot = -1;
    if (sc.ids.x == self) r.slot = 0;
    else if (sc.ids.y == self) r.slot = 1;
    else if (sc.ids.z == self) r.slot = 2;
    else if (sc.ids.w == self) r.slot = 3;
    r.w = r.slot == 0 ? sc.weights.x : (r.slot == 1 ? sc.weights.y : (r.slot == 2 ? sc.weights.z : sc.weights.w));
    return r;
}
// Increment of the rigid slot 0 of an element contact (stampSoft's 6-DOF branch).
__device__ __forceinline__ PointInc soft_rigid_inc(const SoftContactGPU& sc, const SoftForce& f) {
    const float w = f.w;
    return point_inc(M3{f.n * w, f.t1 * w, f.t2 * w}, f.rAW, m3_diag(mk3(f.kN, sc.penalty.y, sc.penalty.z)), f.F);
}

// stampSoft (40_solver.metal:1265-1359).
__device__ void stamp_soft(const Params& P, const DevPtrs& d, const SoftContactGPU& sc, uint32_t self, Accum& acc) {
    const SoftForce f = soft_force(P, d, sc, self);
    if (f.slot < 0) return;
    if (f.slot == 0 && f.rigidA) {
        add_inc(acc, soft_rigid_inc(sc, f));
    } else {
        const float w2 = f.w * f.w;
        acc.lhsLin = m3_add(acc.lhsLin, m3_scale(m3_outer(f.n, f.n), f.kN * w2));
        acc.lhsLin = m3_add(acc.lhsLin, m3_scale(m3_outer(f.t1, f.t1), sc.penalty.y * w2));
        acc.lhsLin = m3_add(acc.lhsLin, m3_scale(m3_outer(f.t2, f.t2), sc.penalty.z * w2));
        acc.rhsLin += (f.n * f.F.x + f.t1 * f.F.y + f.t2 * f.F.z) * f.w;
    }
}

__device__ __forceinline__ void stamp_entry(const Params& P, const DevPtrs& d, uint32_t entry, uint32_t body,
                                            Accum& acc) {
    const uint32_t kind = entry >> ADJ_KIND_SHIFT, idx = entry & ADJ_INDEX_MASK;
    if (kind == FK_TET) stamp_tet(d, d.tets[idx], body, acc);
    else if (kind == FK_MANIFOLD) stamp_manifold(P, d, d.manifolds[idx], body, acc);
    else if (kind == FK_JOINT) stamp_joint(P, d, d.joints[idx], body, acc);
    else if (kind == FK_SPRING) stamp_spring(P, d, d.springs[idx], body, acc);
    else if (kind == FK_SOFT) stamp_soft(P, d, d.soft[idx], body, acc);
    else if (kind == FK_MEMBRANE) stamp_membrane(d, d.membranes[idx], body, acc);
    else if (kind == FK_BEND) stamp_bend(d, d.bends[idx], body, acc);
}

__device__ __forceinline__ float3 shfl3(unsigned mask, float3 v, int o) {
    return mk3(__shfl_xor_sync(mask, v.x, o, 8), __shfl_xor_sync(mask, v.y, o, 8), __shfl_xor_sync(mask, v.z, o, 8));
}
__device__ __forceinline__ void add_shfl3(unsigned mask, float3& v, int o) { v = v + shfl3(mask, v, o); }

// Isotropic-OGC conservative-bound truncation (ogcTruncate,
// 40_solver.metal:1361-1382): the displacement since the bound's anchor stays
// within max(0.45 * bound distance, 0.2 * radius); every clamped step is
// counted for the mid-solve refresh.
__device__ __forceinline__ float3 ogc_truncate(const DevPtrs& d, uint32_t body, float3 dxLin, float3 cur, float partR) {
    const float d2 = __uint_as_float(d.ogcBounds[body]);
    if (d2 >= 1e37f) return dxLin;
    const float bv = mx(0.45f * sqrtf(d2), 0.2f * partR);
    const float3 x0 = xyz(d.ogcPrev[body]);
    float3 tot = (cur + dxLin) - x0;
    const float t2 = dot(tot, tot);
    if (t2 > bv * bv) {
        tot *= bv * rsq(t2);
        dxLin = (x0 + tot) - cur;
        atomicAdd(d.ogcExceed, 1u);
    }
    return dxLin;
}

// A skipped update (non-finite step) still publishes the unchanged pose
// when the color commits through posNext.
__device__ __forceinline__ void keep_body(const Params& P, const DevPtrs& d, uint32_t body, float4 pl, bool rigid) {
    if (!P.colorJacobi) return;
    d.posNext[body] = pl;
    if (rigid) d.angNext[body] = d.posAng[body];
}

// The 8 lanes' partial systems of one body (lane l stamped entries l,
// l + 8, ...) folded by an xor butterfly; lane 0 solves and writes.
__device__ __forceinline__ void body_commit(const Params& P, const DevPtrs& d, uint32_t body, float4 shp,
                                            uint32_t lane, unsigned mask, Accum acc) {
    const bool rigid = shp.w >= 0.0f;
#pragma unroll
    for (int o = 4; o >= 1; o >>= 1) {
        add_shfl3(mask, acc.lhsLin.r0, o);
        add_shfl3(mask, acc.lhsLin.r1, o);
        add_shfl3(mask, acc.lhsLin.r2, o);
        add_shfl3(mask, acc.rhsLin, o);
        if (rigid) {
            add_shfl3(mask, acc.lhsAng.r0, o);
            add_shfl3(mask, acc.lhsAng.r1, o);
            add_shfl3(mask, acc.lhsAng.r2, o);
            add_shfl3(mask, acc.lhsCross.r0, o);
            add_shfl3(mask, acc.lhsCross.r1, o);
            add_shfl3(mask, acc.lhsCross.r2, o);
            add_shfl3(mask, acc.rhsAng, o);
        }
    }
    if (lane != 0) return;
    const float4 pl = d.posLin[body];
    const float mass = pl.w;
    const float dt2 = P.dt * P.dt;
    acc.lhsLin = m3_add(acc.lhsLin, m3_diag(s3(mass / dt2)));
    acc.rhsLin += (xyz(pl) - xyz(d.inertLin[body])) * (mass / dt2);
    float3 dxLin = s3(0), dxAng = s3(0);
    if (rigid) {
        const float4 q = d.posAng[body];
        const M3 inertia = m3_scale(world_inertia(q, xyz(d.props[body])), 1.0f / dt2);
        acc.lhsAng = m3_add(acc.lhsAng, inertia);
        acc.rhsAng += m3_mul(inertia, q_sub(q, d.inertAng[body]));
        solve6x6(acc.lhsLin, acc.lhsAng, acc.lhsCross, -acc.rhsLin, -acc.rhsAng, dxLin, dxAng);
        if (!finite3(dxLin) || !finite3(dxAng)) { keep_body(P, d, body, pl, rigid); return; }
        const float ang2 = dot(dxAng, dxAng);
        const float maxAng = 0.5f;
        if (ang2 > maxAng * maxAng) dxAng *= maxAng * rsq(ang2);
    } else {
        solve6x6(acc.lhsLin, m3_identity(), m3_zero(), -acc.rhsLin, s3(0), dxLin, dxAng);
        if (!finite3(dxLin)) { keep_body(P, d, body, pl, rigid); return; }
    }
    const float maxLin = 0.35f * fabsf(shp.w);
    const float lin2 = dot(dxLin, dxLin);
    if (lin2 > maxLin * maxLin) dxLin *= maxLin * rsq(lin2);
    if (!rigid && P.ogc) dxLin = ogc_truncate(d, body, dxLin, xyz(pl), -shp.w);
    if (P.colorJacobi) {
        d.posNext[body] = mk4(xyz(pl) + dxLin, mass);
        if (rigid) d.angNext[body] = q_addw(d.posAng[body], dxAng);
        return;
    }
    d.posLin[body] = mk4(xyz(pl) + dxLin, mass);
    if (rigid) d.posAng[body] = q_addw(d.posAng[body], dxAng);
}

// One body on an 8-lane group; lane 0 writes the result.
__device__ void primal_body(const Params& P, const DevPtrs& d, uint32_t body, uint32_t lane, unsigned mask) {
    const float4 shp = d.shape[body];
    Accum acc{m3_zero(), m3_zero(), m3_zero(), s3(0), s3(0)};
    const AdjView v = adj_view(d, body);
    const uint32_t cnt = v.count();
    for (uint32_t k = lane; k < cnt; k += 8) stamp_entry(P, d, v.at(k), body, acc);
    body_commit(P, d, body, shp, lane, mask, acc);
}

__global__ void k_primal(const Params P, const DevPtrs d, uint32_t color, uint32_t count) {
    pdl_prologue();
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t lane = tid & 7u, groups = (gridDim.x * blockDim.x) >> 3;
    const uint32_t s = d.colorStart[color];
    const uint32_t n = count != 0xFFFFFFFFu ? count : d.colorStart[color + 1] - s;
    const unsigned mask = 0xFFu << (threadIdx.x & 24u);
    // one 8-lane group per body, striding over the color (uniform across
    // the group)
    for (uint32_t slot = tid >> 3; slot < n; slot += groups) primal_body(P, d, d.colorList[s + slot], lane, mask);
}

// ---------------------------------------------------------------------------
// Wide primal: one block per body, for a static color's non-lean bodies
// (rigid bodies and particles with joints).  A rigid body under a pile of
// particles carries hundreds of contact entries; on an 8-lane group its
// lanes would stamp them one after another while the rest of the color has
// long finished.  Here the block evaluates the contact points of every
// manifold entry and every rigid element-contact slot at once into shared
// memory, then 8 lanes add them in the 8-lane order (lane l: entries l,
// l + 8, ...; each entry's points in order) — every accumulator component
// takes one add per point, so the sums are those of the sequential stamps.
// Other entries, and points past the staging capacity, are stamped inline
// by the folding lanes in the same order.
// ---------------------------------------------------------------------------
constexpr int kWideThreads = 128;
constexpr int kWideEntries = 512;          // entries whose points may be staged
constexpr int kWidePoints = 320;           // staged points (33 floats each)
constexpr uint32_t kWideInline = 0xFFFFFFFFu;

__global__ void __launch_bounds__(kWideThreads) k_primal_wide(const Params P, const DevPtrs d, uint32_t color,
                                                             uint32_t first, uint32_t start) {
    __shared__ PointInc pts[kWidePoints];
    __shared__ uint32_t entOff[kWideEntries];  // (first point << 8) | points, or kWideInline
    __shared__ uint32_t warpSums[kWideThreads / 32];
    pdl_trigger();
    const uint32_t tid = threadIdx.x, lane32 = tid & 31u, warp = tid >> 5;
    // with the start known on the host, the static data (launch order,
    // shape, static segment) is read before waiting for the previous grid
    if (start == NO_HOST_START) pdl_wait();
    const uint32_t body = d.colorLaunch[(start == NO_HOST_START ? d.colorStart[color] : start) + first + blockIdx.x];
    const float4 shp = d.shape[body];
    const uint4 seg = d.staticSeg[body];
    const uint32_t nTet = d.postTets[body];
    if (start != NO_HOST_START) pdl_wait();
    const AdjView v = adj_view_from(d, body, seg, nTet);
    const uint32_t cnt = v.count();
    const uint32_t staged = min(cnt, (uint32_t)kWideEntries);
    uint32_t base = 0;                          // points taken by earlier chunks
    for (uint32_t c0 = 0; c0 < staged; c0 += kWideThreads) {
        const uint32_t k = c0 + tid;
        uint32_t entry = 0, np = 0;
        if (k < staged) {
            entry = v.at(k);
            const uint32_t kind = entry >> ADJ_KIND_SHIFT, idx = entry & ADJ_INDEX_MASK;
            if (kind == FK_MANIFOLD) {
                np = d.manifolds[idx].header.z;
            } else if (kind == FK_SOFT) {
                const SoftContactGPU& sc = d.soft[idx];
                const bool rigidA = (__float_as_uint(sc.anchorA.w) & SCF_RIGID_A) != 0;
                np = (rigidA && sc.ids.x == body) ? 1u : 0u;
            }
        }
        // exclusive scan of the chunk's point counts
        uint32_t incl = np;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if ((int)lane32 >= o) incl += y;
        }
        if (lane32 == 31) warpSums[warp] = incl;
        __syncthreads();
        uint32_t before = base, total = 0;
#pragma unroll
        for (int w = 0; w < kWideThreads / 32; w++) {
            const uint32_t ws = warpSums[w];
            if (w < (int)warp) before += ws;
            total += ws;
        }
        const uint32_t off = before + incl - np;
        const bool fits = np > 0 && off + np <= (uint32_t)kWidePoints;
        if (k < staged) entOff[k] = fits ? ((off << 8) | np) : kWideInline;
        if (fits) {
            const uint32_t kind = entry >> ADJ_KIND_SHIFT, idx = entry & ADJ_INDEX_MASK;
            if (kind == FK_MANIFOLD) {
                const ManifoldGPU& m = d.manifolds[idx];
                const ManifoldCtx x = manifold_ctx(d, m, body);
                for (uint32_t i = 0; i < np; i++) pts[off + i] = manifold_point_inc(P, x, m.contacts[i]);
            } else {
                const SoftContactGPU& sc = d.soft[idx];
                pts[off] = soft_rigid_inc(sc, soft_force(P, d, sc, body));
            }
        }
        base += total;
        __syncthreads();                        // warpSums is reused by the next chunk
    }
    if (tid >= 8) return;
    Accum acc{m3_zero(), m3_zero(), m3_zero(), s3(0), s3(0)};
    for (uint32_t k = tid; k < cnt; k += 8) {
        const uint32_t eo = k < (uint32_t)kWideEntries ? entOff[k] : kWideInline;
        if (eo != kWideInline) {
            const uint32_t off = eo >> 8, np = eo & 0xFFu;
            for (uint32_t i = 0; i < np; i++) add_inc(acc, pts[off + i]);
        } else {
            stamp_entry(P, d, v.at(k), body, acc);
        }
    }
    body_commit(P, d, body, shp, tid, 0xFFu, acc);
}

void launch_primal_wide(const Params& P, const DevPtrs& d, uint32_t color, uint32_t count, uint32_t first,
                        uint32_t start, cudaStream_t st) {
    if (count) launch_pdl(k_primal_wide, count, kWideThreads, st, P, d, color, first, start);
}

// ---------------------------------------------------------------------------
// Residual of the augmented-Lagrangian objective: the primal right-hand side
// of every dynamic body (inertia + every stamped force) at the current pose,
// squared and summed.  The square root is r_k of the iterations-to-tolerance
// measurement.  Bodies come from the color lists (every dynamic body once).
// ---------------------------------------------------------------------------
// Squared AL gradient of one rigid body (linear and angular parts) by an
// 8-lane group: lanes stamp entries lane, lane + 8, ..., an xor butterfly
// folds them and lane 0 writes *out.
__device__ void rigid_residual(const Params& P, const DevPtrs& d, uint32_t body, uint32_t lane, unsigned mask,
                               float* out) {
    Accum acc{m3_zero(), m3_zero(), m3_zero(), s3(0), s3(0)};
    const AdjView v = adj_view(d, body);
    const uint32_t cnt = v.count();
    for (uint32_t k = lane; k < cnt; k += 8) stamp_entry(P, d, v.at(k), body, acc);
#pragma unroll
    for (int o = 4; o >= 1; o >>= 1) {
        add_shfl3(mask, acc.rhsLin, o);
        add_shfl3(mask, acc.rhsAng, o);
    }
    if (lane != 0) return;
    const float4 pl = d.posLin[body];
    const float dt2 = P.dt * P.dt;
    const float3 rl = acc.rhsLin + (xyz(pl) - xyz(d.inertLin[body])) * (pl.w / dt2);
    const float4 q = d.posAng[body];
    const M3 inertia = m3_scale(world_inertia(q, xyz(d.props[body])), 1.0f / dt2);
    const float3 ra = acc.rhsAng + m3_mul(inertia, q_sub(q, d.inertAng[body]));
    *out = dot(rl, rl) + dot(ra, ra);
}

// Fixed-order sum of n values in one block (double accumulation): thread t
// sums the float4 groups t, t + 1024, ... (16-byte coalesced loads; v is a
// device allocation, so 16-byte aligned), then tail element 4 * (n / 4) + t;
// a warp shuffle tree and a second tree over the warps combine the threads,
// always in the same order.
__global__ void __launch_bounds__(1024) k_sum_fixed(const float* v, uint32_t n, double* out) {
    __shared__ double part[32];
    const uint32_t t = threadIdx.x, n4 = n / 4u;
    const float4* v4 = reinterpret_cast<const float4*>(v);
    double s = 0.0;
    for (uint32_t i = t; i < n4; i += blockDim.x) {
        const float4 q = v4[i];
        s += (double)q.x;
        s += (double)q.y;
        s += (double)q.z;
        s += (double)q.w;
    }
    if (4u * n4 + t < n) s += (double)v[4u * n4 + t];
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((t & 31u) == 0) part[t >> 5] = s;
    __syncthreads();
    if (t < 32) {
        s = t < (blockDim.x >> 5) ? part[t] : 0.0;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (t == 0) *out = s;
    }
}


// ---------------------------------------------------------------------------
// Warp-per-body primal for particles.  The 8-lane kernel above makes each
// lane walk 2-3 tets as chains of dependent loads.  Here all 32 lanes of a
// warp evaluate the force terms of 32 adjacency entries at once, and lanes
// 0-7 then fold them in the 8-lane order — logical lane l takes entries
// l, l+8, l+16, l+24 — applying exactly the additions the stamp would have
// made, so every float is unchanged.  Entries whose terms do not fit the
// shipped record (joints, multi-contact manifolds) are stamped by the
// logical lane itself during the fold.
// ---------------------------------------------------------------------------
enum : uint32_t {
    TERM_NONE = 0, TERM_TET = 1, TERM_MANIFOLD = 2, TERM_SERIAL = 3, TERM_SPRING = 4, TERM_MEMBRANE = 5,
    TERM_BEND = 6, TERM_SOFT = 7
};
struct ParticleTerms {
    float3 rhs;          // the stamp's right-hand-side contribution
    float3 a, b, c, e;   // tet: (G00, G11, G22), (G01, G02, G12), (dd, -, -); manifold: rows of J^T K J;
                         // spring: n; membrane: g11, g22, g12, gtr; soft: n, t1, t2
    float3 s;            // spring: (k, ft, -); membrane: (2 mu A, 4 mu A, lambda A); bend: (s k^2, -, -);
                         // soft: (kN w^2, kT1 w^2, kT2 w^2)
    uint32_t kind;       // TERM_*
};

// Stable Neo-Hookean tet terms of vertex `self` (stampTet, 40_solver.metal:972-1024)
__device__ __forceinline__ void tet_terms(const DevPtrs& d, const TetGPU& tt, uint32_t self, ParticleTerms& t) {
    const float3 x0 = xyz(d.posLin[tt.ids.x]), x1 = xyz(d.posLin[tt.ids.y]);
    const float3 x2 = xyz(d.posLin[tt.ids.z]), x3 = xyz(d.posLin[tt.ids.w]);
    const float muV = tt.r1.w, lamV = tt.r2.w;
    const float alphaT = 1.0f + muV / mx(lamV, 1e-9f);
    const float3 d0 = x1 - x0, d1 = x2 - x0, d2 = x3 - x0;
    const float3 m0 = xyz(tt.r0), m1 = xyz(tt.r1), m2 = xyz(tt.r2);
    const float3 f0 = d0 * m0.x + d1 * m1.x + d2 * m2.x;
    const float3 f1 = d0 * m0.y + d1 * m1.y + d2 * m2.y;
    const float3 f2 = d0 * m0.z + d1 * m1.z + d2 * m2.z;
    const float J = dot(f0, cross(f1, f2));
    const float3 j0 = cross(f1, f2), j1 = cross(f2, f0), j2 = cross(f0, f1);
    const float s2 = lamV * (J - alphaT);
    const float3 p0 = muV * f0 + s2 * j0;
    const float3 p1 = muV * f1 + s2 * j1;
    const float3 p2 = muV * f2 + s2 * j2;
    float3 w;
    if (self == tt.ids.y) w = m0;
    else if (self == tt.ids.z) w = m1;
    else if (self == tt.ids.w) w = m2;
    else w = -mk3(m0.x + m1.x + m2.x, m0.y + m1.y + m2.y, m0.z + m1.z + m2.z);
    t.rhs = p0 * w.x + p1 * w.y + p2 * w.z;
    const float3 g = j0 * w.x + j1 * w.y + j2 * w.z;
    // lamV * outer(g, g) is exactly symmetric: g_i g_j == g_j g_i
    t.a = mk3((g.x * g.x) * lamV, (g.y * g.y) * lamV, (g.z * g.z) * lamV);
    t.b = mk3((g.y * g.x) * lamV, (g.z * g.x) * lamV, (g.z * g.y) * lamV);
    t.c = mk3(muV * dot(w, w), 0.0f, 0.0f);
    t.kind = 1;
}

template <bool CLOTH>
__device__ __forceinline__ void particle_terms(const Params& P, const DevPtrs& d, uint32_t entry,
                                               uint32_t self, ParticleTerms& t) {
    const uint32_t kind = entry >> ADJ_KIND_SHIFT, idx = entry & ADJ_INDEX_MASK;
    t.kind = 3;
    if (kind == FK_TET) {
        tet_terms(d, d.tets[idx], self, t);
    } else if (kind == FK_MANIFOLD) {
        const ManifoldGPU& m = d.manifolds[idx];
        const u4 h = m.header;
        if (h.z != 1u) return;
        const uint32_t a = h.x, b = h.y;
        const bool isA = self == a;
        const bool sphA = (h.w & 2u) != 0, sphB = (h.w & 4u) != 0;
        const float4 qa = d.posAng[a], qb = d.posAng[b];
        const float3 dqALin = xyz(d.posLin[a]) - xyz(d.initLin[a]);
        const float3 dqAAng = q_sub(qa, d.initAng[a]);
        const float3 dqBLin = xyz(d.posLin[b]) - xyz(d.initLin[b]);
        const float3 dqBAng = q_sub(qb, d.initAng[b]);
        const float3 nrm = xyz(m.basisN), t1 = xyz(m.basisT1), t2 = cross(nrm, t1);
        const ContactGPU c = m.contacts[0];
        const float3 rAW = sphA ? xyz(c.rA) : q_rotate(qa, xyz(c.rA));
        const float3 rBW = sphB ? xyz(c.rB) : q_rotate(qb, xyz(c.rB));
        float3 C;
        float fs, bnd;
        const float3 F = contact_force(c, nrm, t1, t2, m.basisN.w, m.basisT1.w, P.alpha, dqALin, dqAAng, dqBLin,
                                       dqBAng, rAW, rBW, C, fs, bnd);
        const float sg = isA ? 1.0f : -1.0f;
        const M3 jLin = M3{nrm * sg, t1 * sg, t2 * sg};
        const M3 K = m3_diag(xyz(c.penalty));
        const M3 jLinT = m3_transpose(jLin);
        const M3 M = m3_mulm(m3_mulm(jLinT, K), jLin);
        t.a = M.r0;
        t.b = M.r1;
        t.c = M.r2;
        t.rhs = m3_mul(jLinT, F);
        t.kind = 2;
    } else if (!CLOTH) {
        return;
    } else if (kind == FK_SPRING) {
        // stamp_spring's linear block: outer(+-n, +-n) equals outer(n, n) bit for bit
        const SpringGPU sp = d.springs[idx];
        const uint32_t a = sp.header.x, b = sp.header.y;
        float stiffness = sp.rA.w;
        const float3 pA = xform(xyz(d.posLin[a]), d.posAng[a], xyz(sp.rA));
        const float3 pB = xform(xyz(d.posLin[b]), d.posAng[b], xyz(sp.rB));
        const float3 dd = pA - pB;
        const float dLen = len3(dd);
        t.kind = TERM_NONE;
        if (dLen <= 1.0e-6f) return;
        const float3 n = dd / dLen;
        float f;
        if (sp.header.z != 0) {
            const float C = dLen - sp.rB.w - sp.dual.z * P.alpha;
            stiffness = sp.dual.y;
            f = stiffness * C + sp.dual.x;
            if (f <= 0.0f) return;
        } else {
            f = stiffness * (dLen - sp.rB.w);
        }
        const float3 jLin = self == a ? n : -n;
        t.rhs = jLin * f;
        t.a = n;
        t.s = mk3(stiffness, mx(f, 0.0f) / dLen, 0.0f);
        t.kind = TERM_SPRING;
    } else if (kind == FK_MEMBRANE) {
        const MembraneGPU mb = d.membranes[idx];
        const float3 x0 = xyz(d.posLin[mb.ids.x]), x1 = xyz(d.posLin[mb.ids.y]), x2 = xyz(d.posLin[mb.ids.z]);
        const float muA = mb.mat.x, lamA = mb.mat.y;
        const float3 d0 = x1 - x0, d1 = x2 - x0;
        const float a = mb.dm.x, b = mb.dm.y, c = mb.dm.z, dm = mb.dm.w;
        const float3 f1 = d0 * a + d1 * b;
        const float3 f2 = d0 * c + d1 * dm;
        const float E11 = 0.5f * (dot(f1, f1) - 1.0f);
        const float E22 = 0.5f * (dot(f2, f2) - 1.0f);
        const float E12 = 0.5f * dot(f1, f2);
        const float trE = E11 + E22;
        const float S11 = 2.0f * muA * E11 + lamA * trE;
        const float S22 = 2.0f * muA * E22 + lamA * trE;
        const float S12 = 2.0f * muA * E12;
        const float3 p1 = f1 * S11 + f2 * S12;
        const float3 p2 = f1 * S12 + f2 * S22;
        float wx, wy;
        if (self == mb.ids.y) { wx = a; wy = c; }
        else if (self == mb.ids.z) { wx = b; wy = dm; }
        else { wx = -a - b; wy = -c - dm; }
        t.rhs = p1 * wx + p2 * wy;
        t.a = f1 * wx;
        t.b = f2 * wy;
        t.c = (f2 * wx + f1 * wy) * 0.5f;
        t.e = t.a + t.b;
        t.s = mk3(2.0f * muA, 4.0f * muA, lamA);
        t.kind = TERM_MEMBRANE;
    } else if (kind == FK_BEND) {
        const BendGPU bd = d.bends[idx];
        const float sc = bd.mat.x;
        const float3 m = xyz(d.posLin[bd.ids.x]) * bd.K.x + xyz(d.posLin[bd.ids.y]) * bd.K.y +
                         xyz(d.posLin[bd.ids.z]) * bd.K.z + xyz(d.posLin[bd.ids.w]) * bd.K.w;
        float k;
        if (self == bd.ids.x) k = bd.K.x;
        else if (self == bd.ids.y) k = bd.K.y;
        else if (self == bd.ids.z) k = bd.K.z;
        else k = bd.K.w;
        t.rhs = m * (sc * k);
        t.s = mk3(sc * k * k, 0.0f, 0.0f);
        t.kind = TERM_BEND;
    } else if (kind == FK_SOFT) {
        const SoftContactGPU& sc = d.soft[idx];
        float3 n, t1, t2, rAW;
        bool rigidA;
        const float3 C = soft_c(P, d, sc, n, t1, t2, rAW, rigidA);
        float3 F = xyz(sc.penalty) * C + xyz(sc.lambda);
        float kN = sc.penalty.x;
        const float rT = sc.anchorA.x;
        const uint32_t kindB = (__float_as_uint(sc.anchorA.w) >> SCF_KIND_SHIFT) & 3u;
        if (rT > 0.0f && kindB != SC_RT && C.x < -0.5f * rT) {
            const float dsep = mx(C.x + rT, 0.02f * rT);
            const float kp = 0.25f * rT * rT * sc.penalty.x;
            F.x = -kp / dsep + sc.lambda.x;
            kN = kp / (dsep * dsep);
        }
        F.x = mn(F.x, 0.0f);
        const float bounds = fabsf(F.x) * sc.normal.w;
        const float fs = sqrtf(F.y * F.y + F.z * F.z);
        if (fs > bounds && fs > 0.0f) {
            const float r = bounds / fs;
            F.y *= r;
            F.z *= r;
        }
        int slot = -1;
        if (sc.ids.x == self) slot = 0;
        else if (sc.ids.y == self) slot = 1;
        else if (sc.ids.z == self) slot = 2;
        else if (sc.ids.w == self) slot = 3;
        t.kind = TERM_NONE;
        if (slot < 0) return;
        if (slot == 0 && rigidA) { t.kind = TERM_SERIAL; return; }
        const float w = slot == 0 ? sc.weights.x : (slot == 1 ? sc.weights.y : (slot == 2 ? sc.weights.z : sc.weights.w));
        const float w2 = w * w;
        t.a = n;
        t.b = t1;
        t.c = t2;
        t.s = mk3(kN * w2, sc.penalty.y * w2, sc.penalty.z * w2);
        t.rhs = (n * F.x + t1 * F.y + t2 * F.z) * w;
        t.kind = TERM_SOFT;
    }
}

__device__ __forceinline__ float3 shfl_idx3(float3 v, int src) {
    return mk3(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src),
               __shfl_sync(0xffffffffu, v.z, src));
}

// Linear block of a particle's system: the only part its solve reads.
struct ParticleAccum { M3 lhs; float3 rhs; };

// Rare entries (joints, springs, multi-contact manifolds) go through the
// generic stamp, which changes lhsLin/rhsLin exactly as it would inside a
// full accumulator.  Scenes that cannot produce them (every dynamic body a
// particle whose adjacency holds only tets and sphere contacts — known at
// upload) use the GENERAL = false instance, which drops these paths and
// their registers.
__device__ __forceinline__ void stamp_entry_particle(const Params& P, const DevPtrs& d, uint32_t entry,
                                                     uint32_t body, ParticleAccum* acc) {
    Accum full{acc->lhs, m3_zero(), m3_zero(), acc->rhs, s3(0)};
    stamp_entry(P, d, entry, body, full);
    acc->lhs = full.lhsLin;
    acc->rhs = full.rhsLin;
}

// Terms of adjacency entry k of particle `body`.  A tet entry reads its
// record from the body's incidence slot (contiguous over consecutive k)
// instead of through the entry; `entry` is what the generic stamp needs.
template <bool CLOTH>
__device__ __forceinline__ void particle_entry_terms(const Params& P, const DevPtrs& d, const AdjView& v,
                                                     uint32_t body, uint32_t k, ParticleTerms& t, uint32_t& entry) {
    const uint32_t kt = k - v.nPre - v.nMan;
    if (d.tetInc && k >= v.nPre + v.nMan && kt < v.nTet) {
        entry = (FK_TET << ADJ_KIND_SHIFT);
        tet_terms(d, d.tetInc[v.postBase + kt], body, t);
    } else {
        entry = v.at(k);
        particle_terms<CLOTH>(P, d, entry, body, t);
    }
}

// Adds one entry's terms to a particle's linear system, in the order of
// operations of the stamps (every instance folds through this function, so
// any lane layout yields the same floats).
template <bool GENERAL, bool CLOTH>
__device__ __forceinline__ void fold_particle_term(const Params& P, const DevPtrs& d, const ParticleTerms& u,
                                                   uint32_t e, uint32_t body, ParticleAccum& acc) {
    if (u.kind == 1u) {
        acc.rhs += u.rhs;
        acc.lhs = m3_add(acc.lhs, m3_diag(s3(u.c.x)));
        acc.lhs = m3_add(acc.lhs, M3{mk3(u.a.x, u.b.x, u.b.y), mk3(u.b.x, u.a.y, u.b.z),
                                     mk3(u.b.y, u.b.z, u.a.z)});
    } else if (u.kind == 2u) {
        acc.lhs = m3_add(acc.lhs, M3{u.a, u.b, u.c});
        acc.rhs += u.rhs;
    } else if (CLOTH && u.kind == TERM_MEMBRANE) {
        acc.rhs += u.rhs;
        acc.lhs = m3_add(acc.lhs, m3_scale(m3_outer(u.a, u.a), u.s.x));
        acc.lhs = m3_add(acc.lhs, m3_scale(m3_outer(u.b, u.b), u.s.x));
        acc.lhs = m3_add(acc.lhs, m3_scale(m3_outer(u.c, u.c), u.s.y));
        acc.lhs = m3_add(acc.lhs, m3_scale(m3_outer(u.e, u.e), u.s.z));
    } else if (CLOTH && u.kind == TERM_BEND) {
        acc.rhs += u.rhs;
        acc.lhs = m3_add(acc.lhs, m3_diag(s3(u.s.x)));
    } else if (CLOTH && u.kind == TERM_SPRING) {
        acc.lhs = m3_add(acc.lhs, m3_scale(m3_outer(u.a, u.a), u.s.x));
        acc.rhs += u.rhs;
        if (u.s.y > 0.0f)
            acc.lhs = m3_add(acc.lhs, m3_add(m3_diag(s3(u.s.y)), m3_scale(m3_outer(u.a, u.a), -u.s.y)));
    } else if (CLOTH && u.kind == TERM_SOFT) {
        acc.lhs = m3_add(acc.lhs, m3_scale(m3_outer(u.a, u.a), u.s.x));
        acc.lhs = m3_add(acc.lhs, m3_scale(m3_outer(u.b, u.b), u.s.y));
        acc.lhs = m3_add(acc.lhs, m3_scale(m3_outer(u.c, u.c), u.s.z));
        acc.rhs += u.rhs;
    } else if (GENERAL && u.kind != TERM_NONE) {
        stamp_entry_particle(P, d, e, body, &acc);
    }
}


// The particle system's angular block is the identity and its cross block
// zero.  Every term of the 6x6 LDL^T that involves them is then an exact
// "x - (+0)" (L4x..L6x, y4..y6, z4..z6 and xAng are all +0), so this 3x3
// sequence returns bit for bit the linear part of solve6x6(lhs, I, 0, b, 0);
// with non-finite input both produce a non-finite step and the update is
// skipped.
__device__ __forceinline__ float3 solve3x3_particle(const M3& a, float3 b) {
    const float s1 = rsq(mx(a.r0.x, 1e-30f));
    const float s2 = rsq(mx(a.r1.y, 1e-30f));
    const float s3_ = rsq(mx(a.r2.z, 1e-30f));
    const float A11 = 1.0f, A22 = 1.0f, A33 = 1.0f;
    const float A21 = a.r1.x * s2 * s1;
    const float A31 = a.r2.x * s3_ * s1, A32 = a.r2.y * s3_ * s2;
    b = mk3(b.x * s1, b.y * s2, b.z * s3_);
    const float L21 = A21 / A11, L31 = A31 / A11;
    const float eps = 1e-6f;
    const float D1 = mx(A11, eps);
    const float D2 = mx(A22 - L21 * L21 * D1, eps);
    const float L32 = (A32 - L21 * L31 * D1) / D2;
    const float D3 = mx(A33 - (L31 * L31 * D1 + L32 * L32 * D2), eps);
    const float y1 = b.x;
    const float y2 = b.y - L21 * y1;
    const float y3 = b.z - L31 * y1 - L32 * y2;
    const float z1 = y1 / D1, z2 = y2 / D2, z3 = y3 / D3;
    float3 x;
    x.z = z3;
    x.y = z2 - L32 * x.z;
    x.x = z1 - L21 * x.y - L31 * x.z;
    return mk3(x.x * s1, x.y * s2, x.z * s3_);
}

// Inertia, solve, trust region, OGC bound and commit of a particle whose
// stamped system is (acc.lhs, acc.rhs); lane 0 of its group calls this.
__device__ __forceinline__ void particle_commit(const Params& P, const DevPtrs& d, uint32_t body, float4 shp,
                                                float4 pl, float4 inert, ParticleAccum acc) {
    const float mass = pl.w;
    const float dt2 = P.dt * P.dt;
    acc.lhs = m3_add(acc.lhs, m3_diag(s3(mass / dt2)));
    acc.rhs += (xyz(pl) - xyz(inert)) * (mass / dt2);
    float3 dxLin = solve3x3_particle(acc.lhs, -acc.rhs);
    if (!finite3(dxLin)) { keep_body(P, d, body, pl, false); return; }
    const float maxLin = 0.35f * fabsf(shp.w);
    const float lin2 = dot(dxLin, dxLin);
    if (lin2 > maxLin * maxLin) dxLin *= maxLin * rsq(lin2);
    if (P.ogc) dxLin = ogc_truncate(d, body, dxLin, xyz(pl), -shp.w);
    if (P.colorJacobi) { d.posNext[body] = mk4(xyz(pl) + dxLin, mass); return; }
    d.posLin[body] = mk4(xyz(pl) + dxLin, mass);
}

// Primal for one color with LANES consecutive lanes per body (8, 16 or 32,
// chosen per color from its bodies' adjacency sizes).  Lane p of a group
// evaluates entry base + p; logical lane l < 8 then folds entries
// base + l, base + l + 8, ... in order.  Any LANES gives the same floats.
// RESID: evaluate instead of solve — lane 0 stores the body's squared
// right-hand side (the AL gradient) in d.learnResidBodies[slot] and leaves
// the pose alone (particle-only scenes; called over all colors at once).
// GENERAL instances keep four blocks per SM (at most 128 registers): the
// rigid-body path would otherwise take ~160 registers for every thread and
// cap large colors at three blocks (measured 7% slower mixed frames).
#ifndef AVBD_PRIMAL_UNROLL
#define AVBD_PRIMAL_UNROLL 1
#endif
constexpr int kPrimalUnroll = AVBD_PRIMAL_UNROLL;
#ifndef AVBD_PARTICLE_PRIMAL_MIN_BLOCKS
#define AVBD_PARTICLE_PRIMAL_MIN_BLOCKS 1
#endif
#ifndef AVBD_LEAN_CLOTH_MIN_BLOCKS
#define AVBD_LEAN_CLOTH_MIN_BLOCKS 5
#endif
template <int LANES, bool GENERAL, bool CLOTH, bool RESID = false>
__global__ void __launch_bounds__(128, GENERAL ? 4 : (CLOTH ? AVBD_LEAN_CLOTH_MIN_BLOCKS : AVBD_PARTICLE_PRIMAL_MIN_BLOCKS)) k_primal_group(const Params P, const DevPtrs d, uint32_t color,
                                                      uint32_t count, uint32_t first, uint32_t start) {
    constexpr int GROUPS = 32 / LANES;
    pdl_trigger();
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t slot = tid / LANES;
    const uint32_t lane = tid & (LANES - 1);
    // The solve takes its body from the color's launch order (lean
    // particles first); the residual pass walks the color list itself.
    // With the color's start known on the host, the launch order, the
    // body's shape and its static adjacency segment (none written after
    // upload) are read before waiting for the previous grid.
    uint32_t s, body;
    float4 shp;
    uint4 seg;
    uint32_t nTet;
    if (!RESID && start != NO_HOST_START) {
        s = start;
        if (slot >= count) return;                           // uniform across the group
        body = d.colorLaunch[s + first + slot];
        shp = d.shape[body];
        seg = d.staticSeg[body];
        nTet = d.postTets[body];
        pdl_wait();
    } else {
        pdl_wait();
        s = d.colorStart[color];
        const uint32_t n = count != 0xFFFFFFFFu ? count : d.colorStart[color + 1] - s;
        if (slot >= n) return;                               // uniform across the group
        body = RESID ? d.colorList[s + slot] : d.colorLaunch[s + first + slot];
        shp = d.shape[body];
        seg = d.staticSeg[body];
        nTet = d.postTets[body];
    }
    const unsigned mask = LANES == 32 ? 0xffffffffu
                                      : (((1u << LANES) - 1u) << ((threadIdx.x & 31u) & ~(uint32_t)(LANES - 1)));
    (void)GROUPS;
    if (GENERAL && shp.w >= 0.0f) {                          // rigid: the 8-lane path
        const unsigned mask8 = mask & (0xFFu << ((threadIdx.x & 31u) & ~(uint32_t)(LANES - 1)));
        if (RESID) {
            if (lane < 8) rigid_residual(P, d, body, lane, mask8, d.learnResidBodies + s + slot);
        } else if (lane < 8) {
            primal_body(P, d, body, lane, mask8);
        }
        return;
    }
    // lane 0 needs these after the reduction; issue the loads now
    float4 pl = make_float4(0, 0, 0, 0), inert = make_float4(0, 0, 0, 0);
    if (lane == 0) { pl = d.posLin[body]; inert = d.inertLin[body]; }
    ParticleAccum acc{m3_zero(), s3(0)};
    const AdjView v = adj_view_from(d, body, seg, nTet);
    const uint32_t cnt = v.count();
#pragma unroll (kPrimalUnroll)
    for (uint32_t base = 0; base < cnt; base += LANES) {
        const uint32_t k = base + lane;
        ParticleTerms t;
        t.kind = 0;
        uint32_t entry = 0;
        if (k < cnt) particle_entry_terms<CLOTH>(P, d, v, body, k, t, entry);
#pragma unroll
        for (int j = 0; j < LANES / 8; j++) {
            const int src = (int)(lane & 7u) + 8 * j;
            ParticleTerms u;
            uint32_t e;
            if (j == 0) {
                // logical lane l already holds entry base + l
                u = t;
                e = entry;
            } else {
            u.kind = __shfl_sync(mask, t.kind, src, LANES);
            u.rhs = mk3(__shfl_sync(mask, t.rhs.x, src, LANES), __shfl_sync(mask, t.rhs.y, src, LANES),
                        __shfl_sync(mask, t.rhs.z, src, LANES));
            u.a = mk3(__shfl_sync(mask, t.a.x, src, LANES), __shfl_sync(mask, t.a.y, src, LANES),
                      __shfl_sync(mask, t.a.z, src, LANES));
            u.b = mk3(__shfl_sync(mask, t.b.x, src, LANES), __shfl_sync(mask, t.b.y, src, LANES),
                      __shfl_sync(mask, t.b.z, src, LANES));
            u.c = mk3(__shfl_sync(mask, t.c.x, src, LANES), __shfl_sync(mask, t.c.y, src, LANES),
                      __shfl_sync(mask, t.c.z, src, LANES));
            if (CLOTH) {
                u.e = mk3(__shfl_sync(mask, t.e.x, src, LANES), __shfl_sync(mask, t.e.y, src, LANES),
                          __shfl_sync(mask, t.e.z, src, LANES));
                u.s = mk3(__shfl_sync(mask, t.s.x, src, LANES), __shfl_sync(mask, t.s.y, src, LANES),
                          __shfl_sync(mask, t.s.z, src, LANES));
            }
            e = __shfl_sync(mask, entry, src, LANES);
            }
            if (lane < 8) fold_particle_term<GENERAL, CLOTH>(P, d, u, e, body, acc);
        }
    }
    // xor butterfly over the 8 logical lanes (offsets 4, 2, 1)
#pragma unroll
    for (int o = 4; o >= 1; o >>= 1) {
        acc.lhs.r0 = acc.lhs.r0 + mk3(__shfl_xor_sync(mask, acc.lhs.r0.x, o, LANES), __shfl_xor_sync(mask, acc.lhs.r0.y, o, LANES), __shfl_xor_sync(mask, acc.lhs.r0.z, o, LANES));
        acc.lhs.r1 = acc.lhs.r1 + mk3(__shfl_xor_sync(mask, acc.lhs.r1.x, o, LANES), __shfl_xor_sync(mask, acc.lhs.r1.y, o, LANES), __shfl_xor_sync(mask, acc.lhs.r1.z, o, LANES));
        acc.lhs.r2 = acc.lhs.r2 + mk3(__shfl_xor_sync(mask, acc.lhs.r2.x, o, LANES), __shfl_xor_sync(mask, acc.lhs.r2.y, o, LANES), __shfl_xor_sync(mask, acc.lhs.r2.z, o, LANES));
        acc.rhs = acc.rhs + mk3(__shfl_xor_sync(mask, acc.rhs.x, o, LANES), __shfl_xor_sync(mask, acc.rhs.y, o, LANES), __shfl_xor_sync(mask, acc.rhs.z, o, LANES));
    }
    if (lane != 0) return;
    if (RESID) {
        const float3 r = acc.rhs + (xyz(pl) - xyz(inert)) * (pl.w / (P.dt * P.dt));
        d.learnResidBodies[s + slot] = dot(r, r);
        return;
    }
    particle_commit(P, d, body, shp, pl, inert, acc);
}

template <bool GENERAL, bool CLOTH>
static void launch_primal_group(const Params& P, const DevPtrs& d, uint32_t color, uint32_t count,
                                uint32_t first, uint32_t start, uint32_t lanes, cudaStream_t st) {
    const int T = 128;
    const uint32_t blocks = (count * lanes + T - 1) / T;
    if (lanes <= 8) launch_pdl(k_primal_group<8, GENERAL, CLOTH>, blocks, T, st, P, d, color, count, first, start);
    else if (lanes <= 16)
        launch_pdl(k_primal_group<16, GENERAL, CLOTH>, blocks, T, st, P, d, color, count, first, start);
    else launch_pdl(k_primal_group<32, GENERAL, CLOTH>, blocks, T, st, P, d, color, count, first, start);
}

// ---------------------------------------------------------------------------
// Staged primal.  A block takes 16 bodies of the color (one 8-lane group
// each, the reference's SIMD layout) and evaluates the terms of all their
// adjacency entries as one flat list — every thread of the block on
// consecutive entries, whatever each body's entry count — into shared
// memory; each group then folds its body's entries in the fixed order
// (logical lane l: entries l, l + 8, ...; xor butterfly 4, 2, 1) and lane 0
// solves.  The grouped kernel above idles the lanes past a body's last
// entry and moves every term through warp shuffles; here the evaluation
// runs dense and the fold reads shared memory.  Entries past the block's
// staging capacity are evaluated inline by the fold, in the same order.
// Rigid bodies (GENERAL) take the 8-lane 6x6 path unchanged.
// ---------------------------------------------------------------------------
constexpr int kStagedThreads = 128;
constexpr int kStagedGroups = kStagedThreads / 8;
constexpr int kStagedSlots = 512;       // staged entries per block
constexpr int kStagedWords = 16;        // kind, rhs, a, b, c, s (e = a + b is recomputed)

struct StagedBody {
    uint32_t body, cnt, staged, off;
    uint32_t preBase, nPre, dynBase, nMan, nDyn, postBase, nTet, nPost;
};

__device__ __forceinline__ AdjView staged_view(const DevPtrs& d, const StagedBody& b) {
    AdjView v;
    v.pre = d.preList + b.preBase; v.nPre = b.nPre;
    v.dyn = d.dynList + b.dynBase; v.nDyn = b.nDyn; v.nMan = b.nMan;
    v.post = d.postList + b.postBase; v.nPost = b.nPost; v.nTet = b.nTet; v.postBase = b.postBase;
    return v;
}

template <bool GENERAL, bool CLOTH>
__global__ void __launch_bounds__(kStagedThreads, GENERAL ? 4 : 5)
k_primal_staged(const Params P, const DevPtrs d, uint32_t color, uint32_t count, uint32_t first, uint32_t start) {
    __shared__ float slots[kStagedWords][kStagedSlots];
    __shared__ StagedBody info[kStagedGroups];
    __shared__ uint32_t offs[kStagedGroups + 1];
    pdl_trigger();
    const uint32_t tid = threadIdx.x;
    const uint32_t head = blockIdx.x * kStagedGroups;
    const bool early = start != NO_HOST_START;
    // bodies of the block, their adjacency views and an exclusive scan of
    // their entry counts (warp 0, one lane per group); with the start known
    // on the host the static part (launch order, shape, static segment) is
    // read before waiting for the previous grid
    if (!early) pdl_wait();
    const uint32_t s = (early ? start : d.colorStart[color]) + first;
    uint32_t cnt = 0, body = 0xFFFFFFFFu;
    StagedBody sb{};
    const bool mine = tid < kStagedGroups && head + tid < count;
    float4 bodyShape = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (mine) {
        body = d.colorLaunch[s + head + tid];
        bodyShape = d.shape[body];
        const uint4 seg = d.staticSeg[body];
        sb.preBase = seg.x; sb.nPre = seg.y; sb.postBase = seg.z; sb.nPost = seg.w;
        sb.nTet = d.postTets[body];
    }
    if (early) pdl_wait();                                   // every thread, before any per-frame read
    if (tid < 32) {
        if (mine) {
            sb.dynBase = d.dynStart[body]; sb.nDyn = d.dynCount[body]; sb.nMan = d.dynSplit[body];
            cnt = sb.nPre + sb.nDyn + sb.nPost;
            sb.cnt = cnt;
            if (GENERAL && bodyShape.w >= 0.0f) cnt = 0;           // rigid: stages nothing
        }
        uint32_t incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if ((int)tid >= o) incl += y;
        }
        const uint32_t off = incl - cnt;
        if (tid < kStagedGroups) {
            sb.body = body;
            sb.off = off;
            sb.staged = off >= (uint32_t)kStagedSlots ? 0u : min(cnt, (uint32_t)kStagedSlots - off);
            info[tid] = sb;
            offs[tid] = off;
        }
        if (tid == kStagedGroups - 1) offs[kStagedGroups] = min(incl, (uint32_t)kStagedSlots);
    }
    __syncthreads();
    // every staged entry of the block, dense over the threads
    const uint32_t total = offs[kStagedGroups];
    for (uint32_t i = tid; i < total; i += kStagedThreads) {
        uint32_t g = 0;
#pragma unroll
        for (uint32_t step = kStagedGroups / 2; step >= 1; step >>= 1)
            if (offs[g + step] <= i) g += step;
        const StagedBody& b = info[g];
        const AdjView v = staged_view(d, b);
        ParticleTerms t;
        uint32_t entry = 0;
        particle_entry_terms<CLOTH>(P, d, v, b.body, i - b.off, t, entry);
        slots[0][i] = __uint_as_float(t.kind);
        slots[1][i] = t.kind == TERM_SERIAL ? __uint_as_float(entry) : t.rhs.x;
        slots[2][i] = t.rhs.y;  slots[3][i] = t.rhs.z;
        slots[4][i] = t.a.x;    slots[5][i] = t.a.y;    slots[6][i] = t.a.z;
        slots[7][i] = t.b.x;    slots[8][i] = t.b.y;    slots[9][i] = t.b.z;
        slots[10][i] = t.c.x;   slots[11][i] = t.c.y;   slots[12][i] = t.c.z;
        if (CLOTH) { slots[13][i] = t.s.x; slots[14][i] = t.s.y; slots[15][i] = t.s.z; }
    }
    __syncthreads();
    // the fold: group g, logical lane l
    const uint32_t g = tid >> 3, lane = tid & 7u;
    if (head + g >= count) return;
    const StagedBody b = info[g];
    const unsigned mask8 = 0xFFu << (tid & 24u);
    const float4 shp = d.shape[b.body];
    if (GENERAL && shp.w >= 0.0f) {
        primal_body(P, d, b.body, lane, mask8);
        return;
    }
    float4 pl = make_float4(0, 0, 0, 0), inert = make_float4(0, 0, 0, 0);
    if (lane == 0) { pl = d.posLin[b.body]; inert = d.inertLin[b.body]; }
    ParticleAccum acc{m3_zero(), s3(0)};
    for (uint32_t k = lane; k < b.cnt; k += 8) {
        ParticleTerms u;
        uint32_t e = 0;
        if (k < b.staged) {
            const uint32_t i = b.off + k;
            u.kind = __float_as_uint(slots[0][i]);
            e = __float_as_uint(slots[1][i]);
            u.rhs = mk3(slots[1][i], slots[2][i], slots[3][i]);
            u.a = mk3(slots[4][i], slots[5][i], slots[6][i]);
            u.b = mk3(slots[7][i], slots[8][i], slots[9][i]);
            u.c = mk3(slots[10][i], slots[11][i], slots[12][i]);
            if (CLOTH) {
                u.s = mk3(slots[13][i], slots[14][i], slots[15][i]);
                u.e = u.a + u.b;                             // as the membrane terms form it
            }
        } else {
            particle_entry_terms<CLOTH>(P, d, staged_view(d, b), b.body, k, u, e);
        }
        fold_particle_term<GENERAL, CLOTH>(P, d, u, e, b.body, acc);
    }
#pragma unroll
    for (int o = 4; o >= 1; o >>= 1) {
        add_shfl3(mask8, acc.lhs.r0, o);
        add_shfl3(mask8, acc.lhs.r1, o);
        add_shfl3(mask8, acc.lhs.r2, o);
        add_shfl3(mask8, acc.rhs, o);
    }
    if (lane != 0) return;
    particle_commit(P, d, b.body, shp, pl, inert, acc);
}

template <bool GENERAL, bool CLOTH>
static void launch_primal_staged(const Params& P, const DevPtrs& d, uint32_t color, uint32_t count,
                                 uint32_t first, uint32_t start, cudaStream_t st) {
    const uint32_t blocks = (count + kStagedGroups - 1) / kStagedGroups;
    launch_pdl(k_primal_staged<GENERAL, CLOTH>, blocks, kStagedThreads, st, P, d, color, count, first, start);
}

void launch_primal_color(const Params& P, const DevPtrs& d, const Sizes& z, uint32_t color, uint32_t count,
                         uint32_t lanes, cudaStream_t st, cudaStream_t side, cudaEvent_t fork, cudaEvent_t join) {
    const int T = 128;
    const uint32_t upper = count != 0xFFFFFFFFu ? count : z.numDynamicBodies;
    if (upper == 0) return;
    if (z.dynamicColoring) {
        // dynamic coloring: the color's size is known on the device only, so
        // one resident wave (4 blocks per SM at 128 registers) strides over
        // it instead of a grid sized for every dynamic body (batched worlds
        // 1.007 -> 0.965 ms per frame; half a wave measured 1.22 ms)
        const uint32_t TT = z.dynThreads ? z.dynThreads : (uint32_t)T;
        const uint32_t need = (upper * 8 + TT - 1) / TT, wave = z.dynBlocks ? z.dynBlocks : 148u * 4u;
        launch_pdl(k_primal, need < wave ? need : wave, TT, st, P, d, color, count);
    } else {
        // The grouped and staged kernels need the color's body count on the
        // host.  The color's lean particles (the head of its launch order)
        // run in the instance without the rigid and generic-stamp paths,
        // which needs far fewer registers; the rest in the general one.
        const bool cloth = P.cloth || P.ogc;
        const uint32_t lean = z.particleFastPath ? upper : (z.colorLean ? min(z.colorLean[color], upper) : 0u);
        const uint32_t rest = upper - lean;
        const uint32_t start = z.colorStartHost ? z.colorStartHost[color] : NO_HOST_START;
        const bool split = rest && lean && side && fork && join;
        if (split) {
            cudaEventRecord(fork, st);
            cudaStreamWaitEvent(side, fork, 0);
            launch_primal_wide(P, d, color, rest, lean, start, side);
        }
        if (lean) {
            if (lanes == AVBD_PRIMAL_STAGED) {
                if (cloth) launch_primal_staged<false, true>(P, d, color, lean, 0, start, st);
                else launch_primal_staged<false, false>(P, d, color, lean, 0, start, st);
            } else {
                const uint32_t lanes_ = lanes < 8 ? 8 : (lanes > 32 ? 32 : lanes);
                const uint32_t w = lanes_ <= 8 ? 8 : (lanes_ <= 16 ? 16 : 32);
                if (cloth) launch_primal_group<false, true>(P, d, color, lean, 0, start, w, st);
                else launch_primal_group<false, false>(P, d, color, lean, 0, start, w, st);
            }
        }
        // the rest: a block per body (rigid bodies with many contacts)
        if (split) {
            cudaEventRecord(join, side);
            cudaStreamWaitEvent(st, join, 0);
        } else {
            launch_primal_wide(P, d, color, rest, lean, start, st);
        }
    }
}

void launch_residual(const Params& P, const DevPtrs& d, const Sizes& z, float* perBody, double* total,
                     cudaStream_t st) {
    const uint32_t n = z.numDynamicBodies;
    if (n && z.numDynamicRigid == 0) {
        // particle-only: the group stamping of the primal over all colors at
        // once, writing the per-body values to perBody
        DevPtrs g = d;
        g.learnResidBodies = perBody;
        auto run = [&](uint32_t color, uint32_t count, uint32_t lanes) {
            const uint32_t w = lanes <= 8 ? 8u : (lanes <= 16 ? 16u : 32u);
            const uint32_t blocks = (count * w + 127) / 128;
            if (z.particleFastPath) {
                if (w == 8) k_primal_group<8, false, false, true><<<blocks, 128, 0, st>>>(P, g, color, count, 0u, NO_HOST_START);
                else if (w == 16) k_primal_group<16, false, false, true><<<blocks, 128, 0, st>>>(P, g, color, count, 0u, NO_HOST_START);
                else k_primal_group<32, false, false, true><<<blocks, 128, 0, st>>>(P, g, color, count, 0u, NO_HOST_START);
            } else if (P.cloth || P.ogc) {
                k_primal_group<32, true, true, true><<<(count * 32 + 127) / 128, 128, 0, st>>>(P, g, color, count, 0u, NO_HOST_START);
            } else {
                k_primal_group<32, true, false, true><<<(count * 32 + 127) / 128, 128, 0, st>>>(P, g, color, count, 0u, NO_HOST_START);
            }
        };
        // every body at once: 8 lanes per body keep the most bodies in
        // flight (measured faster than 16 or 32 for the 13,824-body soft cube)
        run(0u, n, 8u);
    } else if (n) {
        // rigid bodies present: particles through the primal's particle
        // terms, rigid bodies through the generic stamps, 8 lanes per body
        DevPtrs g = d;
        g.learnResidBodies = perBody;
        const uint32_t blocks = (n * 8 + 127) / 128;
        if (P.cloth || P.ogc) k_primal_group<8, true, true, true><<<blocks, 128, 0, st>>>(P, g, 0u, n, 0u, NO_HOST_START);
        else k_primal_group<8, true, false, true><<<blocks, 128, 0, st>>>(P, g, 0u, n, 0u, NO_HOST_START);
    }
    k_sum_fixed<<<1, 1024, 0, st>>>(perBody, n, total);
}

// ---------------------------------------------------------------------------
// Dual (40_solver.metal:1729-1906)
// ---------------------------------------------------------------------------
__device__ void dual_joint(const Params& P, const DevPtrs& d, uint32_t gid) {
    JointGPU& j = d.joints[gid];
    if (j.header.z != 0) return;
    const uint32_t a = j.header.x, b = j.header.y;
    const float torqueArm = j.C0Lin.w, stiffLin = j.rA.w, stiffAng = j.rB.w;
    const float3 penLin = xyz(j.penaltyLin);
    if (dot(penLin, penLin) > 0.0f) {
        const float3 pA = a == WORLD_BODY ? xyz(j.rA) : xform(xyz(d.posLin[a]), d.posAng[a], xyz(j.rA));
        const float3 pB = xform(xyz(d.posLin[b]), d.posAng[b], xyz(j.rB));
        float3 C = pA - pB;
        if (j.header.w & 1) {
            C -= xyz(j.C0Lin) * P.alpha;
            const float3 l = clamp3(penLin * C + xyz(j.lambdaLin), s3(-P.lambdaMax), s3(P.lambdaMax));
            j.lambdaLin = tof4(l, j.lambdaLin.w);
        }
        const float cap = mn(stiffLin, PENALTY_MAX);
        j.penaltyLin = tof4(mn3(penLin + abs3(C) * P.betaLin, s3(cap)), j.penaltyLin.w);
    }
    const float3 penAng = xyz(j.penaltyAng);
    if (dot(penAng, penAng) > 0.0f) {
        const float4 qA = a == WORLD_BODY ? make_float4(0, 0, 0, 1) : d.posAng[a];
        const float4 restRel = tof(j.restRel);
        float3 C;
        if (j.hingeAxis.w != 0.0f) {
            const float3 axis = xyz(j.hingeAxis);
            const float3 aB = q_rotate(d.posAng[b], axis);
            const float3 aA = q_rotate(q_mul(qA, restRel), axis);
            C = cross(aA, aB) * torqueArm;
        } else {
            C = q_sub(q_mul(qA, restRel), d.posAng[b]) * torqueArm;
        }
        if (j.header.w & 2) {
            C -= xyz(j.C0Ang) * P.alpha;
            const float3 l = clamp3(penAng * C + xyz(j.lambdaAng), s3(-P.lambdaMax), s3(P.lambdaMax));
            j.lambdaAng = tof4(l, j.lambdaAng.w);
        }
        const float cap = mn(stiffAng, PENALTY_MAX);
        j.penaltyAng = tof4(mn3(penAng + abs3(C) * P.betaAng, s3(cap)), j.penaltyAng.w);
    }
    const float fracture = j.C0Ang.w;
    const float3 la = xyz(j.lambdaAng);
    const float3 ll = xyz(j.lambdaLin);
    const float lin2 = (j.header.w & 8) ? dot(ll, ll) : 0.0f;
    if ((j.header.w & 4) && dot(la, la) + lin2 > fracture * fracture) {
        j.penaltyLin = f4{0, 0, 0, 0};
        j.penaltyAng = f4{0, 0, 0, 0};
        j.lambdaLin = f4{0, 0, 0, 0};
        j.lambdaAng = f4{0, 0, 0, 0};
        j.header.z = 1;
    }
}

__device__ void dual_spring(const Params& P, const DevPtrs& d, uint32_t si) {
    SpringGPU& sp = d.springs[si];
    const uint32_t a = sp.header.x, b = sp.header.y;
    const float3 pA = xform(xyz(d.posLin[a]), d.posAng[a], xyz(sp.rA));
    const float3 pB = xform(xyz(d.posLin[b]), d.posAng[b], xyz(sp.rB));
    const float C = len3(pA - pB) - sp.rB.w - sp.dual.z * P.alpha;
    const float mA = d.posLin[a].w, mB = d.posLin[b].w;
    const float mMin = mn(mA > 0.0f ? mA : FLT_BIG, mB > 0.0f ? mB : FLT_BIG);
    const float cap = mn(P.lambdaMax, mx(2.0f, 5.0e3f * mMin));
    sp.dual.x = clampf(0.98f * sp.dual.x + sp.dual.y * C, 0.0f, cap);
    if (C > 0.0f) sp.dual.y = mn(sp.dual.y + C * P.betaLin, mn(sp.rA.w, PENALTY_MAX));
}

__device__ void dual_manifold(const Params& P, const DevPtrs& d, uint32_t gid) {
    ManifoldGPU& m = d.manifolds[gid];
    const u4 h = m.header;
    const uint32_t n = h.z;
    if (n == 0) return;
    const uint32_t a = h.x, b = h.y;
    const bool sphA = (h.w & 2u) != 0, sphB = (h.w & 4u) != 0;
    const float4 pa4 = d.posLin[a], pb4 = d.posLin[b], qa = d.posAng[a], qb = d.posAng[b];
    const float3 dqALin = xyz(pa4) - xyz(d.initLin[a]);
    const float3 dqAAng = q_sub(qa, d.initAng[a]);
    const float3 dqBLin = xyz(pb4) - xyz(d.initLin[b]);
    const float3 dqBAng = q_sub(qb, d.initAng[b]);
    const float minMass = mn(pa4.w > 0.0f ? pa4.w : FLT_BIG, pb4.w > 0.0f ? pb4.w : FLT_BIG);
    const float lamCap = mn(P.lambdaMax, mx(10.0f, 1.0e5f * minMass));
    const float3 nrm = xyz(m.basisN), t1 = xyz(m.basisT1), t2 = cross(nrm, t1);
    const float dynF = m.basisN.w, statF = m.basisT1.w;
    for (uint32_t i = 0; i < n; i++) {
        ContactGPU& c = m.contacts[i];
        const float3 rAW = sphA ? xyz(c.rA) : q_rotate(qa, xyz(c.rA));
        const float3 rBW = sphB ? xyz(c.rB) : q_rotate(qb, xyz(c.rB));
        float3 C;
        float fs, bounds;
        float3 F = contact_force(c, nrm, t1, t2, dynF, statF, P.alpha, dqALin, dqAAng, dqBLin, dqBAng,
                                 rAW, rBW, C, fs, bounds);
        F.x = mx(F.x, -lamCap);
        c.lambda = tof4(F, 0.0f);
        float3 pen = xyz(c.penalty);
        if (F.x < 0.0f) pen.x = mn(pen.x + P.betaLin * fabsf(C.x), PENALTY_MAX);
        if (fs <= bounds) {
            pen.y = mn(pen.y + P.betaLin * fabsf(C.y), PENALTY_MAX_T);
            pen.z = mn(pen.z + P.betaLin * fabsf(C.z), PENALTY_MAX_T);
            c.rB.w = sqrtf(C.y * C.y + C.z * C.z) < STICK_THRESH ? 1.0f : 0.0f;
        }
        c.penalty = tof4(pen, 0.0f);
    }
}

// dual_soft_one (40_solver.metal:1689-1727): quadratic stage only.
__device__ void dual_soft(const Params& P, const DevPtrs& d, uint32_t i) {
    SoftContactGPU& sc = d.soft[i];
    float3 n, t1, t2, rAW;
    bool rigidA;
    const float3 C = soft_c(P, d, sc, n, t1, t2, rAW, rigidA);
    float3 F = xyz(sc.penalty) * C + xyz(sc.lambda);
    F.x = mn(F.x, 0.0f);
    const float bnd = fabsf(F.x) * sc.normal.w;
    const float fs = sqrtf(F.y * F.y + F.z * F.z);
    if (fs > bnd && fs > 0.0f) {
        const float r = bnd / fs;
        F.y *= r;
        F.z *= r;
    }
    F.x = mx(F.x, -sc.C0.w);
    sc.lambda = tof4(F, sc.lambda.w);
    float3 pen = xyz(sc.penalty);
    if (F.x < 0.0f) pen.x = mn(pen.x + P.betaLin * fabsf(C.x), PENALTY_MAX_T);
    if (fs <= bnd) {
        pen.y = mn(pen.y + P.betaLin * fabsf(C.y), PENALTY_MAX_T);
        pen.z = mn(pen.z + P.betaLin * fabsf(C.z), PENALTY_MAX_T);
    }
    sc.penalty = tof4(pen, sc.penalty.w);
}

__device__ __forceinline__ void dual_item(const Params& P, const DevPtrs& d, const Sizes& z, uint32_t g,
                                          uint32_t numPairs) {
    if (g < z.numActiveJoints) { dual_joint(P, d, d.activeJoints[g]); return; }
    g -= z.numActiveJoints;
    if (g < z.numHardSprings) { dual_spring(P, d, d.hardSprings[g]); return; }
    g -= z.numHardSprings;
    if (g < numPairs) { dual_manifold(P, d, g); return; }
    dual_soft(P, d, g - numPairs);
}

__global__ void k_dual(const Params P, const DevPtrs d, const Sizes z) {
    pdl_prologue();
    const uint32_t numPairs = d.counters->numPairs;
    const uint32_t numSoft = (P.cloth || P.ogc) ? d.counters->numSoft : 0u;
    const uint32_t total = z.numActiveJoints + z.numHardSprings + numPairs + numSoft;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x)
        dual_item(P, d, z, g, numPairs);
}

void launch_dual(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    const uint32_t upper = z.numActiveJoints + z.numHardSprings + z.maxPairs + ((P.cloth || P.ogc) ? z.maxSoft : 0u);
    launch_pdl(k_dual, stride_blocks(upper, 128), 128, st, P, d, z);
}

// ---------------------------------------------------------------------------
// Small scenes: the whole iteration loop in one thread block.  Colors and the
// dual are separated by __syncthreads(), which orders the same way as the
// per-color launches.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_solve_small(const Params P, const DevPtrs d, const Sizes z,
                                                     uint32_t colorBound) {
    const uint32_t groups = blockDim.x >> 3;
    const uint32_t group = threadIdx.x >> 3, lane = threadIdx.x & 7u;
    const unsigned mask = 0xFFu << (threadIdx.x & 24u);
    // the color offsets do not change during the solve: one copy in shared
    // memory instead of a dependent global load per color per iteration
    __shared__ uint32_t cs[MAX_COLORS + 1];
    for (uint32_t c = threadIdx.x; c <= colorBound && c <= (uint32_t)MAX_COLORS; c += blockDim.x) cs[c] = d.colorStart[c];
    __syncthreads();
    uint32_t last = 0;                           // one past the last non-empty color
    for (uint32_t c = 0; c < colorBound; c++) if (cs[c + 1] != cs[c]) last = c + 1;
    for (uint32_t it = 0; it < P.iterations; it++) {
        for (uint32_t c = 0; c < last; c++) {
            const uint32_t s = cs[c], e = cs[c + 1];
            if (s == e) continue;                // block-uniform
            for (uint32_t slot = group; s + slot < e; slot += groups)
                primal_body(P, d, d.colorList[s + slot], lane, mask);
            __syncthreads();
        }
        const uint32_t numPairs = d.counters->numPairs;
        const uint32_t total = z.numActiveJoints + z.numHardSprings + numPairs;
        for (uint32_t g = threadIdx.x; g < total; g += blockDim.x) dual_item(P, d, z, g, numPairs);
        __syncthreads();
    }
}

void launch_solve_small(const Params& P, const DevPtrs& d, const Sizes& z, uint32_t colorBound, cudaStream_t st) {
    k_solve_small<<<1, 256, 0, st>>>(P, d, z, colorBound);
}

// Dynamic coloring: the frame graph launches colors [0, first) one by one
// and this single block handles any colors from `first` up (rare: a frame
// that needs more colors than the graph was built for), color after color
// with a block barrier between them — the same per-body solve in the same
// color order.
__global__ void __launch_bounds__(256) k_primal_tail(const Params P, const DevPtrs d, uint32_t first) {
    pdl_prologue();
    const uint32_t groups = blockDim.x >> 3;
    const uint32_t group = threadIdx.x >> 3, lane = threadIdx.x & 7u;
    const unsigned mask = 0xFFu << (threadIdx.x & 24u);
    for (uint32_t c = first; c < (uint32_t)MAX_COLORS; c++) {
        const uint32_t s = d.colorStart[c], e = d.colorStart[c + 1];
        if (s == e) continue;                    // block-uniform
        for (uint32_t slot = group; s + slot < e; slot += groups)
            primal_body(P, d, d.colorList[s + slot], lane, mask);
        __syncthreads();
    }
}

void launch_primal_tail(const Params& P, const DevPtrs& d, const Sizes& z, uint32_t first, cudaStream_t st) {
    if (first < (uint32_t)MAX_COLORS) launch_pdl(k_primal_tail, 1, 256, st, P, d, first);
}

// ---------------------------------------------------------------------------
// BDF1 velocity finalize (40_solver.metal:2108-2147)
// ---------------------------------------------------------------------------
__global__ void k_finalize(const Params P, const DevPtrs d) {
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= P.numBodies) return;
    const float4 vold = d.velLin[gid];
    d.prevVelLin[gid] = vold;
    const float4 pl = d.posLin[gid];
    if (pl.w <= 0.0f) return;
    const float4 shp = d.shape[gid];
    const float3 oldV = xyz(vold);
    float3 v = (xyz(pl) - xyz(d.initLin[gid])) / P.dt;
    const float s2 = dot(v, v);
    if (s2 > P.maxSpeed * P.maxSpeed) v *= P.maxSpeed * rsq(s2);
    if (shp.w < 0.0f && P.particleDamping > 0.0f) {
        const float3 ballistic = oldV + mk3(0, 0, P.gravity * d.gravityScale[gid]) * P.dt;
        v = ballistic + (v - ballistic) / (1.0f + P.particleDamping * P.dt);
    }
    if (shp.w >= 0.0f && P.rigidLinearDamping > 0.0f) v *= expf(-P.rigidLinearDamping * P.dt);
    float3 omega = q_sub(d.posAng[gid], d.initAng[gid]) / P.dt;
    if (shp.w >= 0.0f && P.rigidAngularDamping > 0.0f) omega *= expf(-P.rigidAngularDamping * P.dt);
    d.velLin[gid] = mk4(v, 0.0f);
    d.velAng[gid] = mk4(omega, 0.0f);
}

void launch_finalize(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    k_finalize<<<(P.numBodies + 127) / 128, 128, 0, st>>>(P, d);
}

// ---------------------------------------------------------------------------
// max joint violation / contact penetration (40_solver.metal:2189-2229).
// Manifolds were swapped at frame end: the last frame's are prevManifolds.
// ---------------------------------------------------------------------------
__global__ void k_diag(const Params P, const DevPtrs d, const Sizes z) {
    const uint32_t numPairs = d.counters->numPairs;
    const uint32_t total = P.numJoints + numPairs;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
        float err = 0.0f;
        if (g < P.numJoints) {
            const JointGPU& j = d.joints[g];
            if (!(j.header.z == 0 && (j.rA.w > 0.0f || j.rB.w > 0.0f))) continue;
            const uint32_t a = j.header.x, b = j.header.y;
            const float3 pA = a == WORLD_BODY ? xyz(j.rA) : xform(xyz(d.posLin[a]), d.posAng[a], xyz(j.rA));
            const float3 pB = xform(xyz(d.posLin[b]), d.posAng[b], xyz(j.rB));
            err = len3(pA - pB);
        } else {
            const ManifoldGPU& m = d.prevManifolds[g - P.numJoints];
            const u4 h = m.header;
            const bool sphA = (h.w & 2u) != 0, sphB = (h.w & 4u) != 0;
            for (uint32_t i = 0; i < h.z; i++) {
                const float3 xA = sphA ? xyz(d.posLin[h.x]) + xyz(m.contacts[i].rA)
                                       : xform(xyz(d.posLin[h.x]), d.posAng[h.x], xyz(m.contacts[i].rA));
                const float3 xB = sphB ? xyz(d.posLin[h.y]) + xyz(m.contacts[i].rB)
                                       : xform(xyz(d.posLin[h.y]), d.posAng[h.y], xyz(m.contacts[i].rB));
                const float pen = dot(xyz(m.basisN), xA - xB) + P.collisionMargin;
                err = mx(err, mx(0.0f, -pen));
            }
        }
        atomicMax(reinterpret_cast<uint32_t*>(d.diag), __float_as_uint(err));
    }
}

void launch_max_constraint_error(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    cudaMemsetAsync(d.diag, 0, sizeof(float), st);
    k_diag<<<stride_blocks(P.numJoints + z.maxPairs, 128), 128, 0, st>>>(P, d, z);
}

// ---------------------------------------------------------------------------
// set_body_states: clear the AL state of every constraint incident to a
// reset body (GPUSolver.swift:2429-2471).
// ---------------------------------------------------------------------------
__global__ void k_reset_incident(const Params P, const DevPtrs d, const Sizes z) {
    const uint32_t total = P.numJoints + P.numSprings + 2 * z.maxPairs;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
        if (g < P.numJoints) {
            JointGPU& j = d.joints[g];
            const uint32_t a = j.header.x, b = j.header.y;
            if (d.resetFlags[b] || (a != WORLD_BODY && d.resetFlags[a])) {
                j.lambdaLin = f4{0, 0, 0, 0};
                j.lambdaAng = f4{0, 0, 0, 0};
                j.motor.z = 0.0f;
                j.dynamics.y = 0.0f;
                j.dynamics.z = 0.0f;
                j.penaltyLin = tof4(d.initPenLin[g]);
                j.penaltyAng = tof4(d.initPenAng[g]);
            }
            continue;
        }
        g -= P.numJoints;
        if (g < P.numSprings) {
            SpringGPU& sp = d.springs[g];
            if (d.resetFlags[sp.header.x] || d.resetFlags[sp.header.y]) sp.dual = f4{0, 0, 0, 0};
            continue;
        }
        g -= P.numSprings;
        ManifoldGPU* buf = g < z.maxPairs ? d.manifolds : d.prevManifolds;
        const uint32_t m = g < z.maxPairs ? g : g - z.maxPairs;
        const u4 h = buf[m].header;
        const bool hitA = h.x < P.numBodies && d.resetFlags[h.x];
        const bool hitB = h.y < P.numBodies && d.resetFlags[h.y];
        if (hitA || hitB) {
            uint4* w = reinterpret_cast<uint4*>(&buf[m]);
            for (int k = 0; k < (int)(sizeof(ManifoldGPU) / 16); k++) w[k] = make_uint4(0, 0, 0, 0);
        }
    }
}

void launch_reset_bodies(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    k_reset_incident<<<stride_blocks(P.numJoints + P.numSprings + 2 * z.maxPairs, 128), 128, 0, st>>>(P, d, z);
}

// ---------------------------------------------------------------------------
// End of frame: kinematic spinners and legacy rate motors advance only after
// a complete frame (GPUSolver.swift:4359-4363, :4407-4427), then the frame's
// counters are checked and the first failure is latched with its frame index
// (the checks of `retire`, GPUSolver.swift:2885-2918).
// ---------------------------------------------------------------------------
__global__ void k_frame_end(const Params P, const DevPtrs d, const Sizes z, float dt) {
    const uint32_t t = threadIdx.x;
    for (uint32_t i = t; i < d.numRateMotors; i += blockDim.x) {
        JointGPU& j = d.joints[d.rateJoint[i]];
        float target = j.motor.x + d.rateValue[i] * dt;
        target -= 6.28318530717958647692f * roundf(target / 6.28318530717958647692f);
        j.motor.x = target;
    }
    for (uint32_t i = t; i < d.numSpinners; i += blockDim.x) {
        const uint32_t b = d.spinnerBody[i];
        const float4 ao = d.spinnerAxisOmega[i];
        const float half = 0.5f * ao.w * dt;
        const float sn = sinf(half);
        const float4 dq = make_float4(ao.x * sn, ao.y * sn, ao.z * sn, cosf(half));
        const float4 nq = q_mul(dq, d.posAng[b]);
        d.posAng[b] = nq / sqrtf(dot4(nq, nq));
    }
    if (t == 0) {
        const uint32_t frame = d.frameCounter[0] + 1u;
        d.frameCounter[0] = frame;
        uint32_t kind = 0, detail = 0;
        const Counters* c = d.counters;
        if (c->pairCandidates > P.maxPairs) { kind = AVBD_FAIL_RIGID_PAIR_CAPACITY_; detail = c->pairCandidates; }
        else if ((P.cloth || P.ogc) && c->softRaw > P.maxSoft) { kind = 3; detail = c->softRaw; }
        else if (P.cloth && c->datPairsPeak > P.maxDatPairs) { kind = 6; detail = c->datPairsPeak; }
        else if (P.cloth && c->datGridOverflow > 0) { kind = 7; detail = c->datGridOverflow; }
        else if (P.cloth && c->datInvalidAnchor > 0) { kind = 8; detail = c->datInvalidAnchor; }
        else if (z.dynamicColoring && c->colorConflicts > 0) { kind = AVBD_FAIL_UNRESOLVED_COLORING_; detail = c->colorConflicts; }
        if (kind != 0 && d.failureLatch[0] == 0u) {
            d.failureLatch[0] = kind;
            d.failureLatch[1] = frame;
            d.failureLatch[2] = detail;
        }
        // peak dynamic palette size, read by the host to size the color launches
        if (z.dynamicColoring && c->usedColors > d.failureLatch[3]) d.failureLatch[3] = c->usedColors;
        // OGC bound exceeders of the last pass (the counter the reference
        // leaves at frame end: every earlier pass is consumed by a refresh)
        if (P.ogc) d.counters->ogcExceeded = P.iterations ? c->ogcSlots[(P.iterations - 1u) & 1u] : 0u;
    }
}

void launch_frame_end(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    k_frame_end<<<1, 64, 0, st>>>(P, d, z, P.dt);
}

}  // namespace avbd
