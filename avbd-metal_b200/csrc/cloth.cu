// cloth.cu — the Planar-DAT element-contact pipeline of shell scenes:
// element grid, Planar-DAT pair streams, rigid-triangle and vertex-triangle /
// edge-edge contact emission, the soft persistence map and the Planar-DAT
// truncation passes.  Rigid-triangle emission, the soft map and velocity
// smoothing also serve the isotropic-OGC pipeline (ogc.cu).
//
// Follows Shaders/25_cloth.metal (element grid :147-267, soft map :79-145,
// softEmit :269-333, rigid-triangle emission :942-1142),
// Shaders/27_planar_dat.metal (pair streams :35-228, contact emission
// :344-510, truncation :525-561, :752-946, :1179-1310) and the stage order
// of GPUSolver.swift:3683-3871.
//
// Every list this file produces has a fixed order, so a frame is the same on
// every run:
//   * pair streams: V-T pairs by (particle, triangle), then E-E pairs by
//     (edge, other edge).  One warp owns a query; pairs are counted, scanned
//     over the queries and emitted, then each warp sorts its own segment;
//   * element contacts: rigid-triangle records by triangle (at most four per
//     triangle, in visiting order), then vertex-triangle / edge-edge records
//     in pair order;
//   * truncation fractions are minima (order-free atomics on float bits of
//     non-negative values).
// A color's solve is published by the color pass (launch_dat_color): the
// primal writes posNext, so bodies of one color read each other's pre-color
// pose.
#include "elements.cuh"
#include "pdl.cuh"

namespace avbd {

namespace {

// Tight AABB of element gid (triangles, then edges).
__device__ void elem_tight(const Params& P, const DevPtrs& d, uint32_t gid, float3& lo, float3& hi) {
    if (gid < P.numTris) {
        const uint4 t = d.tris[gid];
        const float3 a = xyz(d.posLin[t.x]), b = xyz(d.posLin[t.y]), c = xyz(d.posLin[t.z]);
        lo = vmin(vmin(a, b), c);
        hi = vmax(vmax(a, b), c);
    } else {
        const uint2 e = d.edges[gid - P.numTris];
        const float3 a = xyz(d.posLin[e.x]), b = xyz(d.posLin[e.y]);
        lo = vmin(a, b);
        hi = vmax(a, b);
    }
}

// Element AABB padded by the Planar-DAT query radius (25_cloth.metal:147-180),
// from the tight box stored by the binning pass (min/max are exact, so the
// padded bounds carry the same bits as when computed from the vertices).
__device__ __forceinline__ void elem_bounds(const Params& P, const DevPtrs& d, uint32_t gid, float3& lo, float3& hi) {
    const float4 l = d.elemBox[2 * gid], h = d.elemBox[2 * gid + 1];
    lo = xyz(l) - s3(P.queryRadius);
    hi = xyz(h) + s3(P.queryRadius);
}

// A conservative reach for box prefilters: anything within the query radius
// by the exact float test also lies within this distance of the tight box.
__device__ __forceinline__ float prefilter_reach(const Params& P) { return P.queryRadius * 1.001f + 1.0e-5f; }

// ---------------------------------------------------------------------------
// Element grid: every triangle and edge in each distinct bucket of its
// (at most 4x4x4) cell cover.  Triangles and edges are binned into separate
// halves of the count array ([0, H) triangles, [H, 2H) edges) so that a V-T
// query scans only triangles and an E-E query only edges; the candidate
// sets they accept are unchanged.
// ---------------------------------------------------------------------------
template <bool SCATTER>
__global__ void k_elem_bin(const Params P, const DevPtrs d, uint32_t total) {
    for (uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x; gid < total; gid += gridDim.x * blockDim.x) {
        float3 lo, hi;
        if (!SCATTER) {
            elem_tight(P, d, gid, lo, hi);
            d.elemBox[2 * gid] = mk4(lo, 0.0f);
            d.elemBox[2 * gid + 1] = mk4(hi, 0.0f);
        }
        elem_bounds(P, d, gid, lo, hi);
        if (!finite3(lo) || !finite3(hi)) {
            if (!SCATTER) {
                atomicAdd(&d.counters->datInvalidAnchor, 1u);
                atomicAdd(&d.counters->datNonfinite, 1u);
            }
            continue;
        }
        const I3 c0 = cell_of(lo, P.elemCellSize), raw = cell_of(hi, P.elemCellSize);
        if (!SCATTER && (raw.x - c0.x > 3 || raw.y - c0.y > 3 || raw.z - c0.z > 3))
            atomicAdd(&d.counters->datGridOverflow, 1u);
        const I3 c1 = imin3(raw, iadd(c0, 3));
        // the range the candidate tests compare against (they computed it
        // from the same padded box, to the same bits)
        if (!SCATTER)
            d.elemRange[gid] = make_int4(c0.x, c0.y, c0.z, (c1.x - c0.x) | ((c1.y - c0.y) << 2) | ((c1.z - c0.z) << 4));
        const bool tri = gid < P.numTris;
        const uint32_t entry = tri ? gid : gid - P.numTris;
        const uint32_t half = tri ? 0u : P.elemHashSize;
        uint32_t seen[64];
        uint32_t ns = 0;
        for (int z = c0.z; z <= c1.z; z++)
            for (int y = c0.y; y <= c1.y; y++)
                for (int x = c0.x; x <= c1.x; x++) {
                    const uint32_t h = elem_hash(I3{x, y, z}, P.elemHashSize);
                    bool dup = false;
                    for (uint32_t i = 0; i < ns; i++) dup = dup || seen[i] == h;
                    if (dup) continue;
                    seen[ns++] = h;
                    if (SCATTER) d.elemCells[atomicAdd(&d.elemCursor[half + h], 1u)] = entry;
                    else atomicAdd(&d.elemCellCount[half + h], 1u);
                }
    }
}

// ---------------------------------------------------------------------------
// Pair streams (27_planar_dat.metal:35-206): one warp per query owner —
// owners [0, numParticles) are V-T queries of surface particles, the rest
// E-E queries of edges.
// ---------------------------------------------------------------------------
// The reference's V-T acceptance is a conjunction of pure predicates
// (27_planar_dat.metal:75-101); they are evaluated cheapest first, after a
// conservative box test that every accepted pair passes.
// The conjunction is split in two: the cheap predicates (index, cell range,
// box prefilter) and the rest (topology, exact distance, exclusions), so the
// pair kernel can run the second part only on the candidates that pass the
// first, packed onto full warps.
__device__ __forceinline__ bool vt_cheap(const Params& P, const DevPtrs& d, float3 p, I3 cell, uint32_t entry) {
    if (entry >= P.numTris) return false;
    // the triangle's binned cell range (from its padded box) must hold the
    // query cell; then the box prefilter (independent predicates, so the
    // cheaper one goes first)
    const int4 rg = d.elemRange[entry];
    const I3 tc0{rg.x, rg.y, rg.z};
    const I3 tc1{rg.x + (rg.w & 3), rg.y + ((rg.w >> 2) & 3), rg.z + ((rg.w >> 4) & 3)};
    if (cell.x < tc0.x || cell.y < tc0.y || cell.z < tc0.z || cell.x > tc1.x || cell.y > tc1.y || cell.z > tc1.z)
        return false;
    const float4 bl = d.elemBox[2 * entry], bh = d.elemBox[2 * entry + 1];
    const float r = prefilter_reach(P);
    return !(p.x < bl.x - r || p.y < bl.y - r || p.z < bl.z - r || p.x > bh.x + r || p.y > bh.y + r || p.z > bh.z + r);
}
__device__ __forceinline__ bool vt_full(const Params& P, const DevPtrs& d, uint32_t v, float3 p, uint32_t ns,
                                        uint32_t ne, uint32_t entry, float query2) {
    const uint4 t = d.tris[entry];
    if (t.x == v || t.y == v || t.z == v) return false;
    float3 bary;
    const float3 q = closest_pt_triangle(p, xyz(d.posLin[t.x]), xyz(d.posLin[t.y]), xyz(d.posLin[t.z]), bary);
    const float3 dd = p - q;
    if (dot(dd, dd) > query2) return false;
    const uint32_t group = d.clothGroup[v];
    const bool same = group != 0u && d.clothGroup[t.x] == group && d.clothGroup[t.y] == group &&
                      d.clothGroup[t.z] == group;
    if (same && d.selfCollision[v] == 0u) return false;
    if (same && (nbr_contains(d.nbrList, ns, ne, t.x) || nbr_contains(d.nbrList, ns, ne, t.y) ||
                 nbr_contains(d.nbrList, ns, ne, t.z)))
        return false;
    return true;
}

// E-E acceptance (27_planar_dat.metal:155-204), cheapest predicates first
// after a conservative box-separation test.
__device__ __forceinline__ bool ee_cheap(const Params& P, const DevPtrs& d, uint32_t gid, float3 alo, float3 ahi,
                                         I3 ac0, I3 ac1, I3 cell, uint32_t other) {
    if (other <= gid || other >= P.numEdges) return false;
    // the pair is taken in the first cell the two binned ranges share (each
    // range from the element's padded box, stored by the binning pass); this
    // rejects the pair in every other shared cell before the box prefilter
    // (independent predicates, so the cheaper one goes first)
    const int4 rg = d.elemRange[P.numTris + other];
    const I3 bc0{rg.x, rg.y, rg.z};
    const I3 bc1{rg.x + (rg.w & 3), rg.y + ((rg.w >> 2) & 3), rg.z + ((rg.w >> 4) & 3)};
    const I3 o0 = imax3(ac0, bc0), o1 = imin3(ac1, bc1);
    if (o0.x > o1.x || o0.y > o1.y || o0.z > o1.z) return false;
    if (cell.x != o0.x || cell.y != o0.y || cell.z != o0.z) return false;
    const float4 bl = d.elemBox[2 * (P.numTris + other)], bh = d.elemBox[2 * (P.numTris + other) + 1];
    const float r = prefilter_reach(P);
    return !(bl.x - ahi.x > r || bl.y - ahi.y > r || bl.z - ahi.z > r || alo.x - bh.x > r || alo.y - bh.y > r ||
             alo.z - bh.z > r);
}
__device__ __forceinline__ bool ee_full(const Params& P, const DevPtrs& d, uint32_t gid, uint2 a, float3 a0,
                                        float3 a1, uint32_t other, float query2, uint32_t& flags) {
    const uint2 b = d.edges[other];
    if (b.x == a.x || b.x == a.y || b.y == a.x || b.y == a.y) return false;
    float sb, tb;
    const float3 b0 = xyz(d.posLin[b.x]), b1 = xyz(d.posLin[b.y]);
    closest_seg_seg(a0, a1, b0, b1, sb, tb);
    const float3 ca = a0 + (a1 - a0) * sb, cb = b0 + (b1 - b0) * tb;
    const float3 dd = ca - cb;
    if (dot(dd, dd) > query2) return false;
    const uint32_t group = d.clothGroup[a.x];
    const bool same = group != 0u && d.clothGroup[a.y] == group && d.clothGroup[b.x] == group &&
                      d.clothGroup[b.y] == group;
    if (same && d.selfCollision[a.x] == 0u) return false;
    if (same) {
        const uint32_t ns0 = d.nbrStart[a.x], ne0 = ns0 + d.nbrCount[a.x];
        const uint32_t ns1 = d.nbrStart[a.y], ne1 = ns1 + d.nbrCount[a.y];
        if (nbr_contains(d.nbrList, ns0, ne0, b.x) || nbr_contains(d.nbrList, ns0, ne0, b.y) ||
            nbr_contains(d.nbrList, ns1, ne1, b.x) || nbr_contains(d.nbrList, ns1, ne1, b.y))
            return false;
    }
    flags = DAT_PAIR_TRUNCATE;
    if ((gid < P.numSurfaceEdges && other < P.numSurfaceEdges) || (same && d.selfCollision[a.x] != 0u))
        flags |= DAT_PAIR_CONTACT;
    return true;
}

// Insertion sort of one owner's pair segment by the `other` index.
__device__ void sort_segment(uint4* seg, uint32_t n) {
    for (uint32_t i = 1; i < n; i++) {
        const uint4 v = seg[i];
        uint32_t j = i;
        while (j > 0 && seg[j - 1].z > v.z) { seg[j] = seg[j - 1]; j--; }
        seg[j] = v;
    }
}

// Pairs per owner kept from the counting pass (other, flags): an owner with
// at most this many is written from them instead of a second grid scan.
constexpr uint32_t kDatCache = 16;

// Eight blocks per SM (at most 64 registers, no spills): the pair scan is
// latency bound and gains from the extra warps (cloth frame 4.93 -> 4.66 ms).
// A warp's candidates first pass the cheap predicates on every lane; the
// survivors queue up in shared memory and the rest of the test runs on 32
// of them at a time, so the expensive part (exact distance, exclusions)
// keeps every lane busy instead of the few whose candidate survived.  The
// accepted set is the same; its discovery order differs, and each owner's
// pairs are sorted by `other` after the emitting pass.
template <bool EMIT>
__global__ void __launch_bounds__(128, 8) k_dat_pairs(const Params P, const DevPtrs d, uint32_t owners) {
    __shared__ uint32_t survivors[4][64];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const float query2 = P.queryRadius * P.queryRadius;
    const uint32_t below = (1u << lane) - 1u;
    uint32_t* q = survivors[threadIdx.x >> 5];
    for (uint32_t owner = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; owner < owners; owner += warps) {
        uint32_t count = 0, qn = 0;                           // qn: queued survivors (warp-uniform)
        const uint32_t base = EMIT ? d.datOwnerStart[owner] : 0u;
        uint2* cache = d.datCache + (size_t)owner * kDatCache;
        // one full-test result per lane: count it, cache the first ones, emit
        auto record = [&](bool pass, uint32_t kind, uint32_t id, uint32_t entry, uint32_t flags) {
            const uint32_t ballot = __ballot_sync(0xffffffffu, pass);
            if (EMIT && pass) {
                const uint32_t slot = base + count + __popc(ballot & below);
                if (slot < P.maxDatPairs) d.datPairs[slot] = make_uint4(kind, id, entry, flags);
            }
            if (!EMIT && pass && count + __popc(ballot & below) < kDatCache)
                cache[count + __popc(ballot & below)] = make_uint2(entry, flags);
            count += __popc(ballot);
        };
        // queue this lane's survivor of the cheap predicates
        auto enqueue = [&](bool cand, uint32_t entry) {
            const uint32_t ballot = __ballot_sync(0xffffffffu, cand);
            if (cand) q[qn + __popc(ballot & below)] = entry;
            qn += __popc(ballot);
            __syncwarp();
        };
        // take up to 32 queued entries (one per lane) and move the rest to
        // the head of the queue
        auto dequeue = [&](uint32_t& entry) -> bool {
            const uint32_t take = qn < 32u ? qn : 32u;
            const bool mine = lane < take;
            if (mine) entry = q[lane];
            const uint32_t rest = qn - take;
            uint32_t moved = 0;
            if (lane < rest) moved = q[take + lane];
            __syncwarp();
            if (lane < rest) q[lane] = moved;
            __syncwarp();
            qn = rest;
            return mine;
        };
        if (EMIT) {
            const uint32_t n = d.datOwnerCount[owner];
            if (n <= kDatCache) {
                const bool vt = owner < P.numParticles;
                const uint32_t id = vt ? d.particleIdx[owner] : owner - P.numParticles;
                if (lane < n && base + lane < P.maxDatPairs) {
                    const uint2 c = cache[lane];
                    d.datPairs[base + lane] = make_uint4(vt ? DAT_PAIR_VT : DAT_PAIR_EE, id, c.x, c.y);
                }
                __syncwarp();
                if (lane == 0 && n > 1) {
                    const uint32_t end = min(base + n, P.maxDatPairs);
                    if (end > base) sort_segment(d.datPairs + base, end - base);
                }
                continue;
            }
        }
        if (owner < P.numParticles) {
            const uint32_t v = d.particleIdx[owner];
            const float3 p = xyz(d.posLin[v]);
            if (!finite3(p)) {
                if (!EMIT && lane == 0) {
                    atomicAdd(&d.counters->datInvalidAnchor, 1u);
                    atomicAdd(&d.counters->datNonfinite, 1u);
                }
                if (!EMIT && lane == 0) d.datOwnerCount[owner] = 0;
                continue;
            }
            const I3 cell = cell_of(p, P.elemCellSize);
            const uint32_t h = elem_hash(cell, P.elemHashSize);           // triangle half
            const uint32_t s0 = d.elemCellStart[h], e0 = s0 + d.elemCellCount[h];
            const uint32_t ns = d.nbrStart[v], ne = ns + d.nbrCount[v];
            auto drain = [&](bool all) {
                while (qn >= 32u || (all && qn > 0u)) {
                    uint32_t entry = 0;
                    const bool pass = dequeue(entry) && vt_full(P, d, v, p, ns, ne, entry, query2);
                    record(pass, DAT_PAIR_VT, v, entry, DAT_PAIR_TRUNCATE | DAT_PAIR_CONTACT);
                }
            };
            for (uint32_t k0 = s0; k0 < e0; k0 += 32) {
                const uint32_t k = k0 + lane;
                uint32_t entry = 0;
                bool cand = false;
                if (k < e0) {
                    entry = d.elemCells[k];
                    cand = vt_cheap(P, d, p, cell, entry);
                }
                enqueue(cand, entry);
                drain(false);
            }
            drain(true);
        } else {
            const uint32_t gid = owner - P.numParticles;
            const uint2 a = d.edges[gid];
            const float3 a0 = xyz(d.posLin[a.x]), a1 = xyz(d.posLin[a.y]);
            if (!finite3(a0) || !finite3(a1)) {
                if (!EMIT && lane == 0) {
                    atomicAdd(&d.counters->datInvalidAnchor, 1u);
                    atomicAdd(&d.counters->datNonfinite, 1u);
                    d.datOwnerCount[owner] = 0;
                }
                continue;
            }
            const I3 ac0 = cell_of(vmin(a0, a1), P.elemCellSize);
            const I3 raw = cell_of(vmax(a0, a1), P.elemCellSize);
            if (!EMIT && lane == 0 && (raw.x - ac0.x > 3 || raw.y - ac0.y > 3 || raw.z - ac0.z > 3))
                atomicAdd(&d.counters->datGridOverflow, 1u);
            const I3 ac1 = imin3(raw, iadd(ac0, 3));
            const float3 alo = vmin(a0, a1), ahi = vmax(a0, a1);
            auto drain = [&](bool all) {
                while (qn >= 32u || (all && qn > 0u)) {
                    uint32_t entry = 0, flags = 0;
                    const bool pass = dequeue(entry) && ee_full(P, d, gid, a, a0, a1, entry, query2, flags);
                    record(pass, DAT_PAIR_EE, gid, entry, flags);
                }
            };
            for (int z = ac0.z; z <= ac1.z; z++)
                for (int y = ac0.y; y <= ac1.y; y++)
                    for (int x = ac0.x; x <= ac1.x; x++) {
                        const I3 cell{x, y, z};
                        const uint32_t h = P.elemHashSize + elem_hash(cell, P.elemHashSize);   // edge half
                        const uint32_t s0 = d.elemCellStart[h], e0 = s0 + d.elemCellCount[h];
                        for (uint32_t k0 = s0; k0 < e0; k0 += 32) {
                            const uint32_t k = k0 + lane;
                            uint32_t entry = 0;
                            bool cand = false;
                            if (k < e0) {
                                entry = d.elemCells[k];
                                cand = ee_cheap(P, d, gid, alo, ahi, ac0, ac1, cell, entry);
                            }
                            enqueue(cand, entry);
                            drain(false);
                        }
                    }
            drain(true);
        }
        if (!EMIT) {
            if (lane == 0) d.datOwnerCount[owner] = count;
        } else {
            __syncwarp();
            if (lane == 0 && count > 1) {
                const uint32_t end = min(base + count, P.maxDatPairs);
                if (end > base) sort_segment(d.datPairs + base, end - base);
            }
        }
    }
}

// Totals of the pair stream (dat_finalize_pairs, 27_planar_dat.metal:208-228).
__global__ void k_dat_pair_totals(const Params P, const DevPtrs d, uint32_t owners) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Counters* c = d.counters;
    const uint32_t total = owners ? d.datOwnerStart[owners - 1] + d.datOwnerCount[owners - 1] : 0u;
    const uint32_t vt = P.numParticles < owners ? d.datOwnerStart[P.numParticles] : total;
    c->datRaw = total;
    c->datVT = vt;
    c->datEE = total - vt;
    c->datStored = min(total, P.maxDatPairs);
    c->datPairsPeak = max(c->datPairsPeak, total);
    c->datVTPeak = max(c->datVTPeak, vt);
    c->datEEPeak = max(c->datEEPeak, total - vt);
}

// ---------------------------------------------------------------------------
// Rigid feature points vs triangles (25_cloth.metal:942-1142): one thread per
// triangle, at most four records.  Bodies are reached through their
// collider's owner; the grid sweep visits each distinct bucket once.
// ---------------------------------------------------------------------------
// WARP (many global colliders): one warp per triangle, lane 0 takes the
// candidates in the serial order and the warp pre-tests 32 globals at a time with the reach
// test that opens the body test, so lane 0 visits only globals that can pass
// it.  Otherwise one thread per triangle.
// This search runs once per frame: it counts each triangle's records and
// keeps their (body, feature) in the triangle's RT_MAX_PER_TRI slots of
// rtCand; k_rt_write writes the records at the scanned offsets.
template <bool WARP>
__global__ void __launch_bounds__(128, 6) k_rt_emit(const Params P, const DevPtrs d) {
    const uint32_t lane = WARP ? (threadIdx.x & 31u) : 0u;
    const uint32_t step = WARP ? (gridDim.x * blockDim.x) >> 5 : gridDim.x * blockDim.x;
    const uint32_t first = WARP ? (blockIdx.x * blockDim.x + threadIdx.x) >> 5 : blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t gid = first; gid < P.numTris; gid += step) {
        const uint4 tid = d.tris[gid];
        const float3 a = xyz(d.posLin[tid.x]), b = xyz(d.posLin[tid.y]), c = xyz(d.posLin[tid.z]);
        const float3 m = (a + b + c) / 3.0f;
        const float rt_ = mx(fabsf(d.shape[tid.x].w), mx(fabsf(d.shape[tid.y].w), fabsf(d.shape[tid.z].w)));
        const float rT = mx(dist3(m, a), mx(dist3(m, b), dist3(m, c))) + rt_;
        float3 triN = cross(b - a, c - a);
        const float tnLen = len3(triN);
        uint32_t emitted = 0;
        if (!(tnLen < 1e-12f)) {
            triN = triN / tnLen;
            const float3 velT = (xyz(d.velLin[tid.x]) + xyz(d.velLin[tid.y]) + xyz(d.velLin[tid.z])) / 3.0f;
            auto test_body = [&](uint32_t o) {
                const float4 sh = d.shape[o];
                const float rb = fabsf(sh.w);
                const float4 po4 = d.posLin[o];
                const float3 po = xyz(po4);
                const float4 qo = d.posAng[o];
                const uint32_t sk = d.bodyShape[o];
                bool nearO = dist3(po, m) <= rT + rb + P.collisionMargin;
                if (nearO && sk == AVBD_SHAPE_BOX) {
                    const float3 lm = q_rotate(q_conj(qo), m - po);
                    const float3 dq2 = mx3(abs3(lm) - xyz(sh) * 0.5f, s3(0.0f));
                    nearO = len3(dq2) <= rT + P.collisionMargin + 0.05f;
                }
                if (!nearO) return;
                // excluded pairs emit nothing: the test runs before the first
                // record it would prevent (cheaper than before the features)
                int excluded = -1;
                auto is_excluded = [&]() {
                    if (excluded < 0)
                        excluded = (pair_excluded(d, P.numExclusions, min(o, tid.x), max(o, tid.x)) ||
                                    pair_excluded(d, P.numExclusions, min(o, tid.y), max(o, tid.y)) ||
                                    pair_excluded(d, P.numExclusions, min(o, tid.z), max(o, tid.z)))
                                       ? 1
                                       : 0;
                    return excluded == 1;
                };
                float3 fw[4];
                float fr[4];
                uint32_t fid[4];
                int nf = 0;
                if (sk == AVBD_SHAPE_SPHERE) {
                    fw[0] = po; fr[0] = sh.x * 0.5f; fid[0] = 8; nf = 1;
                } else if (sk == AVBD_SHAPE_CAPSULE) {
                    // three spheres along the axis (a torus has no feature
                    // points: 25_cloth.metal:957-971)
                    const float half_ = sh.x * 0.5f, r = sh.y;
                    const float3 ax = q_rotate(qo, mk3(0, 0, 1));
                    for (int i = -1; i <= 1; i++) {
                        const float3 w = po + ax * (half_ * (float)i);
                        if (dist3(w, m) > rT + r + 4.0f * P.collisionMargin) continue;
                        fw[nf] = w; fr[nf] = r; fid[nf] = (uint32_t)(9 + i + 1); nf++;
                    }
                } else if (sk == AVBD_SHAPE_BOX) {
                    const float3 h3 = xyz(sh) * 0.5f;
                    for (uint32_t i = 0; i < 8; i++) {
                        const float3 local = mk3((i & 1) ? h3.x : -h3.x, (i & 2) ? h3.y : -h3.y, (i & 4) ? h3.z : -h3.z);
                        const float3 w = xform(po, qo, local);
                        if (dist3(w, m) > rT + 4.0f * P.collisionMargin) continue;
                        if (nf < 4) { fw[nf] = w; fr[nf] = 0.0f; fid[nf] = i; nf++; }
                    }
                }
                for (int fi = 0; fi < nf && emitted < RT_MAX_PER_TRI; fi++) {
                    float3 bary;
                    const float3 q = closest_pt_triangle(fw[fi], a, b, c, bary);
                    const float3 dv = fw[fi] - q;
                    const float dist = len3(dv);
                    const float hSum = rt_ + fr[fi];
                    const float inflate = mn(len3(xyz(d.velLin[o]) - velT) * P.dt, 0.5f * rT);
                    if (dist - hSum > P.elemMargin + inflate) continue;
                    float minMass = po4.w > 0.0f ? po4.w : FLT_BIG_;
                    const float mA = d.posLin[tid.x].w, mB = d.posLin[tid.y].w, mC = d.posLin[tid.z].w;
                    if (mA > 0.0f) minMass = mn(minMass, mA);
                    if (mB > 0.0f) minMass = mn(minMass, mB);
                    if (mC > 0.0f) minMass = mn(minMass, mC);
                    if (minMass == FLT_BIG_) continue;
                    if (is_excluded()) return;
                    d.rtCand[(size_t)gid * RT_MAX_PER_TRI + emitted] = make_uint2(o, fid[fi]);
                    emitted++;
                }
            };
            if (lane == 0) {
            if (P.numHashedRigid > 0 && P.numHashedRigid <= 8) {
                for (uint32_t ri = 0; ri < P.numHashed && emitted < RT_MAX_PER_TRI; ri++) {
                    const uint32_t col = d.hashedIdx[ri];
                    if (d.colShape[col].w < 0.0f) continue;
                    test_body(d.colOwner[col]);
                }
            } else if (P.numHashedRigid > 0) {
                const int R = min(4, max(1, (int)ceilf((rT + 0.5f * P.cellSize) / P.cellSize)));
                int cx, cy, cz;
                cell_coord(m, P.cellSize, cx, cy, cz);
                uint32_t seen[729];
                uint32_t ns = 0;
                for (int dz = -R; dz <= R && emitted < RT_MAX_PER_TRI; dz++)
                    for (int dy = -R; dy <= R && emitted < RT_MAX_PER_TRI; dy++)
                        for (int dx = -R; dx <= R && emitted < RT_MAX_PER_TRI; dx++) {
                            const uint32_t h = cell_hash(cx + dx, cy + dy, cz + dz, 0u, P.gridHashSize);
                            bool dup = false;
                            for (uint32_t i = 0; i < ns; i++) dup = dup || seen[i] == h;
                            if (dup) continue;
                            seen[ns++] = h;
                            // the bucket's rigid colliders, in bucket order
                            const uint32_t s0 = d.rigidStart[h], e0 = s0 + d.cellRigid[h];
                            for (uint32_t k = s0; k < e0 && emitted < RT_MAX_PER_TRI; k++) {
                                const uint32_t o = d.colOwner[d.rigidCells[k]];
                                if (d.shape[o].w < 0.0f) continue;
                                test_body(o);
                            }
                        }
            }
            }
            if (WARP) {
                emitted = __shfl_sync(0xffffffffu, emitted, 0);
                const uint32_t chunks = (P.numGlobals + 31u) / 32u;
                for (uint32_t c0 = 0; c0 < chunks && emitted < RT_MAX_PER_TRI; c0 += 32) {
                    // a chunk whose bodies all lie beyond the reach test is
                    // skipped; lane l tests chunk c0 + l, so a warp culls 32
                    // chunks with one load instead of one chunk per load
                    bool keep = false;
                    if (c0 + lane < chunks) {
                        const float4* box = d.globalChunk + 4 * (size_t)(c0 + lane);
                        keep = !ball_misses_box(m, rT + P.collisionMargin, box[2], box[3]);
                    }
                    uint32_t live = __ballot_sync(0xffffffffu, keep);
                    while (live && emitted < RT_MAX_PER_TRI) {
                        const uint32_t gb = (c0 + (uint32_t)(__ffs(live) - 1)) * 32u;
                        live &= live - 1u;
                        const uint32_t g = gb + lane;
                        bool cand = false;
                        if (g < P.numGlobals) {
                            // the owner's reach test (its bounding sphere, then a
                            // box's padded extent) on the global's record (pose
                            // and shape, written this frame by the chunk pass):
                            // one load level instead of three
                            const float4 r0 = d.globalRec[3 * (size_t)g];
                            const float3 po = xyz(r0);
                            cand = r0.w >= 0.0f && dist3(po, m) <= rT + fabsf(r0.w) + P.collisionMargin;
                            if (cand) {
                                const float4 r2 = d.globalRec[3 * (size_t)g + 2];
                                if (__float_as_uint(r2.w) == AVBD_SHAPE_BOX) {
                                    const float3 lm = q_rotate(q_conj(d.globalRec[3 * (size_t)g + 1]), m - po);
                                    const float3 dq2 = mx3(abs3(lm) - xyz(r2) * 0.5f, s3(0.0f));
                                    cand = len3(dq2) <= rT + P.collisionMargin + 0.05f;
                                }
                            }
                        }
                        uint32_t ballot = __ballot_sync(0xffffffffu, cand);
                        if (lane == 0) {
                            while (ballot && emitted < RT_MAX_PER_TRI) {
                                const uint32_t j = __ffs(ballot) - 1;
                                ballot &= ballot - 1;
                                test_body(d.globalOwner[gb + j]);
                            }
                        }
                        emitted = __shfl_sync(0xffffffffu, emitted, 0);
                    }
                }
            } else {
                for (uint32_t g = 0; g < P.numGlobals && emitted < RT_MAX_PER_TRI; g++) {
                    const uint32_t o = d.colOwner[d.globalIdx[g]];
                    if (d.shape[o].w < 0.0f) continue;
                    test_body(o);
                }
            }
        }
        if (lane == 0) d.rtCount[gid] = emitted;
    }
}

// A record's feature point from its id (the ids k_rt_emit gives: box corners
// 0-7, sphere centre 8, capsule axis spheres 9-11), by the expressions the
// search evaluates, so the point is the same float.
__device__ __forceinline__ void rt_feature(float4 sh, float3 po, float4 qo, uint32_t sk, uint32_t f, float3& w,
                                           float& r) {
    if (sk == AVBD_SHAPE_SPHERE) {
        w = po; r = sh.x * 0.5f;
    } else if (sk == AVBD_SHAPE_CAPSULE) {
        const float half_ = sh.x * 0.5f;
        const float3 ax = q_rotate(qo, mk3(0, 0, 1));
        w = po + ax * (half_ * (float)((int)f - 10)); r = sh.y;
    } else {
        const float3 h3 = xyz(sh) * 0.5f;
        const float3 local = mk3((f & 1) ? h3.x : -h3.x, (f & 2) ? h3.y : -h3.y, (f & 4) ? h3.z : -h3.z);
        w = xform(po, qo, local); r = 0.0f;
    }
}

// One thread per triangle writes the records k_rt_emit found, in its order,
// from the triangle's scanned offset (25_cloth.metal:1080-1142 is the record).
__global__ void __launch_bounds__(128) k_rt_write(const Params P, const DevPtrs d) {
    for (uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x; gid < P.numTris; gid += gridDim.x * blockDim.x) {
        const uint32_t count = d.rtCount[gid];
        if (count == 0) continue;
        const uint4 tid = d.tris[gid];
        const float3 a = xyz(d.posLin[tid.x]), b = xyz(d.posLin[tid.y]), c = xyz(d.posLin[tid.z]);
        const float rt_ = mx(fabsf(d.shape[tid.x].w), mx(fabsf(d.shape[tid.y].w), fabsf(d.shape[tid.z].w)));
        float3 triN = cross(b - a, c - a);
        triN = triN / len3(triN);
        const uint32_t base = d.rtStart[gid];
        for (uint32_t k = 0; k < count; k++) {
            const uint2 cf = d.rtCand[(size_t)gid * RT_MAX_PER_TRI + k];
            const uint32_t o = cf.x;
            const float4 sh = d.shape[o];
            const float4 po4 = d.posLin[o];
            const float3 po = xyz(po4);
            const float4 qo = d.posAng[o];
            const uint32_t sk = d.bodyShape[o];
            float3 w;
            float fr;
            rt_feature(sh, po, qo, sk, cf.y, w, fr);
            float3 bary;
            const float3 q = closest_pt_triangle(w, a, b, c, bary);
            const float3 dv = w - q;
            const float dist = len3(dv);
            const float hSum = rt_ + fr;
            float minMass = po4.w > 0.0f ? po4.w : FLT_BIG_;
            const float mA = d.posLin[tid.x].w, mB = d.posLin[tid.y].w, mC = d.posLin[tid.z].w;
            if (mA > 0.0f) minMass = mn(minMass, mA);
            if (mB > 0.0f) minMass = mn(minMass, mB);
            if (mC > 0.0f) minMass = mn(minMass, mC);
            const float side = dot(dv, triN) >= 0.0f ? 1.0f : -1.0f;
            const uint32_t keyA = (SC_RT << 28) | o;
            const uint32_t keyB = gid * 16u + cf.y;
            const float proposed = dot(po - q, triN) >= 0.0f ? 1.0f : -1.0f;
            const bool interior = bary.x > 0.02f && bary.y > 0.02f && bary.z > 0.02f;
            const float sMem = interior ? soft_prev_side(P, d, keyA, keyB, proposed) : proposed;
            float3 n;
            float g;
            if (dist > 1e-7f && side == sMem) { n = dv / dist; g = dist; }
            else { n = triN * sMem; g = -dist; }
            const float fricT = (d.props[tid.x].w + d.props[tid.y].w + d.props[tid.z].w) / 3.0f;
            const float friction = sqrtf(mx(d.props[o].w * fricT, 0.0f));
            const bool roundA = sk != AVBD_SHAPE_BOX;
            const float3 anchor = roundA ? (w - po) : q_rotate(q_conj(qo), w - po);
            soft_write(P, d, base + k, make_uint4(o, tid.x, tid.y, tid.z), make_float4(1.0f, -bary.x, -bary.y, -bary.z),
                       n, friction, anchor, g - hSum + P.elemMargin, hSum - P.elemMargin, soft_lambda_cap(P, minMass),
                       minMass, SC_RT, true, roundA, sMem < 0.0f, keyA, keyB);
        }
    }
}

__global__ void k_rt_totals(const Params P, const DevPtrs d) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const uint32_t n = P.numTris;
    d.counters->numSoftRT = n ? d.rtStart[n - 1] + d.rtCount[n - 1] : 0u;
}

// ---------------------------------------------------------------------------
// Element contacts at the accepted pose (dat_emit_contacts,
// 27_planar_dat.metal:344-510): one warp per query owner walks its pair
// segment; records follow pair order after the rigid-triangle block.
// ---------------------------------------------------------------------------
template <bool EMIT>
__device__ bool dat_contact(const Params& P, const DevPtrs& d, uint4 pair, uint32_t slot) {
    if ((pair.w & DAT_PAIR_CONTACT) == 0u) return false;
    if (pair.x == DAT_PAIR_VT) {
        const uint32_t v = pair.y, ti = pair.z;
        if (ti >= P.numTris) return false;
        const uint4 t = d.tris[ti];
        const float3 p = xyz(d.posLin[v]);
        const float3 a = xyz(d.posLin[t.x]), b = xyz(d.posLin[t.y]), c = xyz(d.posLin[t.z]);
        float3 bary;
        const float3 q = closest_pt_triangle(p, a, b, c, bary);
        const float3 dv = p - q;
        const float dist2 = dot(dv, dv);
        const float rv = fabsf(d.shape[v].w);
        const float rt = mx(fabsf(d.shape[t.x].w), mx(fabsf(d.shape[t.y].w), fabsf(d.shape[t.z].w)));
        const float hSum = rv + rt;
        const float3 velT = (xyz(d.velLin[t.x]) + xyz(d.velLin[t.y]) + xyz(d.velLin[t.z])) / 3.0f;
        const float inflate = mn(len3(xyz(d.velLin[v]) - velT) * P.dt, 0.3f * P.surfaceCellSize);
        const float detect = mn(hSum + P.elemMargin + inflate, P.queryRadius);
        if (dist2 > detect * detect) return false;
        const float dist = sqrtf(dist2);
        float3 triN = cross(b - a, c - a);
        const float nl = len3(triN);
        if (nl < DAT_GEOMETRY_EPS) return false;
        triN = triN / nl;
        float minMass = d.posLin[v].w > 0.0f ? d.posLin[v].w : FLT_BIG_;
        const uint32_t ids[4] = {v, t.x, t.y, t.z};
        for (int j = 1; j < 4; j++) {
            const float mm = d.posLin[ids[j]].w;
            if (mm > 0.0f) minMass = mn(minMass, mm);
        }
        if (minMass == FLT_BIG_) return false;
        if (EMIT) {
            const float side = dot(dv, triN) >= 0.0f ? 1.0f : -1.0f;
            const uint32_t keyA = (SC_VT << 28) | v, keyB = ti;
            const bool interior = bary.x > 0.02f && bary.y > 0.02f && bary.z > 0.02f;
            const float remembered = interior ? soft_prev_side(P, d, keyA, keyB, side) : side;
            float3 n;
            float gap;
            if (dist > 1.0e-7f && side == remembered) { n = dv / dist; gap = dist; }
            else { n = triN * remembered; gap = -dist; }
            const float fricT = d.props[t.x].w * bary.x + d.props[t.y].w * bary.y + d.props[t.z].w * bary.z;
            const float friction = sqrtf(mx(d.props[v].w * fricT, 0.0f));
            const float3 dq = (p - xyz(d.initLin[v])) - (a - xyz(d.initLin[t.x])) * bary.x -
                              (b - xyz(d.initLin[t.y])) * bary.y - (c - xyz(d.initLin[t.z])) * bary.z;
            const float Cdetect = gap - hSum + P.elemMargin;
            const float C0n = Cdetect - dot(n, dq);
            soft_write(P, d, slot, make_uint4(v, t.x, t.y, t.z), make_float4(1.0f, -bary.x, -bary.y, -bary.z), n,
                       friction, s3(0), C0n, hSum - P.elemMargin, soft_lambda_cap(P, minMass), minMass, SC_VT, false,
                       false, remembered < 0.0f, keyA, keyB);
        }
        return true;
    }
    const uint32_t ea = pair.y, eb = pair.z;
    if (ea >= P.numEdges || eb >= P.numEdges) return false;
    const uint2 A = d.edges[ea], B = d.edges[eb];
    const float3 a0 = xyz(d.posLin[A.x]), a1 = xyz(d.posLin[A.y]);
    const float3 b0 = xyz(d.posLin[B.x]), b1 = xyz(d.posLin[B.y]);
    float s, t;
    closest_seg_seg(a0, a1, b0, b1, s, t);
    if (s < EE_INTERIOR_EPS || s > 1.0f - EE_INTERIOR_EPS || t < EE_INTERIOR_EPS || t > 1.0f - EE_INTERIOR_EPS)
        return false;
    const float3 ca = a0 + (a1 - a0) * s, cb = b0 + (b1 - b0) * t;
    const float3 dv = ca - cb;
    const float dist = len3(dv);
    const float rA = mx(fabsf(d.shape[A.x].w), fabsf(d.shape[A.y].w));
    const float rB = mx(fabsf(d.shape[B.x].w), fabsf(d.shape[B.y].w));
    const float hSum = rA + rB;
    const float3 va = (xyz(d.velLin[A.x]) + xyz(d.velLin[A.y])) * 0.5f;
    const float3 vb = (xyz(d.velLin[B.x]) + xyz(d.velLin[B.y])) * 0.5f;
    const float inflate = mn(len3(va - vb) * P.dt, 0.3f * P.surfaceCellSize);
    const float detect = mn(hSum + P.elemMargin + inflate, P.queryRadius);
    if (dist > detect) return false;
    const uint32_t keyA = (SC_EE << 28) | ea, keyB = eb;
    const int previous = soft_map_find(P, d, keyA, keyB);
    float3 n;
    float gap = dist;
    if (finite_bits(dist) && dist >= 1.0e-7f) {
        const float3 nGeo = dv / dist;
        n = nGeo;
        if (previous >= 0 && dot(nGeo, xyz(d.prevSoft[previous].normal)) < 0.0f) { n = -nGeo; gap = -dist; }
    } else if (previous >= 0 && finite3(xyz(d.prevSoft[previous].normal))) {
        n = xyz(d.prevSoft[previous].normal);
        gap = 0.0f;
    } else {
        // datEEFallbackNormal (27_planar_dat.metal:304-338)
        const float3 rel = va - vb;
        const float3 ua = a1 - a0, ub = b1 - b0;
        const float3 rawN = cross(ua, ub);
        const float mag = len3(rawN);
        bool valid = true;
        if (finite_bits(mag) && mag >= DAT_GEOMETRY_EPS) {
            n = rawN / mag;
        } else {
            const float la = len3(ua), lb = len3(ub);
            float3 u = la >= lb ? ua : ub;
            const float ul = mx(la, lb);
            if (!finite_bits(ul) || ul < DAT_GEOMETRY_EPS) {
                valid = false;
            } else {
                u = u / ul;
                float3 perp = rel - u * dot(u, rel);
                float pl = len3(perp);
                if (!finite_bits(pl) || pl < DAT_GEOMETRY_EPS) {
                    const float3 axis = fabsf(u.x) < 0.7f ? mk3(1, 0, 0) : mk3(0, 1, 0);
                    perp = cross(u, axis);
                    pl = len3(perp);
                }
                if (!finite_bits(pl) || pl < DAT_GEOMETRY_EPS) valid = false;
                else n = perp / pl;
            }
        }
        if (valid) {
            if (dot(n, rel) > 0.0f) n = -n;
            valid = finite3(n);
        }
        if (!valid) return false;
        gap = 0.0f;
    }
    float minMass = FLT_BIG_;
    const uint32_t ids[4] = {A.x, A.y, B.x, B.y};
    for (int j = 0; j < 4; j++) {
        const float mm = d.posLin[ids[j]].w;
        if (mm > 0.0f) minMass = mn(minMass, mm);
    }
    if (minMass == FLT_BIG_) return false;
    if (EMIT) {
        const float friction = sqrtf(mx((d.props[A.x].w + d.props[A.y].w) * 0.5f * (d.props[B.x].w + d.props[B.y].w) * 0.5f,
                                        0.0f));
        const float3 dq = (a0 - xyz(d.initLin[A.x])) * (1.0f - s) + (a1 - xyz(d.initLin[A.y])) * s -
                          (b0 - xyz(d.initLin[B.x])) * (1.0f - t) - (b1 - xyz(d.initLin[B.y])) * t;
        const float Cdetect = gap - hSum + P.elemMargin;
        const float C0n = Cdetect - dot(n, dq);
        soft_write(P, d, slot, make_uint4(A.x, A.y, B.x, B.y), make_float4(1.0f - s, s, -(1.0f - t), -t), n, friction,
                   s3(0), C0n, hSum - P.elemMargin, soft_lambda_cap(P, minMass), minMass, SC_EE, false, false, false,
                   keyA, keyB);
    }
    return true;
}

template <bool EMIT>
__global__ void __launch_bounds__(128) k_dat_contacts(const Params P, const DevPtrs d, uint32_t owners) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t below = (1u << lane) - 1u;
    const uint32_t stored = d.counters->datStored;
    const uint32_t head = d.counters->numSoftRT;
    for (uint32_t owner = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; owner < owners; owner += warps) {
        const uint32_t s0 = d.datOwnerStart[owner];
        const uint32_t e0 = min(s0 + d.datOwnerCount[owner], stored);
        const uint32_t base = EMIT ? head + d.datEmitStart[owner] : 0u;
        uint32_t count = 0;
        for (uint32_t k0 = s0; k0 < e0; k0 += 32) {
            const uint32_t k = k0 + lane;
            bool emit = false;
            if (k < e0) emit = dat_contact<false>(P, d, d.datPairs[k], 0u);
            const uint32_t ballot = __ballot_sync(0xffffffffu, emit);
            if (EMIT && emit) dat_contact<true>(P, d, d.datPairs[k], base + count + __popc(ballot & below));
            count += __popc(ballot);
        }
        if (!EMIT && lane == 0) d.datEmit[owner] = count;
    }
}

// soft_finalize (25_cloth.metal:1144-1165): raw demand and the stored count.
__global__ void k_soft_totals(const Params P, const DevPtrs d, uint32_t owners) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Counters* c = d.counters;
    const uint32_t dat = owners ? d.datEmitStart[owners - 1] + d.datEmit[owners - 1] : 0u;
    c->softRaw = c->numSoftRT + dat;
    c->numSoft = min(c->softRaw, P.maxSoft);
}

// softmap_insert (25_cloth.metal:111-145).  A record whose keys repeat one of
// the three records before it (the same triangle's rigid features) is not
// inserted, so the first record of a key is the one found.
__global__ void k_softmap_insert(const Params P, const DevPtrs d) {
    const uint32_t n = d.counters->numSoft;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t keyA = __float_as_uint(d.soft[i].lambda.w), keyB = __float_as_uint(d.soft[i].penalty.w);
        bool dup = false;
        for (uint32_t j = i > 3 ? i - 3 : 0; j < i; j++)
            dup = dup || (__float_as_uint(d.soft[j].lambda.w) == keyA && __float_as_uint(d.soft[j].penalty.w) == keyB);
        if (dup) continue;
        uint32_t h = soft_key_hash(keyA, keyB, P.softMapCapacity);
        for (uint32_t probe = 0; probe < P.softMapCapacity; probe++) {
            if (atomicCAS(&d.softKeyA[h], 0u, keyA + 1u) == 0u) {
                d.softKeyB[h] = keyB;
                d.softVal[h] = i;
                break;
            }
            h = (h + 1u) & (P.softMapCapacity - 1u);
        }
    }
}

__global__ void k_reanchor(const Params P, const DevPtrs d) {
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= P.numParticles) return;
    const uint32_t v = d.particleIdx[gid];
    d.ogcPrev[v] = mk4(xyz(d.posLin[v]), 0.0f);
}

// ---------------------------------------------------------------------------
// Planar-DAT truncation (27_planar_dat.metal:536-561, :752-946, :1179-1270)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void count_invalid(const DevPtrs& d, uint32_t* second) {
    atomicAdd(&d.counters->datInvalidAnchor, 1u);
    atomicAdd(second, 1u);
}

__device__ float dat_plane_fraction(const DevPtrs& d, float3 x, float3 dx, float3 n, float3 plane, float side,
                                    float gamma) {
    const float s0 = side * dot(n, x - plane);
    const float q = side * dot(n, dx);
    if (!finite_bits(s0) || !finite_bits(q)) {
        count_invalid(d, &d.counters->datNonfinite);
        return 0.0f;
    }
    if (s0 < -DAT_GEOMETRY_EPS) return 0.0f;
    if (q >= 0.0f || s0 + q > 0.0f) return 1.0f;
    const float hit = mx(s0, 0.0f) / (-q);
    if (hit > 1.0f + DAT_GEOMETRY_EPS) return 1.0f;
    return clampf(mn(gamma * hit, hit - DAT_TIME_MARGIN), 0.0f, 1.0f);
}

__device__ __forceinline__ void trunc_min(const DevPtrs& d, uint32_t b, float t) {
    atomicMin(&d.truncBits[b], __float_as_uint(t));
}

// Position of a pair participant during the pass of `color`: bodies of the
// color carry their pending solve in posNext.
__device__ __forceinline__ float3 cur_pos(const Params& P, const DevPtrs& d, uint32_t b, uint32_t color) {
    if (P.colorJacobi && color != FULL_PASS && d.posLin[b].w > 0.0f && d.colorsA[b] == color)
        return xyz(d.posNext[b]);
    return xyz(d.posLin[b]);
}

__global__ void k_dat_reduce(const Params P, const DevPtrs d, uint32_t color) {
    pdl_prologue();
    const uint32_t count = d.counters->datStored;
    const float relax = P.planarDATRelaxation;
    const bool full = color == FULL_PASS;
    auto active = [&](uint32_t b) { return full || (d.posLin[b].w > 0.0f && d.colorsA[b] == color); };
    auto apply_t = [&](uint32_t b, float3 x, float3 dx, float3 n, float3 plane, float side) {
        const float t = dat_plane_fraction(d, x, dx, n, plane, side, relax);
        if (t < 1.0f) trunc_min(d, b, t);
    };
    for (uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x; gid < count; gid += gridDim.x * blockDim.x) {
        const uint4 pair = d.datPairs[gid];
        if ((pair.w & DAT_PAIR_TRUNCATE) == 0u) continue;
        if (pair.x == DAT_PAIR_VT) {
            const uint32_t v = pair.y;
            const uint4 t = d.tris[pair.z];
            const bool aV = active(v), aA = active(t.x), aB = active(t.y), aC = active(t.z);
            if (!aV && !aA && !aB && !aC) continue;
            const float3 xv = xyz(d.ogcPrev[v]);
            const float3 a = xyz(d.ogcPrev[t.x]), b = xyz(d.ogcPrev[t.y]), c = xyz(d.ogcPrev[t.z]);
            float3 bary;
            const float3 cp = closest_pt_triangle(xv, a, b, c, bary);
            const float3 nh = xv - cp;
            const float gap = len3(nh);
            if (!finite_bits(gap)) {
                count_invalid(d, &d.counters->datNonfinite);
                trunc_min(d, v, 0.0f); trunc_min(d, t.x, 0.0f); trunc_min(d, t.y, 0.0f); trunc_min(d, t.z, 0.0f);
                continue;
            }
            if (gap > P.queryRadius) continue;
            const float3 dv = cur_pos(P, d, v, color) - xv;
            const float3 da = cur_pos(P, d, t.x, color) - a;
            const float3 db = cur_pos(P, d, t.y, color) - b;
            const float3 dc = cur_pos(P, d, t.z, color) - c;
            float3 n;
            if (gap >= DAT_GEOMETRY_EPS) {
                n = nh / gap;
            } else {
                // datVTFallbackNormal (27_planar_dat.metal:292-302)
                const float3 rawN = cross(b - a, c - a);
                const float mag = len3(rawN);
                if (!(finite_bits(mag) && mag >= DAT_GEOMETRY_EPS)) {
                    count_invalid(d, &d.counters->datVTDegenerate);
                    trunc_min(d, v, 0.0f); trunc_min(d, t.x, 0.0f); trunc_min(d, t.y, 0.0f); trunc_min(d, t.z, 0.0f);
                    continue;
                }
                n = rawN / mag;
                if (dot(n, dv - (da + db + dc) / 3.0f) > 0.0f) n = -n;
                atomicAdd(&d.counters->datVTDegenerate, 1u);
            }
            const float approachV = mx(-dot(n, dv), 0.0f);
            const float approachT = mx(mx(dot(n, da), dot(n, db)), mx(dot(n, dc), 0.0f));
            const float lambda = approachV + approachT == 0.0f
                                     ? 0.5f
                                     : clampf(approachT / (approachV + approachT), 0.05f, 0.95f);
            const float3 plane = gap >= DAT_GEOMETRY_EPS ? cp + nh * lambda : cp;
            if (approachV > 0.0f && aV) apply_t(v, xv, dv, n, plane, 1.0f);
            if (approachT > 0.0f) {
                if (aA) apply_t(t.x, a, da, n, plane, -1.0f);
                if (aB) apply_t(t.y, b, db, n, plane, -1.0f);
                if (aC) apply_t(t.z, c, dc, n, plane, -1.0f);
            }
            continue;
        }
        const uint2 A = d.edges[pair.y], B = d.edges[pair.z];
        const bool aA0 = active(A.x), aA1 = active(A.y), aB0 = active(B.x), aB1 = active(B.y);
        if (!aA0 && !aA1 && !aB0 && !aB1) continue;
        const float3 a0 = xyz(d.ogcPrev[A.x]), a1 = xyz(d.ogcPrev[A.y]);
        const float3 b0 = xyz(d.ogcPrev[B.x]), b1 = xyz(d.ogcPrev[B.y]);
        float s, t;
        closest_seg_seg(a0, a1, b0, b1, s, t);
        const float3 ca = a0 + (a1 - a0) * s, cb = b0 + (b1 - b0) * t;
        const float3 nh = ca - cb;
        const float gap = len3(nh);
        if (!finite_bits(gap)) {
            count_invalid(d, &d.counters->datNonfinite);
            trunc_min(d, A.x, 0.0f); trunc_min(d, A.y, 0.0f); trunc_min(d, B.x, 0.0f); trunc_min(d, B.y, 0.0f);
            continue;
        }
        if (gap > P.queryRadius) continue;
        const float3 da0 = cur_pos(P, d, A.x, color) - a0, da1 = cur_pos(P, d, A.y, color) - a1;
        const float3 db0 = cur_pos(P, d, B.x, color) - b0, db1 = cur_pos(P, d, B.y, color) - b1;
        float3 n;
        if (gap > DAT_GEOMETRY_EPS) {
            n = nh / gap;
        } else {
            const float3 rel = (da0 + da1 - db0 - db1) * 0.5f;
            const float3 ua = a1 - a0, ub = b1 - b0;
            const float3 rawN = cross(ua, ub);
            const float mag = len3(rawN);
            bool valid = true;
            if (finite_bits(mag) && mag >= DAT_GEOMETRY_EPS) {
                n = rawN / mag;
            } else {
                const float la = len3(ua), lb = len3(ub);
                float3 u = la >= lb ? ua : ub;
                const float ul = mx(la, lb);
                if (!finite_bits(ul) || ul < DAT_GEOMETRY_EPS) {
                    valid = false;
                } else {
                    u = u / ul;
                    float3 perp = rel - u * dot(u, rel);
                    float pl = len3(perp);
                    if (!finite_bits(pl) || pl < DAT_GEOMETRY_EPS) {
                        const float3 axis = fabsf(u.x) < 0.7f ? mk3(1, 0, 0) : mk3(0, 1, 0);
                        perp = cross(u, axis);
                        pl = len3(perp);
                    }
                    if (!finite_bits(pl) || pl < DAT_GEOMETRY_EPS) valid = false;
                    else n = perp / pl;
                }
            }
            if (valid) {
                if (dot(n, rel) > 0.0f) n = -n;
                valid = finite3(n);
            }
            if (!valid) {
                count_invalid(d, &d.counters->datEEDegenerate);
                trunc_min(d, A.x, 0.0f); trunc_min(d, A.y, 0.0f); trunc_min(d, B.x, 0.0f); trunc_min(d, B.y, 0.0f);
                continue;
            }
            atomicAdd(&d.counters->datEEDegenerate, 1u);
        }
        const float approachA = mx(mx(-dot(n, da0), -dot(n, da1)), 0.0f);
        const float approachB = mx(mx(dot(n, db0), dot(n, db1)), 0.0f);
        const float lambda = approachA + approachB == 0.0f
                                 ? 0.5f
                                 : clampf(approachB / (approachA + approachB), 0.05f, 0.95f);
        const float3 plane = gap > DAT_GEOMETRY_EPS ? cb + nh * lambda : cb;
        if (approachA > 0.0f) {
            if (aA0) apply_t(A.x, a0, da0, n, plane, 1.0f);
            if (aA1) apply_t(A.y, a1, da1, n, plane, 1.0f);
        }
        if (approachB > 0.0f) {
            if (aB0) apply_t(B.x, b0, db0, n, plane, -1.0f);
            if (aB1) apply_t(B.y, b1, db1, n, plane, -1.0f);
        }
    }
}

// Consume a vertex's reduced fraction and move it that far along its
// displacement since the anchor, capped at 0.5 gamma rq.
__device__ __forceinline__ bool dat_apply_one(const Params& P, const DevPtrs& d, uint32_t v, float3 current,
                                              float mass) {
    const Counters* c = d.counters;
    const float3 anchor = xyz(d.ogcPrev[v]);
    float3 dd = current - anchor;
    const bool unsafe = c->datRaw > P.maxDatPairs || c->datPairsPeak > P.maxDatPairs || c->datGridOverflow > 0u ||
                        c->datInvalidAnchor > 0u;
    float t = __uint_as_float(atomicExch(&d.truncBits[v], __float_as_uint(1.0f)));
    if (unsafe) t = 0.0f;
    if (!finite3(dd) || !finite_bits(t)) {
        count_invalid(d, &d.counters->datNonfinite);
        dd = s3(0);
        t = 0.0f;
    }
    bool truncated = t < 1.0f;
    dd *= clampf(t, 0.0f, 1.0f);
    const float maxD = 0.5f * P.planarDATRelaxation * P.queryRadius;
    const float d2 = dot(dd, dd);
    if (d2 > maxD * maxD) {
        dd *= maxD * rsq(d2);
        truncated = true;
    }
    if (truncated) {
        d.posLin[v] = mk4(anchor + dd, mass);
        atomicAdd(&d.counters->datTruncations, 1u);
    }
    return truncated;
}

__global__ void k_dat_apply_particles(const Params P, const DevPtrs d) {
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= P.numParticles) return;
    const uint32_t v = d.particleIdx[gid];
    const float4 cur = d.posLin[v];
    dat_apply_one(P, d, v, xyz(cur), cur.w);
}

// Publish one color's solve: surface vertices through their fraction, every
// other body of the color as solved.
__global__ void k_dat_apply_color(const Params P, const DevPtrs d, uint32_t color, uint32_t count, uint32_t start) {
    pdl_trigger();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    // with the color's start known on the host, the color list and the cloth
    // group (set at upload) are read before waiting for the previous grid
    if (start == NO_HOST_START) pdl_wait();
    const uint32_t v = d.colorList[(start == NO_HOST_START ? d.colorStart[color] : start) + i];
    const bool unclothed = d.clothGroup[v] == 0u;
    if (start != NO_HOST_START) pdl_wait();
    const float mass = d.posLin[v].w;
    const float3 next = xyz(d.posNext[v]);
    if (unclothed) {
        d.posLin[v] = mk4(next, mass);
        d.posAng[v] = d.angNext[v];
        return;
    }
    if (!dat_apply_one(P, d, v, next, mass)) d.posLin[v] = mk4(next, mass);
}

// dat_restore_failed_surface (27_planar_dat.metal:1287-1310)
__global__ void k_dat_restore(const Params P, const DevPtrs d) {
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= P.numBodies || d.shape[gid].w >= 0.0f) return;
    const Counters* c = d.counters;
    const bool failed = c->softRaw > P.maxSoft || c->datPairsPeak > P.maxDatPairs || c->datGridOverflow > 0u ||
                        c->datInvalidAnchor > 0u;
    if (failed) d.posLin[gid] = mk4(xyz(d.initLin[gid]), d.posLin[gid].w);
}

// smooth_particle_velocities (40_solver.metal:2154-2180); velRead is a copy.
__global__ void k_smooth(const Params P, const DevPtrs d, const float4* velRead) {
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= P.numParticles) return;
    const uint32_t v = d.particleIdx[gid];
    const uint32_t s0 = d.nbrStart[v], n = d.nbrCount[v];
    if (n == 0) return;
    float3 avg = s3(0);
    for (uint32_t k = s0; k < s0 + n; k++) avg += xyz(velRead[d.nbrList[k]]);
    avg = avg / (float)n;
    const float3 vel = xyz(velRead[v]);
    d.velLin[v] = mk4(vel + (avg - vel) * P.clothViscosity, 0.0f);
}

uint32_t blocks_for(uint32_t n, uint32_t threads, uint32_t cap = 148u * 16u) {
    const uint32_t need = (n + threads - 1) / threads;
    return need == 0 ? 1u : (need < cap ? need : cap);
}

void build_pairs(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    const uint32_t total = z.numTris + z.numEdges;
    const uint32_t buckets = 2 * z.elemHashSize;
    cudaMemsetAsync(d.elemCellCount, 0, sizeof(uint32_t) * buckets, st);
    k_elem_bin<false><<<blocks_for(total, 128), 128, 0, st>>>(P, d, total);
    launch_exclusive_scan_large(d.elemCellCount, d.elemCellStart, buckets, d.bigScanScratch, st);
    cudaMemcpyAsync(d.elemCursor, d.elemCellStart, sizeof(uint32_t) * buckets, cudaMemcpyDeviceToDevice, st);
    k_elem_bin<true><<<blocks_for(total, 128), 128, 0, st>>>(P, d, total);
    const uint32_t owners = z.numParticles + z.numEdges;
    if (owners == 0) return;
    const uint32_t wblocks = blocks_for(owners * 32u, 128);
    k_dat_pairs<false><<<wblocks, 128, 0, st>>>(P, d, owners);
    launch_exclusive_scan_large(d.datOwnerCount, d.datOwnerStart, owners, d.bigScanScratch, st);
    k_dat_pairs<true><<<wblocks, 128, 0, st>>>(P, d, owners);
    k_dat_pair_totals<<<1, 32, 0, st>>>(P, d, owners);
}

}  // namespace

void launch_rt_emit(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    if (z.numTris == 0) return;
    const bool warp = P.numGlobals > 32;
    if (warp) k_rt_emit<true><<<blocks_for(z.numTris * 32u, 128), 128, 0, st>>>(P, d);
    else k_rt_emit<false><<<blocks_for(z.numTris, 128), 128, 0, st>>>(P, d);
    launch_exclusive_scan_large(d.rtCount, d.rtStart, z.numTris, d.bigScanScratch, st);
    k_rt_write<<<blocks_for(z.numTris, 128), 128, 0, st>>>(P, d);
    k_rt_totals<<<1, 32, 0, st>>>(P, d);
}

void launch_soft_map(const Params& P, const DevPtrs& d, const Sizes& z, uint32_t owners, cudaStream_t st) {
    k_soft_totals<<<1, 32, 0, st>>>(P, d, owners);
    cudaMemsetAsync(d.softKeyA, 0, sizeof(uint32_t) * P.softMapCapacity, st);
    k_softmap_insert<<<blocks_for(z.maxSoft, 128), 128, 0, st>>>(P, d);
}

void launch_cloth_detect(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    build_pairs(P, d, z, st);
    launch_rt_emit(P, d, z, st);
}

void launch_cloth_accept(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    const uint32_t cap = 148u * 16u;
    // predictor pass over the step-start stream
    k_dat_reduce<<<blocks_for(z.maxDatPairs, 128, cap), 128, 0, st>>>(P, d, FULL_PASS);
    if (z.numParticles) k_dat_apply_particles<<<(z.numParticles + 127) / 128, 128, 0, st>>>(P, d);
    // accepted-pose stream, element contacts, soft map
    build_pairs(P, d, z, st);
    const uint32_t owners = z.numParticles + z.numEdges;
    if (owners) {
        const uint32_t wblocks = blocks_for(owners * 32u, 128);
        k_dat_contacts<false><<<wblocks, 128, 0, st>>>(P, d, owners);
        launch_exclusive_scan_large(d.datEmit, d.datEmitStart, owners, d.bigScanScratch, st);
        k_dat_contacts<true><<<wblocks, 128, 0, st>>>(P, d, owners);
    }
    launch_soft_map(P, d, z, owners, st);
    if (z.numParticles) k_reanchor<<<(z.numParticles + 127) / 128, 128, 0, st>>>(P, d);
}

void launch_dat_color(const Params& P, const DevPtrs& d, const Sizes& z, uint32_t color, uint32_t count,
                      cudaStream_t st) {
    if (count == 0) return;
    // programmatic dependent launches, as the primal before them
    launch_pdl(k_dat_reduce, blocks_for(z.maxDatPairs, 128), 128, st, P, d, color);
    launch_pdl(k_dat_apply_color, (count + 127) / 128, 128, st, P, d, color, count,
               z.colorStartHost ? z.colorStartHost[color] : NO_HOST_START);
}

void launch_cloth_restore(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    k_dat_restore<<<(z.numBodies + 127) / 128, 128, 0, st>>>(P, d);
}

void launch_cloth_smoothing(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    if (!(P.clothViscosity > 0.0f) || z.numParticles == 0) return;
    // inertLin is dead after the solve and rewritten by the next warm start
    cudaMemcpyAsync(d.inertLin, d.velLin, sizeof(float4) * z.numBodies, cudaMemcpyDeviceToDevice, st);
    k_smooth<<<(z.numParticles + 127) / 128, 128, 0, st>>>(P, d, d.inertLin);
}

}  // namespace avbd
