// ogc.cu — isotropic-OGC element contacts: tet boundary surfaces, cloth
// under isotropic truncation, and mixed scenes of soft bodies, rigid bodies
// and cloth.
//
// Follows Shaders/25_cloth.metal: the element grid at detection-radius
// cells (:147-267, isotropic cover), vertex-triangle tracking and emission
// (vt_emit :347-614), edge-edge tracking and emission (ee_emit :616-855),
// the conservative bounds and their mid-solve refresh (:857-931); the
// bound truncation itself lives in the primal (solver.cu, 40_solver.metal
// :1361-1382, :1677-1681) and the warm start (40_solver.metal:700-717).
// Stage order: GPUSolver.swift:3683-3790 (detection) and :4236-4276 (refresh).
//
// Everything here is deterministic:
//   * element grid buckets are sorted by element index after the scatter;
//   * every tracker reads the tracked sets of the previous frame (its own and
//     its neighbours') and writes this frame's into the other buffer;
//   * bounds are minima of non-negative squared distances (order-free
//     atomics on float bits);
//   * contact records are counted per query owner, scanned and written in
//     owner order: rigid-triangle records, then V-T by particle, then E-E by
//     edge.
#include "bucket_sort.cuh"
#include "elements.cuh"
#include "pdl.cuh"

namespace avbd {

namespace {

constexpr uint32_t NONE = 0xFFFFFFFFu;

// The four closest elements seen, ascending by squared distance; an equal
// distance goes after the ones already held.
struct Best4 {
    uint32_t id[4];
    float d2[4];
};

__device__ __forceinline__ void best4_init(Best4& b) {
#pragma unroll
    for (int i = 0; i < 4; i++) { b.id[i] = NONE; b.d2[i] = FLT_BIG_; }
}
__device__ __forceinline__ bool best4_has(const Best4& b, uint32_t t) {
    return b.id[0] == t || b.id[1] == t || b.id[2] == t || b.id[3] == t;
}
__device__ __forceinline__ void best4_insert(Best4& b, uint32_t t, float d2) {
    if (d2 >= b.d2[3]) return;
    int i = 3;
    for (; i > 0 && b.d2[i - 1] > d2; i--) { b.id[i] = b.id[i - 1]; b.d2[i] = b.d2[i - 1]; }
    b.id[i] = t;
    b.d2[i] = d2;
}
__device__ __forceinline__ uint32_t u4_at(uint4 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w)); }

__device__ __forceinline__ void bound_min(const DevPtrs& d, uint32_t b, uint32_t bits) { atomicMin(&d.ogcBounds[b], bits); }

// ---------------------------------------------------------------------------
// Element grid with the isotropic cover: every triangle and authored contact
// edge, its box padded by its largest skin radius plus the element margin,
// in each distinct bucket of at most 3x3x3 cells.  Triangles fill the first
// half of the buckets, edges the second.
// ---------------------------------------------------------------------------
__device__ bool iso_bounds(const Params& P, const DevPtrs& d, uint32_t gid, float3& lo, float3& hi) {
    if (gid < P.numTris) {
        const uint4 t = d.tris[gid];
        const float3 a = xyz(d.posLin[t.x]), b = xyz(d.posLin[t.y]), c = xyz(d.posLin[t.z]);
        const float pad = mx(fabsf(d.shape[t.x].w), mx(fabsf(d.shape[t.y].w), fabsf(d.shape[t.z].w))) + P.elemMargin;
        lo = vmin(vmin(a, b), c) - s3(pad);
        hi = vmax(vmax(a, b), c) + s3(pad);
    } else {
        const uint2 e = d.edges[gid - P.numTris];
        const float3 a = xyz(d.posLin[e.x]), b = xyz(d.posLin[e.y]);
        const float pad = mx(fabsf(d.shape[e.x].w), fabsf(d.shape[e.y].w)) + P.elemMargin;
        lo = vmin(a, b) - s3(pad);
        hi = vmax(a, b) + s3(pad);
    }
    // a non-finite element has no cell (the reference leaves the cast of a
    // non-finite coordinate undefined); it is left out of the grid
    return finite3(lo) && finite3(hi);
}

template <bool SCATTER>
__global__ void k_ogc_bin(const Params P, const DevPtrs d, uint32_t total) {
    for (uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x; gid < total; gid += gridDim.x * blockDim.x) {
        float3 lo, hi;
        if (!iso_bounds(P, d, gid, lo, hi)) continue;
        const I3 c0 = cell_of(lo, P.elemCellSize);
        const I3 c1 = imin3(cell_of(hi, P.elemCellSize), iadd(c0, 2));
        const bool tri = gid < P.numTris;
        const uint32_t entry = tri ? gid : gid - P.numTris;
        const uint32_t half = tri ? 0u : P.elemHashSize;
        uint32_t seen[27];
        uint32_t ns = 0;
        for (int z = c0.z; z <= c1.z; z++)
            for (int y = c0.y; y <= c1.y; y++)
                for (int x = c0.x; x <= c1.x; x++) {
                    const uint32_t h = elem_hash(I3{x, y, z}, P.elemHashSize);
                    bool dup = false;
                    for (uint32_t i = 0; i < ns; i++) dup = dup || seen[i] == h;
                    if (dup) continue;
                    seen[ns++] = h;
                    if (SCATTER) d.elemCellsTmp[atomicAdd(&d.elemCursor[half + h], 1u)] = entry;
                    else atomicAdd(&d.elemCellCount[half + h], 1u);
                }
    }
}

// Every bucket in element order (entries of a bucket are distinct element
// indices): the ballot bucket sort of bucket_sort.cuh.
__global__ void k_ogc_sort_cells(const DevPtrs d, uint32_t buckets) {
    rank_sort_buckets(d.elemCellCount, d.elemCellStart, d.elemCellsTmp, d.elemCells, buckets);
}

// ---------------------------------------------------------------------------
// Vertex-triangle tracking (vt_emit, 25_cloth.metal:347-522)
// ---------------------------------------------------------------------------
struct VtQuery {
    uint32_t v;
    float3 pv;
    uint32_t ns, ne, n2s, n2e, gv;
    bool solidV;
    float boundsCap2;
};

// One candidate triangle: topological exclusion (own and 1-ring triangles,
// triangles of the same closed solid), the tracked-set update and the
// conservative-bound contributions (2-ring excluded).
__device__ void vt_consider(const Params& P, const DevPtrs& d, const VtQuery& q, Best4& best, float& ownB2,
                            uint32_t t) {
    if (t >= P.numTris || best4_has(best, t)) return;
    const uint4 tid = d.tris[t];
    if (tid.x == q.v || tid.y == q.v || tid.z == q.v) return;
    if (q.solidV && d.clothGroup[tid.x] == q.gv && d.clothGroup[tid.y] == q.gv && d.clothGroup[tid.z] == q.gv &&
        d.clothVert[tid.x] == 0u && d.clothVert[tid.y] == 0u && d.clothVert[tid.z] == 0u)
        return;
    float3 bary;
    const float3 cp = closest_pt_triangle(q.pv, xyz(d.posLin[tid.x]), xyz(d.posLin[tid.y]), xyz(d.posLin[tid.z]), bary);
    const float3 dd = q.pv - cp;
    const float d2 = dot(dd, dd);
    if (d2 < best.d2[3] && !nbr_contains(d.nbrList, q.ns, q.ne, tid.x) && !nbr_contains(d.nbrList, q.ns, q.ne, tid.y) &&
        !nbr_contains(d.nbrList, q.ns, q.ne, tid.z))
        best4_insert(best, t, d2);
    if (d2 < q.boundsCap2 && !nbr_contains(d.nbr2List, q.n2s, q.n2e, tid.x) &&
        !nbr_contains(d.nbr2List, q.n2s, q.n2e, tid.y) && !nbr_contains(d.nbr2List, q.n2s, q.n2e, tid.z)) {
        const uint32_t db = __float_as_uint(d2);
        ownB2 = fminf(ownB2, d2);
        bound_min(d, tid.x, db);
        bound_min(d, tid.y, db);
        bound_min(d, tid.z, db);
    }
}

// The contact of vertex v against tracked triangle t (emission loop of
// vt_emit, 25_cloth.metal:531-613).  Returns whether a record is made; with
// EMIT it is written to `slot`.
template <bool EMIT>
__device__ bool vt_contact(const Params& P, const DevPtrs& d, uint32_t v, uint32_t t, uint32_t slot) {
    const float4 plv = d.posLin[v];
    const float3 pv = xyz(plv);
    const float massV = plv.w;
    const float rv = fabsf(d.shape[v].w);
    const float3 velV = xyz(d.velLin[v]);
    const uint4 tid = d.tris[t];
    const float3 a = xyz(d.posLin[tid.x]), b = xyz(d.posLin[tid.y]), c = xyz(d.posLin[tid.z]);
    float3 bary;
    const float3 q = closest_pt_triangle(pv, a, b, c, bary);
    const float3 dv = pv - q;
    const float dist2 = dot(dv, dv);
    const float rt = mx(fabsf(d.shape[tid.x].w), mx(fabsf(d.shape[tid.y].w), fabsf(d.shape[tid.z].w)));
    const float hSum = rv + rt;
    const float3 velT = (xyz(d.velLin[tid.x]) + xyz(d.velLin[tid.y]) + xyz(d.velLin[tid.z])) / 3.0f;
    const float inflate = mn(len3(velV - velT) * P.dt, 0.3f * P.surfaceCellSize);
    const float detect = hSum + P.elemMargin + inflate;
    if (dist2 > detect * detect) return false;
    const float dist = sqrtf(dist2);
    float3 triN = cross(b - a, c - a);
    const float tnLen = len3(triN);
    if (tnLen < 1e-12f) return false;
    triN = triN / tnLen;
    float minMass = massV > 0.0f ? massV : FLT_BIG_;
    const uint32_t others[3] = {tid.x, tid.y, tid.z};
    for (int k = 0; k < 3; k++) {
        if (others[k] == WORLD_BODY) continue;
        const float m = d.posLin[others[k]].w;
        if (m > 0.0f) minMass = mn(minMass, m);
    }
    if (minMass == FLT_BIG_) return false;
    if (EMIT) {
        const uint32_t keyB = t, keyA = (SC_VT << 28) | v;
        const float side = dot(dv, triN) >= 0.0f ? 1.0f : -1.0f;
        const bool deepInterior = bary.x > 0.02f && bary.y > 0.02f && bary.z > 0.02f;
        const float sMem = deepInterior ? soft_prev_side(P, d, keyA, keyB, side) : side;
        float3 n;
        float g;
        if (dist > 1e-7f && side == sMem) { n = dv / dist; g = dist; }
        else { n = triN * sMem; g = -dist; }
        const float fricT = d.props[tid.x].w * bary.x + d.props[tid.y].w * bary.y + d.props[tid.z].w * bary.z;
        const float friction = sqrtf(mx(d.props[v].w * fricT, 0.0f));
        soft_write(P, d, slot, make_uint4(v, tid.x, tid.y, tid.z), make_float4(1.0f, -bary.x, -bary.y, -bary.z), n,
                   friction, s3(0), g - hSum + P.elemMargin, hSum - P.elemMargin, soft_lambda_cap(P, minMass), minMass,
                   SC_VT, false, false, sMem < 0.0f, keyA, keyB);
    }
    return true;
}

__device__ void vt_query(const Params& P, const DevPtrs& d, uint32_t gid, VtQuery& q) {
    q.v = d.particleIdx[gid];
    q.pv = xyz(d.posLin[q.v]);
    q.ns = d.nbrStart[q.v];
    q.ne = q.ns + d.nbrCount[q.v];
    q.gv = d.clothGroup[q.v];
    q.solidV = q.gv != 0u && d.clothVert[q.v] == 0u;
    q.n2s = d.nbr2Start[q.v];
    q.n2e = q.n2s + d.nbr2Count[q.v];
    q.boundsCap2 = P.elemCellSize * P.elemCellSize;
}

// Tracked set, triangle adjacency of the best, neighbours' best; returns
// whether this vertex reseeds from the grid this frame.
__device__ bool vt_begin(const Params& P, const DevPtrs& d, const VtQuery& q, uint32_t frame, Best4& best,
                         float& ownB2) {
    const float3 velV = xyz(d.velLin[q.v]);
    const uint4 tracked = d.vtTrackPrev[q.v];
    for (int i = 0; i < 4; i++) vt_consider(P, d, q, best, ownB2, u4_at(tracked, i));
    if (tracked.x < P.numTris) {
        const uint4 adj = d.triAdj[tracked.x];
        for (int i = 0; i < 3; i++) vt_consider(P, d, q, best, ownB2, u4_at(adj, i));
    }
    for (uint32_t k = q.ns; k < q.ne && k < q.ns + 8; k++) vt_consider(P, d, q, best, ownB2, d.vtTrackPrev[d.nbrList[k]].x);
    // staggered reseed, faster where the motion relative to the tracked
    // surface is large
    float3 relV = velV;
    if (best.id[0] < P.numTris) {
        const uint4 bt = d.tris[best.id[0]];
        relV = relV - (xyz(d.velLin[bt.x]) + xyz(d.velLin[bt.y]) + xyz(d.velLin[bt.z])) / 3.0f;
    }
    const float vThresh = 0.25f * P.elemCellSize / mx(P.dt, 1e-6f);
    const uint32_t period = dot(relV, relV) > vThresh * vThresh ? 1u : 7u;
    const bool missing = best.id[0] == NONE;
    return ((q.v + frame) & period) == 0u || (missing && !q.solidV) || (missing && q.solidV && ((q.v + frame) & 3u) == 0u);
}

// Store the tracked set and the vertex's own bound; returns its contact count.
__device__ uint32_t vt_finish(const Params& P, const DevPtrs& d, const VtQuery& q, const Best4& best, float ownB2) {
    d.vtTrack[q.v] = make_uint4(best.id[0], best.id[1], best.id[2], best.id[3]);
    if (ownB2 < FLT_BIG_) bound_min(d, q.v, __float_as_uint(ownB2));
    uint32_t count = 0;
    for (int bi = 0; bi < 4; bi++) {
        if (best.id[bi] >= P.numTris) break;
        if (vt_contact<false>(P, d, q.v, best.id[bi], 0u)) count++;
    }
    return count;
}

// ---------------------------------------------------------------------------
// Edge-edge tracking (ee_emit, 25_cloth.metal:654-784), authored contact
// edges only
// ---------------------------------------------------------------------------
struct EeQuery {
    uint32_t gid;
    uint2 eA;
    float3 a0, a1;
    uint32_t nsx, nex, nsy, ney, n2sx, n2ex, gA;
    bool solidA;
    float boundsCap2;
};

__device__ void ee_consider(const Params& P, const DevPtrs& d, const EeQuery& q, Best4& best, float& ownB2,
                            uint32_t e) {
    if (e >= P.numEdges || e == q.gid || best4_has(best, e)) return;
    const uint2 eB = d.edges[e];
    if (eB.x == q.eA.x || eB.x == q.eA.y || eB.y == q.eA.x || eB.y == q.eA.y) return;
    if (q.solidA && d.clothGroup[eB.x] == q.gA && d.clothGroup[eB.y] == q.gA && d.clothVert[eB.x] == 0u &&
        d.clothVert[eB.y] == 0u)
        return;
    float s, t;
    const float3 b0 = xyz(d.posLin[eB.x]), b1 = xyz(d.posLin[eB.y]);
    closest_seg_seg(q.a0, q.a1, b0, b1, s, t);
    const float3 cA = q.a0 + (q.a1 - q.a0) * s;
    const float3 cB = b0 + (b1 - b0) * t;
    const float3 dd = cA - cB;
    const float d2 = dot(dd, dd);
    if (d2 < best.d2[3] && !nbr_contains(d.nbrList, q.nsx, q.nex, eB.x) &&
        !nbr_contains(d.nbrList, q.nsx, q.nex, eB.y) && !nbr_contains(d.nbrList, q.nsy, q.ney, eB.x) &&
        !nbr_contains(d.nbrList, q.nsy, q.ney, eB.y))
        best4_insert(best, e, d2);
    if (d2 < q.boundsCap2 && !nbr_contains(d.nbr2List, q.n2sx, q.n2ex, eB.x) &&
        !nbr_contains(d.nbr2List, q.n2sx, q.n2ex, eB.y)) {
        const uint32_t db = __float_as_uint(d2);
        ownB2 = fminf(ownB2, d2);
        bound_min(d, eB.x, db);
        bound_min(d, eB.y, db);
    }
}

// Emission loop of ee_emit (25_cloth.metal:792-854): interior closest points,
// each pair once (owned by the smaller edge index).
template <bool EMIT>
__device__ bool ee_contact(const Params& P, const DevPtrs& d, uint32_t gid, uint32_t eBi, uint32_t slot) {
    const uint2 eA = d.edges[gid], eB = d.edges[eBi];
    const float3 a0 = xyz(d.posLin[eA.x]), a1 = xyz(d.posLin[eA.y]);
    const float3 b0 = xyz(d.posLin[eB.x]), b1 = xyz(d.posLin[eB.y]);
    float s, t;
    closest_seg_seg(a0, a1, b0, b1, s, t);
    if (s < EE_INTERIOR_EPS || s > 1.0f - EE_INTERIOR_EPS || t < EE_INTERIOR_EPS || t > 1.0f - EE_INTERIOR_EPS)
        return false;
    const float3 cA = a0 + (a1 - a0) * s;
    const float3 cB = b0 + (b1 - b0) * t;
    const float3 dv = cA - cB;
    const float dist = len3(dv);
    const float rA = mx(fabsf(d.shape[eA.x].w), fabsf(d.shape[eA.y].w));
    const float rB = mx(fabsf(d.shape[eB.x].w), fabsf(d.shape[eB.y].w));
    const float hSum = rA + rB;
    const float3 velA = (xyz(d.velLin[eA.x]) + xyz(d.velLin[eA.y])) * 0.5f;
    const float3 velB = (xyz(d.velLin[eB.x]) + xyz(d.velLin[eB.y])) * 0.5f;
    const float inflate = mn(len3(velA - velB) * P.dt, 0.3f * P.surfaceCellSize);
    if (dist - hSum > P.elemMargin + inflate) return false;
    if (dist < 1e-7f) return false;
    float minMass = FLT_BIG_;
    const uint32_t ids[4] = {eA.x, eA.y, eB.x, eB.y};
    for (int j = 0; j < 4; j++) {
        const float m = d.posLin[ids[j]].w;
        if (m > 0.0f) minMass = mn(minMass, m);
    }
    if (minMass == FLT_BIG_) return false;
    if (EMIT) {
        const float3 nGeo = dv / dist;
        const uint32_t keyA = (SC_EE << 28) | gid, keyB = eBi;
        float3 n = nGeo;
        float g = dist;
        const int prev = soft_map_find(P, d, keyA, keyB);
        if (prev >= 0 && dot(nGeo, xyz(d.prevSoft[prev].normal)) < 0.0f) {
            n = -nGeo;
            g = -dist;
        }
        const float fric = sqrtf(mx((d.props[eA.x].w + d.props[eA.y].w) * 0.5f * (d.props[eB.x].w + d.props[eB.y].w) * 0.5f,
                                    0.0f));
        soft_write(P, d, slot, make_uint4(eA.x, eA.y, eB.x, eB.y), make_float4(1.0f - s, s, -(1.0f - t), -t), n, fric,
                   s3(0), g - hSum + P.elemMargin, hSum - P.elemMargin, soft_lambda_cap(P, minMass), minMass, SC_EE,
                   false, false, false, keyA, keyB);
    }
    return true;
}

__device__ void ee_query(const Params& P, const DevPtrs& d, uint32_t gid, EeQuery& q) {
    q.gid = gid;
    q.eA = d.edges[gid];
    q.a0 = xyz(d.posLin[q.eA.x]);
    q.a1 = xyz(d.posLin[q.eA.y]);
    q.nsx = d.nbrStart[q.eA.x];
    q.nex = q.nsx + d.nbrCount[q.eA.x];
    q.nsy = d.nbrStart[q.eA.y];
    q.ney = q.nsy + d.nbrCount[q.eA.y];
    q.gA = d.clothGroup[q.eA.x];
    q.solidA = q.gA != 0u && d.clothGroup[q.eA.y] == q.gA && d.clothVert[q.eA.x] == 0u && d.clothVert[q.eA.y] == 0u;
    q.n2sx = d.nbr2Start[q.eA.x];
    q.n2ex = q.n2sx + d.nbr2Count[q.eA.x];
    q.boundsCap2 = P.elemCellSize * P.elemCellSize;
}

__device__ bool ee_begin(const Params& P, const DevPtrs& d, const EeQuery& q, uint32_t frame, Best4& best,
                         float& ownB2) {
    const float3 velA = (xyz(d.velLin[q.eA.x]) + xyz(d.velLin[q.eA.y])) * 0.5f;
    const uint4 tracked = d.eeTrackPrev[q.gid];
    for (int i = 0; i < 4; i++) ee_consider(P, d, q, best, ownB2, u4_at(tracked, i));
    for (int side = 0; side < 2; side++) {
        const uint32_t vv = side == 0 ? q.eA.x : q.eA.y;
        const uint32_t es = d.vertEdgeStart[vv], ec = min(d.vertEdgeCount[vv], 6u);
        for (uint32_t k = es; k < es + ec; k++) ee_consider(P, d, q, best, ownB2, d.eeTrackPrev[d.vertEdgeList[k]].x);
    }
    float3 relV = velA;
    if (best.id[0] < P.numEdges) {
        const uint2 bt = d.edges[best.id[0]];
        relV = relV - (xyz(d.velLin[bt.x]) + xyz(d.velLin[bt.y])) * 0.5f;
    }
    const float vThresh = 0.25f * P.elemCellSize / mx(P.dt, 1e-6f);
    const uint32_t period = dot(relV, relV) > vThresh * vThresh ? 1u : 7u;
    const bool missing = best.id[0] == NONE;
    return ((q.gid + frame) & period) == 0u || (missing && !q.solidA) ||
           (missing && q.solidA && ((q.gid + frame) & 3u) == 0u);
}

__device__ uint32_t ee_finish(const Params& P, const DevPtrs& d, const EeQuery& q, const Best4& best, float ownB2) {
    d.eeTrack[q.gid] = make_uint4(best.id[0], best.id[1], best.id[2], best.id[3]);
    if (ownB2 < FLT_BIG_) {
        bound_min(d, q.eA.x, __float_as_uint(ownB2));
        bound_min(d, q.eA.y, __float_as_uint(ownB2));
    }
    uint32_t count = 0;
    for (int bi = 0; bi < 4; bi++) {
        const uint32_t e = best.id[bi];
        if (e >= P.numEdges) break;
        if (e <= q.gid) continue;
        if (ee_contact<false>(P, d, q.gid, e, 0u)) count++;
    }
    return count;
}

__device__ __forceinline__ void save_partial(const DevPtrs& d, uint32_t o, const Best4& b, float ownB2) {
    float4* p = d.ogcPartial + 3 * (size_t)o;
    p[0] = make_float4(__uint_as_float(b.id[0]), __uint_as_float(b.id[1]), __uint_as_float(b.id[2]),
                       __uint_as_float(b.id[3]));
    p[1] = make_float4(b.d2[0], b.d2[1], b.d2[2], b.d2[3]);
    p[2] = make_float4(ownB2, 0.0f, 0.0f, 0.0f);
}
__device__ __forceinline__ void load_partial(const DevPtrs& d, uint32_t o, Best4& b, float& ownB2) {
    const float4* p = d.ogcPartial + 3 * (size_t)o;
    const float4 ids = p[0], d2 = p[1];
    b.id[0] = __float_as_uint(ids.x); b.id[1] = __float_as_uint(ids.y);
    b.id[2] = __float_as_uint(ids.z); b.id[3] = __float_as_uint(ids.w);
    b.d2[0] = d2.x; b.d2[1] = d2.y; b.d2[2] = d2.z; b.d2[3] = d2.w;
    ownB2 = p[2].x;
}

// Owners [0, numParticles) are V-T queries, the rest E-E queries.  The
// first pass evaluates the cheap candidates (tracked sets, adjacency,
// neighbours) and finishes every owner that does not reseed this frame; the
// reseeding owners (a quarter to an eighth of them) are queued so that the
// grid scans run without idle lanes.  Each owner's result is independent of
// the queue order.
__global__ void k_ogc_track(const Params P, const DevPtrs d, uint32_t owners) {
    const uint32_t frame = d.frameCounter[0];
    for (uint32_t o = blockIdx.x * blockDim.x + threadIdx.x; o < owners; o += gridDim.x * blockDim.x) {
        Best4 best;
        best4_init(best);
        float ownB2 = FLT_BIG_;
        bool reseed;
        uint32_t count = 0;
        if (o < P.numParticles) {
            VtQuery q;
            vt_query(P, d, o, q);
            reseed = vt_begin(P, d, q, frame, best, ownB2);
            if (!reseed) count = vt_finish(P, d, q, best, ownB2);
        } else {
            EeQuery q;
            ee_query(P, d, o - P.numParticles, q);
            reseed = ee_begin(P, d, q, frame, best, ownB2);
            if (!reseed) count = ee_finish(P, d, q, best, ownB2);
        }
        if (reseed) {
            save_partial(d, o, best, ownB2);
            d.datOwnerCount[atomicAdd(&d.counters->ogcQueue, 1u)] = o;
        } else {
            d.datEmit[o] = count;
        }
    }
}

// ---------------------------------------------------------------------------
// Grid reseed of the queued owners, one warp per owner.  The serial tracker
// keeps the four closest distinct candidates by (distance, arrival order):
// an equal distance never displaces an earlier arrival, and a candidate that
// is already held is skipped.  So the warp splits the candidate stream
// (buckets in (dz, dy, dx) order, each bucket in element order) over its
// lanes, every lane keeps its own four by (distance, arrival) — lane 0
// starting from the tracked set found before the reseed — and four rounds of
// a warp-wide minimum pick the result, each winner removed from every lane.
// Bound contributions are minima and need no order.
// ---------------------------------------------------------------------------
struct Best4A {
    uint32_t id[4], arr[4];
    float d2[4];
};

__device__ __forceinline__ void best4a_init(Best4A& b) {
#pragma unroll
    for (int i = 0; i < 4; i++) { b.id[i] = NONE; b.arr[i] = NONE; b.d2[i] = FLT_BIG_; }
}
// arrivals of one lane increase, so (d2, arrival) order is the serial rule
__device__ __forceinline__ void best4a_insert(Best4A& b, uint32_t t, float d2, uint32_t arr) {
    if (b.id[0] == t || b.id[1] == t || b.id[2] == t || b.id[3] == t) return;
    if (d2 >= b.d2[3]) return;
    int i = 3;
    for (; i > 0 && b.d2[i - 1] > d2; i--) { b.id[i] = b.id[i - 1]; b.d2[i] = b.d2[i - 1]; b.arr[i] = b.arr[i - 1]; }
    b.id[i] = t;
    b.d2[i] = d2;
    b.arr[i] = arr;
}

__device__ void warp_merge(Best4A& loc, Best4& out, uint32_t lane) {
    for (int r = 0; r < 4; r++) {
        float d2 = loc.d2[0];
        uint32_t arr = loc.arr[0], id = loc.id[0];
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
            const float od = __shfl_xor_sync(0xffffffffu, d2, o);
            const uint32_t oa = __shfl_xor_sync(0xffffffffu, arr, o);
            const uint32_t oi = __shfl_xor_sync(0xffffffffu, id, o);
            if (od < d2 || (od == d2 && oa < arr)) { d2 = od; arr = oa; id = oi; }
        }
        out.id[r] = id;
        out.d2[r] = d2;
        if (id == NONE) continue;
        // drop the winner from every lane, keeping each list in order
        int w = 0;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            if (loc.id[i] == id) continue;
            loc.id[w] = loc.id[i]; loc.d2[w] = loc.d2[i]; loc.arr[w] = loc.arr[i];
            w++;
        }
        for (; w < 4; w++) { loc.id[w] = NONE; loc.d2[w] = FLT_BIG_; loc.arr[w] = NONE; }
    }
    (void)lane;
}

// The serial tracked-set update of vt_consider without the held-set test
// (duplicates are removed by the merge; their bound contributions repeat).
// Split in two for the reseed's packed lanes: the topological rejections
// (index, own triangle, same closed solid) and the rest, which is only run
// on the candidates the first part keeps.
__device__ __forceinline__ bool vt_kept(const Params& P, const DevPtrs& d, const VtQuery& q, uint32_t t) {
    if (t >= P.numTris) return false;
    const uint4 tid = d.tris[t];
    if (tid.x == q.v || tid.y == q.v || tid.z == q.v) return false;
    return !(q.solidV && d.clothGroup[tid.x] == q.gv && d.clothGroup[tid.y] == q.gv && d.clothGroup[tid.z] == q.gv &&
             d.clothVert[tid.x] == 0u && d.clothVert[tid.y] == 0u && d.clothVert[tid.z] == 0u);
}
__device__ void vt_consider_kept(const Params& P, const DevPtrs& d, const VtQuery& q, Best4A& loc, float& ownB2,
                                 uint32_t t, uint32_t arr) {
    const uint4 tid = d.tris[t];
    float3 bary;
    const float3 cp = closest_pt_triangle(q.pv, xyz(d.posLin[tid.x]), xyz(d.posLin[tid.y]), xyz(d.posLin[tid.z]), bary);
    const float3 dd = q.pv - cp;
    const float d2 = dot(dd, dd);
    if (d2 < loc.d2[3] && !nbr_contains(d.nbrList, q.ns, q.ne, tid.x) && !nbr_contains(d.nbrList, q.ns, q.ne, tid.y) &&
        !nbr_contains(d.nbrList, q.ns, q.ne, tid.z))
        best4a_insert(loc, t, d2, arr);
    if (d2 < q.boundsCap2 && !nbr_contains(d.nbr2List, q.n2s, q.n2e, tid.x) &&
        !nbr_contains(d.nbr2List, q.n2s, q.n2e, tid.y) && !nbr_contains(d.nbr2List, q.n2s, q.n2e, tid.z)) {
        const uint32_t db = __float_as_uint(d2);
        ownB2 = fminf(ownB2, d2);
        bound_min(d, tid.x, db);
        bound_min(d, tid.y, db);
        bound_min(d, tid.z, db);
    }
}

__device__ __forceinline__ bool ee_kept(const Params& P, const DevPtrs& d, const EeQuery& q, uint32_t e) {
    if (e >= P.numEdges || e == q.gid) return false;
    const uint2 eB = d.edges[e];
    if (eB.x == q.eA.x || eB.x == q.eA.y || eB.y == q.eA.x || eB.y == q.eA.y) return false;
    return !(q.solidA && d.clothGroup[eB.x] == q.gA && d.clothGroup[eB.y] == q.gA && d.clothVert[eB.x] == 0u &&
             d.clothVert[eB.y] == 0u);
}
__device__ void ee_consider_kept(const Params& P, const DevPtrs& d, const EeQuery& q, Best4A& loc, float& ownB2,
                                 uint32_t e, uint32_t arr) {
    const uint2 eB = d.edges[e];
    float s, t;
    const float3 b0 = xyz(d.posLin[eB.x]), b1 = xyz(d.posLin[eB.y]);
    closest_seg_seg(q.a0, q.a1, b0, b1, s, t);
    const float3 cA = q.a0 + (q.a1 - q.a0) * s;
    const float3 cB = b0 + (b1 - b0) * t;
    const float3 dd = cA - cB;
    const float d2 = dot(dd, dd);
    if (d2 < loc.d2[3] && !nbr_contains(d.nbrList, q.nsx, q.nex, eB.x) &&
        !nbr_contains(d.nbrList, q.nsx, q.nex, eB.y) && !nbr_contains(d.nbrList, q.nsy, q.ney, eB.x) &&
        !nbr_contains(d.nbrList, q.nsy, q.ney, eB.y))
        best4a_insert(loc, e, d2, arr);
    if (d2 < q.boundsCap2 && !nbr_contains(d.nbr2List, q.n2sx, q.n2ex, eB.x) &&
        !nbr_contains(d.nbr2List, q.n2sx, q.n2ex, eB.y)) {
        const uint32_t db = __float_as_uint(d2);
        ownB2 = fminf(ownB2, d2);
        bound_min(d, eB.x, db);
        bound_min(d, eB.y, db);
    }
}

__global__ void __launch_bounds__(128) k_ogc_reseed(const Params P, const DevPtrs d) {
    // per warp: the queue of candidates kept by the topological tests
    // (element, arrival), drained 32 at a time onto the lanes
    __shared__ uint32_t keptId[4][64], keptArr[4][64];
    const uint32_t n = d.counters->ogcQueue;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t w = threadIdx.x >> 5, below = (1u << lane) - 1u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        const uint32_t o = d.datOwnerCount[i];
        Best4 start;
        float ownB2;
        load_partial(d, o, start, ownB2);
        if (lane != 0) ownB2 = FLT_BIG_;
        Best4A loc;
        best4a_init(loc);
        if (lane == 0)
            for (int k = 0; k < 4; k++) { loc.id[k] = start.id[k]; loc.d2[k] = start.d2[k]; loc.arr[k] = (uint32_t)k; }
        const bool vt = o < P.numParticles;
        VtQuery qv;
        EeQuery qe;
        I3 cc;
        uint32_t half = 0;
        if (vt) {
            vt_query(P, d, o, qv);
            cc = cell_of(qv.pv, P.elemCellSize);
        } else {
            ee_query(P, d, o - P.numParticles, qe);
            cc = cell_of((qe.a0 + qe.a1) * 0.5f, P.elemCellSize);
            half = P.elemHashSize;
        }
        // Candidate j of the stream arrives as 4 + j.  Every lane applies the
        // topological rejections to consecutive candidates; the kept ones
        // queue in arrival order and the distance part runs on 32 of them
        // at a time, lane l taking the l-th of each batch — every lane still
        // sees its candidates in increasing arrival order, which is all the
        // per-lane lists and the warp merge need.  Lane c < 27 first loads
        // the range of bucket c (cells in (dz, dy, dx) order), so the 27
        // buckets cost one dependent load, not 27.
        uint32_t cellS = 0, cellN = 0;
        if (lane < 27) {
            const int dz = (int)(lane / 9u) - 1, dy = (int)((lane / 3u) % 3u) - 1, dx = (int)(lane % 3u) - 1;
            const uint32_t h = half + elem_hash(I3{cc.x + dx, cc.y + dy, cc.z + dz}, P.elemHashSize);
            cellS = d.elemCellStart[h];
            cellN = d.elemCellCount[h];
        }
        uint32_t qn = 0;                                      // queued (warp-uniform)
        auto drain = [&](bool all) {
            while (qn >= 32u || (all && qn > 0u)) {
                const uint32_t take = qn < 32u ? qn : 32u, rest = qn - take;
                const bool mine = lane < take;
                uint32_t id = 0, arr = 0, mid = 0, marr = 0;
                if (mine) { id = keptId[w][lane]; arr = keptArr[w][lane]; }
                if (lane < rest) { mid = keptId[w][take + lane]; marr = keptArr[w][take + lane]; }
                __syncwarp();
                if (lane < rest) { keptId[w][lane] = mid; keptArr[w][lane] = marr; }
                __syncwarp();
                qn = rest;
                if (mine) {
                    if (vt) vt_consider_kept(P, d, qv, loc, ownB2, id, arr);
                    else ee_consider_kept(P, d, qe, loc, ownB2, id, arr);
                }
            }
        };
        uint32_t base = 0;
        for (uint32_t c = 0; c < 27; c++) {
            const uint32_t s0 = __shfl_sync(0xffffffffu, cellS, (int)c);
            const uint32_t cnt = __shfl_sync(0xffffffffu, cellN, (int)c);
            for (uint32_t k0 = 0; k0 < cnt; k0 += 32) {
                const uint32_t k = k0 + lane;
                uint32_t id = 0;
                bool kept = false;
                if (k < cnt) {
                    id = d.elemCells[s0 + k];
                    kept = vt ? vt_kept(P, d, qv, id) : ee_kept(P, d, qe, id);
                }
                const uint32_t ballot = __ballot_sync(0xffffffffu, kept);
                if (kept) {
                    keptId[w][qn + __popc(ballot & below)] = id;
                    keptArr[w][qn + __popc(ballot & below)] = 4u + base + k;
                }
                qn += __popc(ballot);
                __syncwarp();
                drain(false);
            }
            base += cnt;
        }
        drain(true);
        Best4 best;
        warp_merge(loc, best, lane);
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) ownB2 = fminf(ownB2, __shfl_xor_sync(0xffffffffu, ownB2, off));
        if (lane == 0) d.datEmit[o] = vt ? vt_finish(P, d, qv, best, ownB2) : ee_finish(P, d, qe, best, ownB2);
        __syncwarp();
    }
}

__global__ void k_ogc_emit(const Params P, const DevPtrs d, uint32_t owners) {
    const uint32_t head = d.counters->numSoftRT;
    for (uint32_t o = blockIdx.x * blockDim.x + threadIdx.x; o < owners; o += gridDim.x * blockDim.x) {
        uint32_t slot = head + d.datEmitStart[o];
        if (o < P.numParticles) {
            const uint32_t v = d.particleIdx[o];
            const uint4 best = d.vtTrack[v];
            for (int bi = 0; bi < 4; bi++) {
                const uint32_t t = u4_at(best, bi);
                if (t >= P.numTris) break;
                if (vt_contact<false>(P, d, v, t, 0u)) { vt_contact<true>(P, d, v, t, slot); slot++; }
            }
        } else {
            const uint32_t gid = o - P.numParticles;
            const uint4 best = d.eeTrack[gid];
            for (int bi = 0; bi < 4; bi++) {
                const uint32_t e = u4_at(best, bi);
                if (e >= P.numEdges) break;
                if (e <= gid) continue;
                if (ee_contact<false>(P, d, gid, e, 0u)) { ee_contact<true>(P, d, gid, e, slot); slot++; }
            }
        }
    }
}

__global__ void k_ogc_totals(const Params P, const DevPtrs d, uint32_t owners) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const uint32_t vt = P.numParticles < owners ? d.datEmitStart[P.numParticles]
                                                : (owners ? d.datEmitStart[owners - 1] + d.datEmit[owners - 1] : 0u);
    const uint32_t all = owners ? d.datEmitStart[owners - 1] + d.datEmit[owners - 1] : 0u;
    d.counters->numSoftVT = vt;
    d.counters->numSoftEE = all - vt;
}

// ---------------------------------------------------------------------------
// Mid-solve bound refresh (ogc_refresh_args + ogc_bounds_refresh,
// 25_cloth.metal:857-931): when more than 1% of the surface vertices were
// bound-limited in the last pass, re-anchor at the live pose and recompute
// every bound from the tracked sets.
// ---------------------------------------------------------------------------
__global__ void k_ogc_refresh(const Params P, const DevPtrs d, const uint32_t* readSlot, uint32_t* zeroSlot) {
    pdl_prologue();
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid == 0) *zeroSlot = 0u;
    if (!(*readSlot * 100u > P.numParticles) || gid >= P.numParticles) return;
    const uint32_t v = d.particleIdx[gid];
    const float3 pv = xyz(d.posLin[v]);
    const uint32_t n2s = d.nbr2Start[v], n2e = n2s + d.nbr2Count[v];
    float dmin2 = 3.0e38f;
    const uint4 tracked = d.vtTrack[v];
    for (int i = 0; i < 4; i++) {
        const uint32_t t = u4_at(tracked, i);
        if (t >= P.numTris) break;
        const uint4 tid = d.tris[t];
        if (nbr_contains(d.nbr2List, n2s, n2e, tid.x) || nbr_contains(d.nbr2List, n2s, n2e, tid.y) ||
            nbr_contains(d.nbr2List, n2s, n2e, tid.z))
            continue;
        float3 bary;
        const float3 q = closest_pt_triangle(pv, xyz(d.posLin[tid.x]), xyz(d.posLin[tid.y]), xyz(d.posLin[tid.z]), bary);
        const float3 dd = pv - q;
        dmin2 = fminf(dmin2, dot(dd, dd));
    }
    const uint32_t es = d.vertEdgeStart[v], ec = min(d.vertEdgeCount[v], 6u);
    for (uint32_t k = es; k < es + ec; k++) {
        const uint32_t myE = d.vertEdgeList[k];
        const uint32_t other = d.eeTrack[myE].x;
        if (other >= P.numEdges) continue;
        const uint2 eo = d.edges[other];
        if (nbr_contains(d.nbr2List, n2s, n2e, eo.x) || nbr_contains(d.nbr2List, n2s, n2e, eo.y)) continue;
        const uint2 em = d.edges[myE];
        const float3 a0 = xyz(d.posLin[em.x]), a1 = xyz(d.posLin[em.y]);
        const float3 b0 = xyz(d.posLin[eo.x]), b1 = xyz(d.posLin[eo.y]);
        float s, t;
        closest_seg_seg(a0, a1, b0, b1, s, t);
        const float3 dd = (a0 + (a1 - a0) * s) - (b0 + (b1 - b0) * t);
        dmin2 = fminf(dmin2, dot(dd, dd));
    }
    d.ogcBounds[v] = __float_as_uint(dmin2);
    d.ogcPrev[v] = d.posLin[v];
}

// Color-Jacobi commit of one color (the primal of the color wrote posNext).
__global__ void k_publish_color(const DevPtrs d, uint32_t color, uint32_t count, uint32_t start) {
    pdl_trigger();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    // with the start known on the host, the color list and the shape (set
    // at upload) are read before waiting for the previous grid
    if (start == NO_HOST_START) pdl_wait();
    const uint32_t v = d.colorList[(start == NO_HOST_START ? d.colorStart[color] : start) + i];
    const bool rigid = d.shape[v].w >= 0.0f;
    if (start != NO_HOST_START) pdl_wait();
    d.posLin[v] = mk4(xyz(d.posNext[v]), d.posLin[v].w);
    if (rigid) d.posAng[v] = d.angNext[v];
}

uint32_t grid_for(uint32_t n, uint32_t threads, uint32_t cap = 148u * 16u) {
    const uint32_t need = (n + threads - 1) / threads;
    return need == 0 ? 1u : (need < cap ? need : cap);
}

}  // namespace

void launch_ogc_detect(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st) {
    // bounds start "far" (0x7F7F7F7F ~ 3.4e38) every frame
    cudaMemsetAsync(d.ogcBounds, 0x7F, sizeof(uint32_t) * z.numBodies, st);
    const uint32_t total = z.numTris + P.numEdges;
    const uint32_t buckets = 2 * z.elemHashSize;
    cudaMemsetAsync(d.elemCellCount, 0, sizeof(uint32_t) * buckets, st);
    k_ogc_bin<false><<<grid_for(total, 128), 128, 0, st>>>(P, d, total);
    launch_exclusive_scan_large(d.elemCellCount, d.elemCellStart, buckets, d.bigScanScratch, st);
    cudaMemcpyAsync(d.elemCursor, d.elemCellStart, sizeof(uint32_t) * buckets, cudaMemcpyDeviceToDevice, st);
    k_ogc_bin<true><<<grid_for(total, 128), 128, 0, st>>>(P, d, total);
    k_ogc_sort_cells<<<grid_for(buckets * 32u, 128), 128, 0, st>>>(d, buckets);
    const uint32_t owners = z.numParticles + P.numEdges;
    if (owners) {
        k_ogc_track<<<grid_for(owners, 128), 128, 0, st>>>(P, d, owners);
        k_ogc_reseed<<<grid_for(owners * 32u, 128), 128, 0, st>>>(P, d);
    }
    launch_rt_emit(P, d, z, st);
    if (owners) {
        launch_exclusive_scan_large(d.datEmit, d.datEmitStart, owners, d.bigScanScratch, st);
        k_ogc_emit<<<grid_for(owners, 128), 128, 0, st>>>(P, d, owners);
        k_ogc_totals<<<1, 32, 0, st>>>(P, d, owners);
    }
    launch_soft_map(P, d, z, owners, st);
}

void launch_publish_color(const Params& P, const DevPtrs& d, uint32_t color, uint32_t count, uint32_t start,
                          cudaStream_t st) {
    (void)P;
    if (count == 0) return;
    launch_pdl(k_publish_color, (count + 127) / 128, 128, st, d, color, count, start);
}

void launch_ogc_refresh(const Params& P, const DevPtrs& d, const Sizes& z, uint32_t* readSlot, uint32_t* zeroSlot,
                        cudaStream_t st) {
    launch_pdl(k_ogc_refresh, (z.numParticles + 127) / 128, 128, st, P, d, readSlot, zeroSlot);
}

}  // namespace avbd
