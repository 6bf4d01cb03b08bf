// oracle_cloth.cpp — CPU oracle of the cloth stages: element topology,
// membranes and bends, element contacts and Planar-DAT truncation.
//
// TEST INFRASTRUCTURE, NOT PRODUCT CODE (see avbd_oracle.cpp).  Restates
//   upload           GPUSolver.swift:1289-1680 (topology, membranes, bends, params)
//   element grid     25_cloth.metal:147-267
//   pair streams     27_planar_dat.metal:35-228
//   rigid-triangle   25_cloth.metal:942-1142
//   contact emission 27_planar_dat.metal:344-510, softEmit 25_cloth.metal:269-333
//   soft map         25_cloth.metal:79-145
//   DAT passes       27_planar_dat.metal:525-561, :752-946, :1179-1310
//   stamps / dual    40_solver.metal:1088-1153, :1236-1359, :1689-1727
//   smoothing        40_solver.metal:2150-2180
//   isotropic OGC    25_cloth.metal:147-267 (isotropic cover), :347-931
//                    (V-T / E-E trackers, bounds, refresh), topology
//                    GPUSolver.swift:1338-1460
//
// Deterministic where the reference is scheduling-dependent (each choice is
// one of the orders the reference can produce):
//   * pair streams are ordered V-T by (particle, triangle), then E-E by
//     (edge, other edge); the reference appends them with atomics;
//   * element contacts are numbered rigid-triangle first by triangle, then in
//     pair order; the reference takes slots with atomics;
//   * bends are numbered by ascending edge key; the reference walks a Swift
//     dictionary whose order is seeded per process;
//   * isotropic trackers read the tracked sets of the previous frame (own and
//     neighbours'); the reference reads neighbours' sets while they are
//     being rewritten; element grid buckets hold elements in index order;
//     triangle adjacency is filled in ascending edge-key order;
//   * a body's solve reads the pre-color pose of bodies in its own color
//     (a Jacobi step inside the color); the reference's reads race with the
//     writes of same-color neighbours (membrane diagonals, bend stencils,
//     element contacts between vertices of one color).
#include "oracle_solver.h"

#include <unordered_set>

namespace oracle {

static const uint32_t FULL_PASS = 0xFFFFFFFFu;

static inline F3 pos_of(const avbd_scene_desc* s, int i) {
    return f3(s->bodies[i].position[0], s->bodies[i].position[1], s->bodies[i].position[2]);
}
static inline F3 vmin3(F3 a, F3 b) { return F3{std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
static inline F3 vmax3(F3 a, F3 b) { return F3{std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }

struct I3 { int x, y, z; };
static inline I3 cell_of(F3 p, float cs) {
    return I3{(int)std::floor(p.x / cs), (int)std::floor(p.y / cs), (int)std::floor(p.z / cs)};
}
static inline uint32_t elem_hash(I3 c, uint32_t size) { return cell_hash(c.x, c.y, c.z, 0u, size); }

// Closest point on triangle (Ericson 5.1.5; 25_cloth.metal:27-63).
static F3 closest_pt_triangle(F3 p, F3 a, F3 b, F3 c, F3& bary) {
    F3 ab = b - a, ac = c - a, ap = p - a;
    float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) { bary = f3(1, 0, 0); return a; }
    F3 bp = p - b;
    float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) { bary = f3(0, 1, 0); return b; }
    float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        float v = d1 / fmax_(d1 - d3, 1e-12f);
        bary = f3(1 - v, v, 0);
        return a + ab * v;
    }
    F3 cp = p - c;
    float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) { bary = f3(0, 0, 1); return c; }
    float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        float w = d2 / fmax_(d2 - d6, 1e-12f);
        bary = f3(1 - w, 0, w);
        return a + ac * w;
    }
    float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        float w = (d4 - d3) / fmax_((d4 - d3) + (d5 - d6), 1e-12f);
        bary = f3(0, 1 - w, w);
        return b + (c - b) * w;
    }
    float denom = va + vb + vc;
    if (std::fabs(denom) < 1e-20f) { bary = f3(1, 0, 0); return a; }
    float v = vb / denom, w = vc / denom;
    bary = f3(1 - v - w, v, w);
    return a + ab * v + ac * w;
}

// Segment-segment closest parameters (25_cloth.metal:632-648).
static void closest_seg_seg_st(F3 p0, F3 p1, F3 q0, F3 q1, float& s, float& t) {
    F3 d1 = p1 - p0, d2 = q1 - q0, r = p0 - q0;
    float a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    s = 0.0f; t = 0.0f;
    if (a <= 1e-12f && e <= 1e-12f) return;
    if (a <= 1e-12f) { t = clampf_(f / e, 0.0f, 1.0f); return; }
    float c = dot(d1, r);
    if (e <= 1e-12f) { s = clampf_(-c / a, 0.0f, 1.0f); return; }
    float b = dot(d1, d2);
    float denom = a * e - b * b;
    if (std::fabs(denom) > 1e-12f) s = clampf_((b * f - c * e) / denom, 0.0f, 1.0f);
    t = (b * s + f) / e;
    if (t < 0.0f) { t = 0.0f; s = clampf_(-c / a, 0.0f, 1.0f); }
    else if (t > 1.0f) { t = 1.0f; s = clampf_((b - c) / a, 0.0f, 1.0f); }
}

static bool nbr_contains(const std::vector<uint32_t>& list, uint32_t s, uint32_t e, uint32_t x) {
    uint32_t lo = s, hi = e;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (list[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo < e && list[lo] == x;
}

static inline uint32_t soft_key_hash(uint32_t a, uint32_t b, uint32_t cap) {
    uint32_t h = (a * 0x9E3779B1u) ^ (b * 0x85EBCA77u);
    h ^= h >> 16;
    h *= 0xC2B2AE3Du;
    h ^= h >> 13;
    return h & (cap - 1u);
}

// ==========================================================================
// Upload (GPUSolver.swift:1289-1680)
// ==========================================================================
int Solver::cloth_upload(const avbd_scene_desc* s, const std::vector<std::array<int, 3>>& boundary) {
    numAuthoredTris = s->num_tris;
    cloth = numAuthoredTris > 0;
    std::vector<std::array<int, 3>> coll;
    for (uint32_t i = 0; i < s->num_tris; i++) coll.push_back({s->tris[i].ids[0], s->tris[i].ids[1], s->tris[i].ids[2]});
    coll.insert(coll.end(), boundary.begin(), boundary.end());
    numTris = (uint32_t)coll.size();
    auto sizex = [&](int i) { return s->bodies[i].size[0]; };

    std::unordered_set<uint64_t> topoSet, contactSet;
    std::vector<uint64_t> topoKeys, contactKeys;
    float maxElemR = 0.0f, maxCollR = 0.0f;
    tris.assign(numTris, U4{});
    for (uint32_t i = 0; i < numTris; i++) {
        int a = coll[i][0], b = coll[i][1], c = coll[i][2];
        tris[i] = U4{(uint32_t)a, (uint32_t)b, (uint32_t)c, 0};
        bool emitsEE = i < numAuthoredTris;
        const int pr[3][2] = {{a, b}, {b, c}, {a, c}};
        for (auto& e : pr) {
            uint64_t key = (uint64_t)std::min(e[0], e[1]) << 32 | (uint64_t)std::max(e[0], e[1]);
            if (topoSet.insert(key).second) topoKeys.push_back(key);
            if (emitsEE && contactSet.insert(key).second) contactKeys.push_back(key);
        }
        F3 pa = pos_of(s, a), pb = pos_of(s, b), pc = pos_of(s, c);
        F3 m = (pa + pb + pc) / 3.0f;
        float thick = fmax_(sizex(a), fmax_(sizex(b), sizex(c))) / 2.0f;
        maxCollR = fmax_(maxCollR, thick);
        maxElemR = fmax_(maxElemR, fmax_(distance(m, pa), fmax_(distance(m, pb), distance(m, pc))) + thick);
    }
    numSurfaceEdges = (uint32_t)contactKeys.size();
    for (uint64_t key : topoKeys)
        if (contactSet.insert(key).second) contactKeys.push_back(key);
    numEdges = (uint32_t)contactKeys.size();
    std::vector<std::vector<uint32_t>> nbr(nb);
    for (uint64_t key : topoKeys) {
        uint32_t a = (uint32_t)(key >> 32), b = (uint32_t)(key & 0xFFFFFFFFu);
        nbr[a].push_back(b);
        nbr[b].push_back(a);
    }
    edges.clear();
    for (uint64_t key : contactKeys) {
        int a = (int)(key >> 32), b = (int)(key & 0xFFFFFFFFu);
        edges.push_back((uint32_t)a);
        edges.push_back((uint32_t)b);
        maxElemR = fmax_(maxElemR, distance(pos_of(s, a), pos_of(s, b)) / 2.0f + fmax_(sizex(a), sizex(b)) / 2.0f);
    }
    nbrStart.assign(nb, 0); nbrCount.assign(nb, 0); nbrList.clear();
    for (uint32_t i = 0; i < nb; i++) {
        std::sort(nbr[i].begin(), nbr[i].end());
        nbrStart[i] = (uint32_t)nbrList.size();
        nbrCount[i] = (uint32_t)nbr[i].size();
        nbrList.insert(nbrList.end(), nbr[i].begin(), nbr[i].end());
    }

    // soft collision groups and self-collision flags (GPUSolver.swift:1476-1535)
    selfCollision.assign(nb, 0);
    std::fill(clothGroup.begin(), clothGroup.end(), 0u);
    std::vector<uint8_t> surf(nb, 0);
    if (!coll.empty()) {
        std::vector<int> parent(nb, -1);
        auto find = [&](int x) {
            int r = x;
            while (parent[r] >= 0 && parent[r] != r) r = parent[r];
            int c = x;
            while (parent[c] >= 0 && parent[c] != r) { int n = parent[c]; parent[c] = r; c = n; }
            if (parent[r] < 0) parent[r] = r;
            return r;
        };
        for (auto& f : coll) { int r = find(f[0]); parent[find(f[1])] = r; parent[find(f[2])] = r; }
        std::set<int> selfRoots;
        for (uint32_t i = 0; i < s->num_tris; i++) selfRoots.insert(find(s->tris[i].ids[0]));
        for (uint32_t i = 0; i < s->num_tets; i++) {
            if (!s->tets[i].self_collision) continue;
            for (int k = 0; k < 4; k++) {
                int id = s->tets[i].ids[k];
                if (parent[id] >= 0) selfRoots.insert(find(id));
            }
        }
        std::map<int, uint32_t> groupIndex;
        for (auto& f : coll) {
            int root = find(f[0]);
            if (!groupIndex.count(root)) { uint32_t g = (uint32_t)groupIndex.size() + 1; groupIndex[root] = g; }
            uint32_t g = groupIndex[root];
            uint32_t sc = selfRoots.count(root) ? 1u : 0u;
            for (int k = 0; k < 3; k++)
                if (isParticle[f[k]]) { clothGroup[f[k]] = g; selfCollision[f[k]] = sc; surf[f[k]] = 1; }
        }
    }
    particleIdx.clear();
    for (uint32_t i = 0; i < nb; i++) if (surf[i]) particleIdx.push_back(i);
    numParticles = numTris == 0 ? 0 : (uint32_t)particleIdx.size();

    // membranes and bends (GPUSolver.swift:1536-1641)
    membranes.clear();
    bends.clear();
    struct Flap { uint32_t mem; int opp; float k; };
    std::map<uint64_t, std::vector<Flap>> edgeTris;
    for (uint32_t ti = 0; ti < s->num_tris; ti++) {
        const avbd_tri_desc& t = s->tris[ti];
        if (!(t.mu > 0.0f)) continue;
        int i0 = t.ids[0], i1 = t.ids[1], i2 = t.ids[2];
        F3 x0 = pos_of(s, i0), x1 = pos_of(s, i1), x2 = pos_of(s, i2);
        F3 d1 = x1 - x0, d2 = x2 - x0;
        F3 nrm = cross(d1, d2);
        float area = length(nrm) / 2.0f;
        if (!(area > 1e-10f)) continue;
        F3 e1 = normalize(d1);
        F3 e2 = normalize(cross(normalize(nrm), e1));
        float a = dot(d1, e1), b = dot(d1, e2);
        float c = dot(d2, e1), dd = dot(d2, e2);
        float det = a * dd - b * c;
        if (!(std::fabs(det) > 1e-12f)) continue;
        MembraneGPU m{};
        m.ids = U4{(uint32_t)i0, (uint32_t)i1, (uint32_t)i2, 0};
        m.dm = f4(dd / det, -b / det, -c / det, a / det);
        m.mat = f4(t.mu * area, t.lambda * area, area, 0.0f);
        membranes.push_back(m);
        if (t.bend > 0.0f) {
            const int fl[3][3] = {{i0, i1, i2}, {i1, i2, i0}, {i0, i2, i1}};
            for (auto& e : fl) {
                uint64_t key = (uint64_t)std::min(e[0], e[1]) << 32 | (uint64_t)std::max(e[0], e[1]);
                edgeTris[key].push_back(Flap{(uint32_t)membranes.size() - 1, e[2], t.bend});
            }
        }
    }
    for (auto& kv : edgeTris) {
        if (kv.second.size() != 2) continue;
        int v0 = (int)(kv.first >> 32), v1 = (int)(kv.first & 0xFFFFFFFFu);
        int opp2 = kv.second[0].opp, opp3 = kv.second[1].opp;
        float k1 = kv.second[0].k, k2 = kv.second[1].k;
        F3 p0 = pos_of(s, v0), p1 = pos_of(s, v1);
        float L = distance(p0, p1);
        if (!(L > 1e-9f)) continue;
        auto unfold = [&](int opp, float side, float& qx, float& qy) {
            float l0 = distance(pos_of(s, opp), p0);
            float l1 = distance(pos_of(s, opp), p1);
            float ax = (L * L + l0 * l0 - l1 * l1) / (2.0f * L);
            float h2 = l0 * l0 - ax * ax;
            if (!(h2 > 1e-12f)) return false;
            qx = ax;
            qy = side * std::sqrt(h2);
            return true;
        };
        float q2x, q2y, q3x, q3y;
        if (!unfold(opp2, 1.0f, q2x, q2y) || !unfold(opp3, -1.0f, q3x, q3y)) continue;
        const float q0x = 0.0f, q0y = 0.0f, q1x = L, q1y = 0.0f;
        const float r2[4] = {q0x, q1x, q2x, q3x};
        const float r3[4] = {q0y, q1y, q2y, q3y};
        auto minor = [&](int c0, int c1, int c2) {
            F3 a = f3(1.0f, r2[c0], r3[c0]), b = f3(1.0f, r2[c1], r3[c1]), c = f3(1.0f, r2[c2], r3[c2]);
            return dot(a, cross(b, c));
        };
        F4 K = f4(minor(1, 2, 3), -minor(0, 2, 3), minor(0, 1, 3), -minor(0, 1, 2));
        auto cot = [](float ax_, float ay, float bx, float by, float cx, float cy) {
            float ux = bx - ax_, uy = by - ay, vx = cx - ax_, vy = cy - ay;
            float cr = ux * vy - uy * vx;
            return std::fabs(cr) > 1e-12f ? (ux * vx + uy * vy) / std::fabs(cr) : 0.0f;
        };
        float want = cot(q0x, q0y, q1x, q1y, q2x, q2y) + cot(q1x, q1y, q0x, q0y, q2x, q2y);
        if (!(std::fabs(K.z) > 1e-12f)) continue;
        K = K * (want / K.z);
        float a1 = std::fabs((q1x - q0x) * q2y) / 2.0f;
        float a2 = std::fabs((q1x - q0x) * q3y) / 2.0f;
        BendGPU bd{};
        bd.ids = U4{(uint32_t)v0, (uint32_t)v1, (uint32_t)opp2, (uint32_t)opp3};
        bd.K = K;
        bd.mat = f4(3.0f * (k1 + k2) / 2.0f / fmax_(a1 + a2, 1e-9f), 0, 0, 0);
        bends.push_back(bd);
    }

    // element-contact parameters (GPUSolver.swift:1643-1680)
    float maxPartR = maxCollR, edgeLenSum = 0.0f;
    for (uint64_t key : topoKeys) {
        int a = (int)(key >> 32), b = (int)(key & 0xFFFFFFFFu);
        maxPartR = fmax_(maxPartR, fmax_(sizex(a), sizex(b)) / 2.0f);
        edgeLenSum += distance(pos_of(s, a), pos_of(s, b));
    }
    float meanEdge = topoKeys.empty() ? 0.2f : edgeLenSum / (float)topoKeys.size();
    elemMargin = fmin_(0.01f, fmax_(0.002f, 0.5f * maxPartR));
    float forceReach = 2.0f * maxPartR + elemMargin;
    queryRadius = fmax_(1.5f * forceReach, 0.75f * meanEdge);
    float reach = (2.0f * maxPartR + elemMargin) / 0.7f;
    surfaceCellSize = fmax_(0.02f, fmax_(fmax_(reach, meanEdge * 1.05f), maxElemR + maxPartR + elemMargin));
    elemCellSize = fmax_(0.02f, fmax_(fmax_(reach, meanEdge * 1.05f), 2.0f * maxElemR + queryRadius));

    // capacities (GPUSolver.swift:395-443)
    uint64_t surfaceParticles = 0;
    for (uint32_t i = 0; i < nb; i++) surfaceParticles += surf[i];
    uint64_t planar = std::max<uint64_t>(1, 64ull * surfaceParticles + 128ull * topoKeys.size());
    uint64_t budget = std::min<uint64_t>(planar, 8ull * surfaceParticles + 8ull * topoKeys.size());
    maxDatPairs = (uint32_t)planar;
    maxSoft = (uint32_t)std::max<uint64_t>(1, 4ull * numTris + budget);
    softMapCapacity = next_pow2(std::max<uint32_t>(64u, 2u * maxSoft));
    elemHashSize = next_pow2(std::max<uint32_t>(64u, 2u * 4u * numTris));

    maxSoftIso = (uint32_t)std::max<uint64_t>(1, 4ull * surfaceParticles + 4ull * numTris + 4ull * numSurfaceEdges);
    softMapCapacityIso = next_pow2(std::max<uint32_t>(64u, 2u * maxSoftIso));
    ogc_topology(coll, nbr);

    soft.assign(maxSoft, SoftContactGPU{});
    prevSoft.assign(maxSoft, SoftContactGPU{});
    softKeyA.assign(softMapCapacity, 0); softKeyB.assign(softMapCapacity, 0); softVal.assign(softMapCapacity, 0);
    truncBits.assign(nb, fbits(1.0f));
    posNext.assign(nb, F4{}); angNext.assign(nb, F4{});
    return AVBD_OK;
}

// ==========================================================================
// Element grid (25_cloth.metal:147-267), Planar-DAT padding.
// ==========================================================================
void Solver::elem_bounds(uint32_t gid, F3& lo, F3& hi) const {
    const float pad = queryRadius;
    if (gid < numTris) {
        U4 t = tris[gid];
        F3 a = xyz(posLin[t.x]), b = xyz(posLin[t.y]), c = xyz(posLin[t.z]);
        lo = vmin3(vmin3(a, b), c) - f3s(pad);
        hi = vmax3(vmax3(a, b), c) + f3s(pad);
    } else {
        uint32_t e = gid - numTris;
        F3 a = xyz(posLin[edges[2 * e]]), b = xyz(posLin[edges[2 * e + 1]]);
        lo = vmin3(a, b) - f3s(pad);
        hi = vmax3(a, b) + f3s(pad);
    }
}

void Solver::elem_grid() {
    std::vector<std::vector<uint32_t>> buckets(elemHashSize);
    const uint32_t total = numTris + numEdges;
    for (uint32_t gid = 0; gid < total; gid++) {
        F3 lo, hi;
        elem_bounds(gid, lo, hi);
        if (!finite3(lo) || !finite3(hi)) { dat.invalidAnchor++; dat.nonfinite++; continue; }
        I3 c0 = cell_of(lo, elemCellSize), r1 = cell_of(hi, elemCellSize);
        if (r1.x - c0.x > 3 || r1.y - c0.y > 3 || r1.z - c0.z > 3) dat.gridOverflow++;
        I3 c1{std::min(r1.x, c0.x + 3), std::min(r1.y, c0.y + 3), std::min(r1.z, c0.z + 3)};
        uint32_t entry = gid < numTris ? gid : (ELEM_EDGE_BIT | (gid - numTris));
        uint32_t seen[64];
        uint32_t ns = 0;
        for (int z = c0.z; z <= c1.z; z++)
            for (int y = c0.y; y <= c1.y; y++)
                for (int x = c0.x; x <= c1.x; x++) {
                    uint32_t h = elem_hash(I3{x, y, z}, elemHashSize);
                    bool dup = false;
                    for (uint32_t i = 0; i < ns; i++) dup = dup || seen[i] == h;
                    if (dup) continue;
                    seen[ns++] = h;
                    buckets[h].push_back(entry);
                }
    }
    elemCellStart.assign(elemHashSize, 0);
    elemCellCount.assign(elemHashSize, 0);
    elemCells.clear();
    for (uint32_t h = 0; h < elemHashSize; h++) {
        elemCellStart[h] = (uint32_t)elemCells.size();
        elemCellCount[h] = (uint32_t)buckets[h].size();
        elemCells.insert(elemCells.end(), buckets[h].begin(), buckets[h].end());
    }
}

// ==========================================================================
// Pair streams (27_planar_dat.metal:35-228)
// ==========================================================================
void Solver::dat_build_pairs() {
    datPairs.clear();
    datRaw = datVT = datEE = 0;
    const float query2 = queryRadius * queryRadius;
    auto append = [&](uint32_t kind, uint32_t owner, uint32_t other, uint32_t flags) {
        uint32_t slot = datRaw++;
        if (kind == DAT_PAIR_VT) datVT++; else datEE++;
        if (slot < maxDatPairs) datPairs.push_back(U4{kind, owner, other, flags});
    };
    auto in_range = [](I3 c, I3 lo, I3 hi) {
        return c.x >= lo.x && c.y >= lo.y && c.z >= lo.z && c.x <= hi.x && c.y <= hi.y && c.z <= hi.z;
    };
    for (uint32_t gid = 0; gid < numParticles; gid++) {
        uint32_t v = particleIdx[gid];
        F3 p = xyz(posLin[v]);
        if (!finite3(p)) { dat.invalidAnchor++; dat.nonfinite++; continue; }
        I3 cell = cell_of(p, elemCellSize);
        uint32_t h = elem_hash(cell, elemHashSize);
        uint32_t s0 = elemCellStart[h], e0 = s0 + elemCellCount[h];
        uint32_t ns = nbrStart[v], ne = ns + nbrCount[v];
        std::vector<uint32_t> cand;
        for (uint32_t k = s0; k < e0; k++) {
            uint32_t entry = elemCells[k];
            if ((entry & ELEM_EDGE_BIT) != 0u || entry >= numTris) continue;
            U4 t = tris[entry];
            if (t.x == v || t.y == v || t.z == v) continue;
            uint32_t group = clothGroup[v];
            bool same = group != 0u && clothGroup[t.x] == group && clothGroup[t.y] == group && clothGroup[t.z] == group;
            if (same && selfCollision[v] == 0u) continue;
            if (same && (nbr_contains(nbrList, ns, ne, t.x) || nbr_contains(nbrList, ns, ne, t.y) ||
                         nbr_contains(nbrList, ns, ne, t.z)))
                continue;
            F3 lo, hi;
            elem_bounds(entry, lo, hi);
            I3 tc0 = cell_of(lo, elemCellSize), th = cell_of(hi, elemCellSize);
            I3 tc1{std::min(th.x, tc0.x + 3), std::min(th.y, tc0.y + 3), std::min(th.z, tc0.z + 3)};
            if (!in_range(cell, tc0, tc1)) continue;
            F3 bary;
            F3 q = closest_pt_triangle(p, xyz(posLin[t.x]), xyz(posLin[t.y]), xyz(posLin[t.z]), bary);
            F3 d = p - q;
            if (dot(d, d) > query2) continue;
            cand.push_back(entry);
        }
        std::sort(cand.begin(), cand.end());
        for (uint32_t e : cand) append(DAT_PAIR_VT, v, e, DAT_PAIR_TRUNCATE | DAT_PAIR_CONTACT);
    }
    for (uint32_t gid = 0; gid < numEdges; gid++) {
        uint32_t ax = edges[2 * gid], ay = edges[2 * gid + 1];
        F3 a0 = xyz(posLin[ax]), a1 = xyz(posLin[ay]);
        if (!finite3(a0) || !finite3(a1)) { dat.invalidAnchor++; dat.nonfinite++; continue; }
        I3 ac0 = cell_of(vmin3(a0, a1), elemCellSize), ra = cell_of(vmax3(a0, a1), elemCellSize);
        if (ra.x - ac0.x > 3 || ra.y - ac0.y > 3 || ra.z - ac0.z > 3) dat.gridOverflow++;
        I3 ac1{std::min(ra.x, ac0.x + 3), std::min(ra.y, ac0.y + 3), std::min(ra.z, ac0.z + 3)};
        uint32_t ns0 = nbrStart[ax], ne0 = ns0 + nbrCount[ax];
        uint32_t ns1 = nbrStart[ay], ne1 = ns1 + nbrCount[ay];
        std::vector<std::pair<uint32_t, uint32_t>> cand;
        for (int z = ac0.z; z <= ac1.z; z++)
            for (int y = ac0.y; y <= ac1.y; y++)
                for (int x = ac0.x; x <= ac1.x; x++) {
                    I3 cell{x, y, z};
                    uint32_t h = elem_hash(cell, elemHashSize);
                    uint32_t s0 = elemCellStart[h], e0 = s0 + elemCellCount[h];
                    for (uint32_t k = s0; k < e0; k++) {
                        uint32_t entry = elemCells[k];
                        if ((entry & ELEM_EDGE_BIT) == 0u) continue;
                        uint32_t other = entry & ~ELEM_EDGE_BIT;
                        if (other <= gid || other >= numEdges) continue;
                        uint32_t bx = edges[2 * other], by = edges[2 * other + 1];
                        if (bx == ax || bx == ay || by == ax || by == ay) continue;
                        uint32_t group = clothGroup[ax];
                        bool same = group != 0u && clothGroup[ay] == group && clothGroup[bx] == group &&
                                    clothGroup[by] == group;
                        if (same && selfCollision[ax] == 0u) continue;
                        if (same && (nbr_contains(nbrList, ns0, ne0, bx) || nbr_contains(nbrList, ns0, ne0, by) ||
                                     nbr_contains(nbrList, ns1, ne1, bx) || nbr_contains(nbrList, ns1, ne1, by)))
                            continue;
                        F3 blo, bhi;
                        elem_bounds(numTris + other, blo, bhi);
                        I3 bc0 = cell_of(blo, elemCellSize), bh = cell_of(bhi, elemCellSize);
                        I3 bc1{std::min(bh.x, bc0.x + 3), std::min(bh.y, bc0.y + 3), std::min(bh.z, bc0.z + 3)};
                        I3 o0{std::max(ac0.x, bc0.x), std::max(ac0.y, bc0.y), std::max(ac0.z, bc0.z)};
                        I3 o1{std::min(ac1.x, bc1.x), std::min(ac1.y, bc1.y), std::min(ac1.z, bc1.z)};
                        if (o0.x > o1.x || o0.y > o1.y || o0.z > o1.z) continue;
                        if (cell.x != o0.x || cell.y != o0.y || cell.z != o0.z) continue;
                        float sb, tb;
                        F3 b0 = xyz(posLin[bx]), b1 = xyz(posLin[by]);
                        closest_seg_seg_st(a0, a1, b0, b1, sb, tb);
                        F3 ca = a0 + (a1 - a0) * sb, cb = b0 + (b1 - b0) * tb;
                        F3 d = ca - cb;
                        if (dot(d, d) > query2) continue;
                        uint32_t flags = DAT_PAIR_TRUNCATE;
                        if ((gid < numSurfaceEdges && other < numSurfaceEdges) || (same && selfCollision[ax] != 0u))
                            flags |= DAT_PAIR_CONTACT;
                        cand.push_back({other, flags});
                    }
                }
        std::sort(cand.begin(), cand.end());
        for (auto& c : cand) append(DAT_PAIR_EE, gid, c.first, c.second);
    }
    dat.pairsPeak = std::max(dat.pairsPeak, datRaw);
    dat.vtPeak = std::max(dat.vtPeak, datVT);
    dat.eePeak = std::max(dat.eePeak, datEE);
}

// ==========================================================================
// Soft persistence map and emission (25_cloth.metal:79-145, :269-355)
// ==========================================================================
int Solver::soft_map_find(uint32_t keyA, uint32_t keyB) const {
    uint32_t h = soft_key_hash(keyA, keyB, softMapCapacity);
    for (uint32_t probe = 0; probe < 64; probe++) {
        uint32_t ka = softKeyA[h];
        if (ka == 0) return -1;
        if (ka == keyA + 1 && softKeyB[h] == keyB) return (int)softVal[h];
        h = (h + 1) & (softMapCapacity - 1u);
    }
    return -1;
}

float Solver::soft_prev_side(uint32_t keyA, uint32_t keyB, float proposed) const {
    int prev = soft_map_find(keyA, keyB);
    if (prev < 0) return proposed;
    uint32_t flags = fbits(prevSoft[prev].anchorA.w);
    return (flags & SCF_SIDE_NEG) ? -1.0f : 1.0f;
}

static inline float soft_lambda_cap(const Params& P, float minMass) {
    return fmin_(P.lambdaMax, fmax_(10.0f, 1.0e5f * minMass));
}

void Solver::soft_emit(U4 ids, F4 weights, F3 n, float friction, F3 anchorA, float C0n, float restT,
                       float lamCap, float minMass, uint32_t kind, bool rigidA, bool roundA, bool sideNeg,
                       uint32_t keyA, uint32_t keyB) {
    F3 lam = f3s(0), pen = f3s(0);
    int prev = soft_map_find(keyA, keyB);
    if (prev >= 0) {
        lam = xyz(prevSoft[prev].lambda) * (P.alpha * P.gamma);
        pen = xyz(prevSoft[prev].penalty);
        F3 nOld = xyz(prevSoft[prev].normal);
        F3 t1o, t2o, t1n, t2n;
        orthonormal(nOld, t1o, t2o);
        orthonormal(n, t1n, t2n);
        F3 lt = t1o * lam.y + t2o * lam.z;
        lam.y = dot(t1n, lt);
        lam.z = dot(t2n, lt);
    }
    float penFloor = fmax_(PENALTY_MIN, minMass / (P.dt * P.dt));
    pen = clamp3(pen * P.gamma, f3s(penFloor), f3s(PENALTY_MAX));
    uint32_t slot = softRaw++;
    if (slot >= maxSoft) return;
    uint32_t flags = (rigidA ? SCF_RIGID_A : 0u) | (sideNeg ? SCF_SIDE_NEG : 0u) | (kind << SCF_KIND_SHIFT) |
                     (roundA ? SCF_ROUND_A : 0u);
    SoftContactGPU& sc = soft[slot];
    sc.ids = ids;
    sc.normal = f4(n, friction);
    sc.anchorA = f4(rigidA ? anchorA : f3(restT, 0, 0), bitsf(flags));
    sc.weights = weights;
    sc.C0 = f4(C0n, 0, 0, lamCap);
    sc.lambda = f4(lam, bitsf(keyA));
    sc.penalty = f4(pen, bitsf(keyB));
}

// Rigid feature points vs triangles (25_cloth.metal:942-1142).  Bodies are
// visited by their collider's owner.  The grid sweep visits each distinct
// hash bucket once.
void Solver::rt_emit() {
    struct Feat { F3 world; float radius; uint32_t id; };
    for (uint32_t gid = 0; gid < numTris; gid++) {
        U4 tid = tris[gid];
        F3 a = xyz(posLin[tid.x]), b = xyz(posLin[tid.y]), c = xyz(posLin[tid.z]);
        F3 m = (a + b + c) / 3.0f;
        float rt_ = fmax_(std::fabs(shape[tid.x].w), fmax_(std::fabs(shape[tid.y].w), std::fabs(shape[tid.z].w)));
        float rT = fmax_(distance(m, a), fmax_(distance(m, b), distance(m, c))) + rt_;
        F3 triN = cross(b - a, c - a);
        float tnLen = length(triN);
        if (tnLen < 1e-12f) continue;
        triN = triN / tnLen;
        F3 velT = (xyz(velLin[tid.x]) + xyz(velLin[tid.y]) + xyz(velLin[tid.z])) / 3.0f;
        uint32_t emitted = 0;
        auto test_body = [&](uint32_t o) {
            float rb = std::fabs(shape[o].w);
            F3 po = xyz(posLin[o]);
            F4 qo = posAng[o];
            uint32_t st = shapeType[o];
            bool nearO = distance(po, m) <= rT + rb + P.collisionMargin;
            if (nearO && st == AVBD_SHAPE_BOX) {
                F3 lm = q_rotate(q_conj(qo), m - po);
                F3 dq2 = fmax3(abs3(lm) - xyz(shape[o]) * 0.5f, f3s(0.0f));
                nearO = length(dq2) <= rT + P.collisionMargin + 0.05f;
            }
            if (!nearO) return;
            bool excl = pair_excluded_bodies(std::min(o, tid.x), std::max(o, tid.x)) ||
                        pair_excluded_bodies(std::min(o, tid.y), std::max(o, tid.y)) ||
                        pair_excluded_bodies(std::min(o, tid.z), std::max(o, tid.z));
            if (excl) return;
            Feat feats[4];
            int nf = 0;
            if (st == AVBD_SHAPE_SPHERE) {
                feats[0] = Feat{po, shape[o].x * 0.5f, 8};
                nf = 1;
            } else if (st == AVBD_SHAPE_CAPSULE) {
                // three spheres along the axis; a torus has none (25_cloth.metal:957-971)
                float half_ = shape[o].x * 0.5f, r = shape[o].y;
                F3 ax = q_rotate(qo, f3(0, 0, 1));
                for (int i = -1; i <= 1; i++) {
                    F3 w = po + ax * (half_ * (float)i);
                    if (distance(w, m) > rT + r + 4.0f * P.collisionMargin) continue;
                    feats[nf++] = Feat{w, r, (uint32_t)(9 + i + 1)};
                }
            } else if (st == AVBD_SHAPE_BOX) {
                F3 h3 = xyz(shape[o]) * 0.5f;
                for (uint32_t i = 0; i < 8; i++) {
                    F3 local = f3((i & 1) ? h3.x : -h3.x, (i & 2) ? h3.y : -h3.y, (i & 4) ? h3.z : -h3.z);
                    F3 w = xform(po, qo, local);
                    if (distance(w, m) > rT + 4.0f * P.collisionMargin) continue;
                    if (nf < 4) feats[nf++] = Feat{w, 0.0f, i};
                }
            }
            for (int fi = 0; fi < nf && emitted < RT_MAX_PER_TRI; fi++) {
                F3 bary;
                F3 q = closest_pt_triangle(feats[fi].world, a, b, c, bary);
                F3 d = feats[fi].world - q;
                float dist = length(d);
                float hSum = rt_ + feats[fi].radius;
                float inflate = fmin_(length(xyz(velLin[o]) - velT) * P.dt, 0.5f * rT);
                if (dist - hSum > elemMargin + inflate) continue;
                float side = dot(d, triN) >= 0.0f ? 1.0f : -1.0f;
                uint32_t keyA = (SC_RT << 28) | o;
                uint32_t keyB = gid * 16u + feats[fi].id;
                float proposed = dot(po - q, triN) >= 0.0f ? 1.0f : -1.0f;
                bool interior = bary.x > 0.02f && bary.y > 0.02f && bary.z > 0.02f;
                float sMem = interior ? soft_prev_side(keyA, keyB, proposed) : proposed;
                F3 n;
                float g;
                if (dist > 1e-7f && side == sMem) { n = d / dist; g = dist; }
                else { n = triN * sMem; g = -dist; }
                float fricT = (props[tid.x].w + props[tid.y].w + props[tid.z].w) / 3.0f;
                float friction = std::sqrt(fmax_(props[o].w * fricT, 0.0f));
                float minMass = posLin[o].w > 0.0f ? posLin[o].w : FLT_MAX;
                float mA = posLin[tid.x].w, mB = posLin[tid.y].w, mC = posLin[tid.z].w;
                if (mA > 0.0f) minMass = fmin_(minMass, mA);
                if (mB > 0.0f) minMass = fmin_(minMass, mB);
                if (mC > 0.0f) minMass = fmin_(minMass, mC);
                if (minMass == FLT_MAX) continue;
                bool roundA = st != AVBD_SHAPE_BOX;
                F3 anchor = roundA ? (feats[fi].world - po) : q_rotate(q_conj(qo), feats[fi].world - po);
                soft_emit(U4{o, tid.x, tid.y, tid.z}, f4(1.0f, -bary.x, -bary.y, -bary.z), n, friction, anchor,
                          g - hSum + elemMargin, hSum - elemMargin, soft_lambda_cap(P, minMass), minMass, SC_RT,
                          true, roundA, sMem < 0.0f, keyA, keyB);
                emitted++;
            }
        };
        if (P.numHashedRigid > 0 && P.numHashedRigid <= 8) {
            for (uint32_t ri = 0; ri < P.numHashedRigid && emitted < RT_MAX_PER_TRI; ri++)
                test_body(colOwner[hashedRigidIdx[ri]]);
        } else if (P.numHashedRigid > 0) {
            int R = std::min(4, std::max(1, (int)std::ceil((rT + 0.5f * P.cellSize) / P.cellSize)));
            int cx, cy, cz;
            cell_coord(m, P.cellSize, cx, cy, cz);
            std::vector<uint32_t> seen;
            for (int dz = -R; dz <= R && emitted < RT_MAX_PER_TRI; dz++)
                for (int dy = -R; dy <= R && emitted < RT_MAX_PER_TRI; dy++)
                    for (int dx = -R; dx <= R && emitted < RT_MAX_PER_TRI; dx++) {
                        uint32_t h = cell_hash(cx + dx, cy + dy, cz + dz, 0u, P.gridHashSize);
                        if (std::find(seen.begin(), seen.end(), h) != seen.end()) continue;
                        seen.push_back(h);
                        uint32_t s0 = cellStart[h], e0 = s0 + cellCount[h];
                        for (uint32_t k = s0; k < e0 && emitted < RT_MAX_PER_TRI; k++) {
                            uint32_t o = colOwner[cellBodies[k]];
                            if (shape[o].w < 0.0f) continue;
                            test_body(o);
                        }
                    }
        }
        for (uint32_t g = 0; g < P.numGlobals && emitted < RT_MAX_PER_TRI; g++) {
            uint32_t o = colOwner[globalIdx[g]];
            if (shape[o].w < 0.0f) continue;
            test_body(o);
        }
    }
}

static F3 dat_vt_fallback_normal(F3 a, F3 b, F3 c, F3 rel, bool& valid) {
    F3 raw = cross(b - a, c - a);
    float mag = length(raw);
    valid = finite_bits(mag) && mag >= DAT_GEOMETRY_EPS;
    if (!valid) return f3s(0);
    F3 n = raw / mag;
    if (dot(n, rel) > 0.0f) n = -n;
    return n;
}

static F3 dat_ee_fallback_normal(F3 a0, F3 a1, F3 b0, F3 b1, F3 rel, bool& valid) {
    F3 ua = a1 - a0, ub = b1 - b0;
    F3 raw = cross(ua, ub);
    float mag = length(raw);
    F3 n;
    if (finite_bits(mag) && mag >= DAT_GEOMETRY_EPS) {
        n = raw / mag;
    } else {
        float la = length(ua), lb = length(ub);
        F3 u = la >= lb ? ua : ub;
        float ul = fmax_(la, lb);
        if (!finite_bits(ul) || ul < DAT_GEOMETRY_EPS) { valid = false; return f3s(0); }
        u = u / ul;
        F3 perp = rel - u * dot(u, rel);
        float pl = length(perp);
        if (!finite_bits(pl) || pl < DAT_GEOMETRY_EPS) {
            F3 axis = std::fabs(u.x) < 0.7f ? f3(1, 0, 0) : f3(0, 1, 0);
            perp = cross(u, axis);
            pl = length(perp);
        }
        if (!finite_bits(pl) || pl < DAT_GEOMETRY_EPS) { valid = false; return f3s(0); }
        n = perp / pl;
    }
    if (dot(n, rel) > 0.0f) n = -n;
    valid = finite3(n);
    return valid ? n : f3s(0);
}

// Pair-parallel OGC contact emission at the accepted pose
// (27_planar_dat.metal:344-510); reference positions are initLin.
void Solver::dat_emit_contacts() {
    const uint32_t count = (uint32_t)datPairs.size();
    for (uint32_t gid = 0; gid < count; gid++) {
        U4 pair = datPairs[gid];
        if ((pair.w & DAT_PAIR_CONTACT) == 0u) continue;
        if (pair.x == DAT_PAIR_VT) {
            uint32_t v = pair.y, ti = pair.z;
            if (ti >= numTris) continue;
            U4 t = tris[ti];
            F3 p = xyz(posLin[v]);
            F3 a = xyz(posLin[t.x]), b = xyz(posLin[t.y]), c = xyz(posLin[t.z]);
            F3 bary;
            F3 q = closest_pt_triangle(p, a, b, c, bary);
            F3 d = p - q;
            float dist2 = dot(d, d);
            float rv = std::fabs(shape[v].w);
            float rt = fmax_(std::fabs(shape[t.x].w), fmax_(std::fabs(shape[t.y].w), std::fabs(shape[t.z].w)));
            float hSum = rv + rt;
            F3 velT = (xyz(velLin[t.x]) + xyz(velLin[t.y]) + xyz(velLin[t.z])) / 3.0f;
            float inflate = fmin_(length(xyz(velLin[v]) - velT) * P.dt, 0.3f * surfaceCellSize);
            float detect = fmin_(hSum + elemMargin + inflate, queryRadius);
            if (dist2 > detect * detect) continue;
            float dist = std::sqrt(dist2);
            F3 triN = cross(b - a, c - a);
            float nl = length(triN);
            if (nl < DAT_GEOMETRY_EPS) continue;
            triN = triN / nl;
            float side = dot(d, triN) >= 0.0f ? 1.0f : -1.0f;
            uint32_t keyA = (SC_VT << 28) | v, keyB = ti;
            bool interior = bary.x > 0.02f && bary.y > 0.02f && bary.z > 0.02f;
            float remembered = interior ? soft_prev_side(keyA, keyB, side) : side;
            F3 n;
            float gap;
            if (dist > 1.0e-7f && side == remembered) { n = d / dist; gap = dist; }
            else { n = triN * remembered; gap = -dist; }
            float fricT = props[t.x].w * bary.x + props[t.y].w * bary.y + props[t.z].w * bary.z;
            float friction = std::sqrt(fmax_(props[v].w * fricT, 0.0f));
            float minMass = posLin[v].w > 0.0f ? posLin[v].w : FLT_MAX;
            const uint32_t ids[4] = {v, t.x, t.y, t.z};
            for (int j = 1; j < 4; j++) {
                float mm = posLin[ids[j]].w;
                if (mm > 0.0f) minMass = fmin_(minMass, mm);
            }
            if (minMass == FLT_MAX) continue;
            F3 dq = (p - xyz(initLin[v])) - (a - xyz(initLin[t.x])) * bary.x - (b - xyz(initLin[t.y])) * bary.y -
                    (c - xyz(initLin[t.z])) * bary.z;
            float Cdetect = gap - hSum + elemMargin;
            float C0n = Cdetect - dot(n, dq);
            soft_emit(U4{v, t.x, t.y, t.z}, f4(1.0f, -bary.x, -bary.y, -bary.z), n, friction, f3s(0), C0n,
                      hSum - elemMargin, soft_lambda_cap(P, minMass), minMass, SC_VT, false, false,
                      remembered < 0.0f, keyA, keyB);
            continue;
        }
        uint32_t ea = pair.y, eb = pair.z;
        if (ea >= numEdges || eb >= numEdges) continue;
        uint32_t ax = edges[2 * ea], ay = edges[2 * ea + 1], bx = edges[2 * eb], by = edges[2 * eb + 1];
        F3 a0 = xyz(posLin[ax]), a1 = xyz(posLin[ay]), b0 = xyz(posLin[bx]), b1 = xyz(posLin[by]);
        float s, t;
        closest_seg_seg_st(a0, a1, b0, b1, s, t);
        if (s < EE_INTERIOR_EPS || s > 1.0f - EE_INTERIOR_EPS || t < EE_INTERIOR_EPS || t > 1.0f - EE_INTERIOR_EPS)
            continue;
        F3 ca = a0 + (a1 - a0) * s, cb = b0 + (b1 - b0) * t;
        F3 d = ca - cb;
        float dist = length(d);
        float rA = fmax_(std::fabs(shape[ax].w), std::fabs(shape[ay].w));
        float rB = fmax_(std::fabs(shape[bx].w), std::fabs(shape[by].w));
        float hSum = rA + rB;
        F3 va = (xyz(velLin[ax]) + xyz(velLin[ay])) * 0.5f;
        F3 vb = (xyz(velLin[bx]) + xyz(velLin[by])) * 0.5f;
        float inflate = fmin_(length(va - vb) * P.dt, 0.3f * surfaceCellSize);
        float detect = fmin_(hSum + elemMargin + inflate, queryRadius);
        if (dist > detect) continue;
        uint32_t keyA = (SC_EE << 28) | ea, keyB = eb;
        int previous = soft_map_find(keyA, keyB);
        F3 n;
        float gap = dist;
        if (finite_bits(dist) && dist >= 1.0e-7f) {
            F3 nGeo = d / dist;
            n = nGeo;
            if (previous >= 0 && dot(nGeo, xyz(prevSoft[previous].normal)) < 0.0f) { n = -nGeo; gap = -dist; }
        } else if (previous >= 0 && finite3(xyz(prevSoft[previous].normal))) {
            n = xyz(prevSoft[previous].normal);
            gap = 0.0f;
        } else {
            bool ok;
            n = dat_ee_fallback_normal(a0, a1, b0, b1, va - vb, ok);
            if (!ok) continue;
            gap = 0.0f;
        }
        float friction = std::sqrt(fmax_((props[ax].w + props[ay].w) * 0.5f * (props[bx].w + props[by].w) * 0.5f, 0.0f));
        float minMass = FLT_MAX;
        const uint32_t ids[4] = {ax, ay, bx, by};
        for (int j = 0; j < 4; j++) {
            float mm = posLin[ids[j]].w;
            if (mm > 0.0f) minMass = fmin_(minMass, mm);
        }
        if (minMass == FLT_MAX) continue;
        F3 dq = (a0 - xyz(initLin[ax])) * (1.0f - s) + (a1 - xyz(initLin[ay])) * s -
                (b0 - xyz(initLin[bx])) * (1.0f - t) - (b1 - xyz(initLin[by])) * t;
        float Cdetect = gap - hSum + elemMargin;
        float C0n = Cdetect - dot(n, dq);
        soft_emit(U4{ax, ay, bx, by}, f4(1.0f - s, s, -(1.0f - t), -t), n, friction, f3s(0), C0n,
                  hSum - elemMargin, soft_lambda_cap(P, minMass), minMass, SC_EE, false, false, false, keyA, keyB);
    }
}

// Clamp the soft count and rebuild the map (soft_finalize, softmap_clear,
// softmap_insert).  A key that is already present keeps its first record.
void Solver::soft_map_rebuild() {
    dat.softCandidates = softRaw;
    numSoft = std::min(softRaw, maxSoft);
    std::fill(softKeyA.begin(), softKeyA.end(), 0u);
    for (uint32_t i = 0; i < numSoft; i++) {
        uint32_t keyA = fbits(soft[i].lambda.w), keyB = fbits(soft[i].penalty.w);
        uint32_t h = soft_key_hash(keyA, keyB, softMapCapacity);
        for (uint32_t probe = 0; probe < softMapCapacity; probe++) {
            if (softKeyA[h] == 0u) {
                softKeyA[h] = keyA + 1;
                softKeyB[h] = keyB;
                softVal[h] = i;
                break;
            }
            if (softKeyA[h] == keyA + 1 && softKeyB[h] == keyB) break;
            h = (h + 1) & (softMapCapacity - 1u);
        }
    }
}

// ==========================================================================
// Planar-DAT passes (27_planar_dat.metal:525-561, :752-946, :1179-1310)
// ==========================================================================
bool Solver::dat_unsafe() const {
    return datRaw > maxDatPairs || dat.pairsPeak > maxDatPairs || dat.gridOverflow > 0 || dat.invalidAnchor > 0;
}

F3 Solver::cur_pos(uint32_t b, uint32_t activeColor) const {
    if (colorJacobi && activeColor != FULL_PASS && posLin[b].w > 0.0f && colorsA[b] == activeColor)
        return xyz(posNext[b]);
    return xyz(posLin[b]);
}

static float dat_plane_fraction(F3 x, F3 dx, F3 n, F3 plane, float side, float gamma,
                                Solver::DatCounters& ctr, bool report) {
    float s0 = side * dot(n, x - plane);
    float q = side * dot(n, dx);
    if (!finite_bits(s0) || !finite_bits(q)) {
        if (report) { ctr.invalidAnchor++; ctr.nonfinite++; }
        return 0.0f;
    }
    if (s0 < -DAT_GEOMETRY_EPS) return 0.0f;
    if (q >= 0.0f || s0 + q > 0.0f) return 1.0f;
    float hit = fmax_(s0, 0.0f) / (-q);
    if (hit > 1.0f + DAT_GEOMETRY_EPS) return 1.0f;
    return clampf_(fmin_(gamma * hit, hit - DAT_TIME_MARGIN), 0.0f, 1.0f);
}

void Solver::dat_reduce(uint32_t activeColor) {
    const float relax = P.planarDATRelaxation;
    const bool full = activeColor == FULL_PASS;
    auto active = [&](uint32_t b) { return full || (posLin[b].w > 0.0f && colorsA[b] == activeColor); };
    auto tmin = [&](uint32_t b, float t) { if (fbits(t) < truncBits[b]) truncBits[b] = fbits(t); };
    auto atomic_t = [&](uint32_t b, F3 x, F3 dx, F3 n, F3 plane, float side) {
        float t = dat_plane_fraction(x, dx, n, plane, side, relax, dat, true);
        if (t < 1.0f) tmin(b, t);
    };
    const uint32_t count = (uint32_t)datPairs.size();
    for (uint32_t gid = 0; gid < count; gid++) {
        U4 pair = datPairs[gid];
        if ((pair.w & DAT_PAIR_TRUNCATE) == 0u) continue;
        if (pair.x == DAT_PAIR_VT) {
            uint32_t v = pair.y;
            U4 t = tris[pair.z];
            bool aV = active(v), aA = active(t.x), aB = active(t.y), aC = active(t.z);
            if (!aV && !aA && !aB && !aC) continue;
            F3 xv = xyz(ogcPrev[v]);
            F3 a = xyz(ogcPrev[t.x]), b = xyz(ogcPrev[t.y]), c = xyz(ogcPrev[t.z]);
            F3 bary;
            F3 cp = closest_pt_triangle(xv, a, b, c, bary);
            F3 nh = xv - cp;
            float gap = length(nh);
            if (!finite_bits(gap)) {
                dat.invalidAnchor++; dat.nonfinite++;
                tmin(v, 0.0f); tmin(t.x, 0.0f); tmin(t.y, 0.0f); tmin(t.z, 0.0f);
                continue;
            }
            if (gap > queryRadius) continue;
            F3 dv = cur_pos(v, activeColor) - xv;
            F3 da = cur_pos(t.x, activeColor) - a;
            F3 db = cur_pos(t.y, activeColor) - b;
            F3 dc = cur_pos(t.z, activeColor) - c;
            F3 n;
            if (gap >= DAT_GEOMETRY_EPS) {
                n = nh / gap;
            } else {
                bool ok;
                n = dat_vt_fallback_normal(a, b, c, dv - (da + db + dc) / 3.0f, ok);
                if (!ok) {
                    dat.invalidAnchor++; dat.vtDegenerate++;
                    tmin(v, 0.0f); tmin(t.x, 0.0f); tmin(t.y, 0.0f); tmin(t.z, 0.0f);
                    continue;
                }
                dat.vtDegenerate++;
            }
            float approachV = fmax_(-dot(n, dv), 0.0f);
            float approachT = fmax_(fmax_(dot(n, da), dot(n, db)), fmax_(dot(n, dc), 0.0f));
            float lambda = approachV + approachT == 0.0f ? 0.5f
                                                         : clampf_(approachT / (approachV + approachT), 0.05f, 0.95f);
            F3 plane = gap >= DAT_GEOMETRY_EPS ? cp + nh * lambda : cp;
            if (approachV > 0.0f && aV) atomic_t(v, xv, dv, n, plane, 1.0f);
            if (approachT > 0.0f) {
                if (aA) atomic_t(t.x, a, da, n, plane, -1.0f);
                if (aB) atomic_t(t.y, b, db, n, plane, -1.0f);
                if (aC) atomic_t(t.z, c, dc, n, plane, -1.0f);
            }
            continue;
        }
        uint32_t ax = edges[2 * pair.y], ay = edges[2 * pair.y + 1];
        uint32_t bx = edges[2 * pair.z], by = edges[2 * pair.z + 1];
        bool aA0 = active(ax), aA1 = active(ay), aB0 = active(bx), aB1 = active(by);
        if (!aA0 && !aA1 && !aB0 && !aB1) continue;
        F3 a0 = xyz(ogcPrev[ax]), a1 = xyz(ogcPrev[ay]), b0 = xyz(ogcPrev[bx]), b1 = xyz(ogcPrev[by]);
        float s, t;
        closest_seg_seg_st(a0, a1, b0, b1, s, t);
        F3 ca = a0 + (a1 - a0) * s, cb = b0 + (b1 - b0) * t;
        F3 nh = ca - cb;
        float gap = length(nh);
        if (!finite_bits(gap)) {
            dat.invalidAnchor++; dat.nonfinite++;
            tmin(ax, 0.0f); tmin(ay, 0.0f); tmin(bx, 0.0f); tmin(by, 0.0f);
            continue;
        }
        if (gap > queryRadius) continue;
        F3 da0 = cur_pos(ax, activeColor) - a0, da1 = cur_pos(ay, activeColor) - a1;
        F3 db0 = cur_pos(bx, activeColor) - b0, db1 = cur_pos(by, activeColor) - b1;
        F3 n;
        if (gap > DAT_GEOMETRY_EPS) {
            n = nh / gap;
        } else {
            bool ok;
            n = dat_ee_fallback_normal(a0, a1, b0, b1, (da0 + da1 - db0 - db1) * 0.5f, ok);
            if (!ok) {
                dat.invalidAnchor++; dat.eeDegenerate++;
                tmin(ax, 0.0f); tmin(ay, 0.0f); tmin(bx, 0.0f); tmin(by, 0.0f);
                continue;
            }
            dat.eeDegenerate++;
        }
        float approachA = fmax_(fmax_(-dot(n, da0), -dot(n, da1)), 0.0f);
        float approachB = fmax_(fmax_(dot(n, db0), dot(n, db1)), 0.0f);
        float lambda = approachA + approachB == 0.0f ? 0.5f
                                                     : clampf_(approachB / (approachA + approachB), 0.05f, 0.95f);
        F3 plane = gap > DAT_GEOMETRY_EPS ? cb + nh * lambda : cb;
        if (approachA > 0.0f) {
            if (aA0) atomic_t(ax, a0, da0, n, plane, 1.0f);
            if (aA1) atomic_t(ay, a1, da1, n, plane, 1.0f);
        }
        if (approachB > 0.0f) {
            if (aB0) atomic_t(bx, b0, db0, n, plane, -1.0f);
            if (aB1) atomic_t(by, b1, db1, n, plane, -1.0f);
        }
    }
}

// Consume the reduced fraction of one vertex and move it along its
// displacement since the anchor (dat_apply / dat_apply_color).
static inline bool dat_apply_one(Solver& S, uint32_t v, F3 current, float mass) {
    F3 anchor = xyz(S.ogcPrev[v]);
    F3 d = current - anchor;
    bool unsafe = S.dat_unsafe();
    float t = bitsf(S.truncBits[v]);
    S.truncBits[v] = fbits(1.0f);
    if (unsafe) t = 0.0f;
    if (!finite3(d) || !finite_bits(t)) {
        S.dat.invalidAnchor++; S.dat.nonfinite++;
        d = f3s(0);
        t = 0.0f;
    }
    bool truncated = t < 1.0f;
    d *= clampf_(t, 0.0f, 1.0f);
    float maxD = 0.5f * S.P.planarDATRelaxation * S.queryRadius;
    float d2 = dot(d, d);
    if (d2 > maxD * maxD) {
        d *= maxD * rsqrt_(d2);
        truncated = true;
    }
    if (truncated) {
        S.posLin[v] = f4(anchor + d, mass);
        S.dat.truncations++;
    }
    return truncated;
}

void Solver::dat_apply_particles() {
    for (uint32_t gid = 0; gid < numParticles; gid++) {
        uint32_t v = particleIdx[gid];
        dat_apply_one(*this, v, xyz(posLin[v]), posLin[v].w);
    }
}

// Commit one color: the pending solve results of its bodies, truncated for
// surface vertices.
void Solver::dat_apply_color(uint32_t c) {
    for (uint32_t i = colorStart[c]; i < colorStart[c + 1]; i++) {
        uint32_t v = colorList[i];
        float mass = posLin[v].w;
        if (clothGroup[v] == 0u) {
            posLin[v] = f4(xyz(posNext[v]), mass);
            posAng[v] = angNext[v];
            continue;
        }
        F3 current = xyz(posNext[v]);
        if (!dat_apply_one(*this, v, current, mass)) posLin[v] = f4(current, mass);
    }
}

void Solver::dat_restore_failed_surface() {
    bool failed = dat.softCandidates > maxSoft || dat.pairsPeak > maxDatPairs || dat.gridOverflow > 0 ||
                  dat.invalidAnchor > 0;
    if (!failed) return;
    for (uint32_t b = 0; b < nb; b++)
        if (shape[b].w < 0.0f) posLin[b] = f4(xyz(initLin[b]), posLin[b].w);
}

void Solver::smooth_particle_velocities() {
    std::vector<F4> velRead = velLin;
    for (uint32_t gid = 0; gid < numParticles; gid++) {
        uint32_t v = particleIdx[gid];
        uint32_t s0 = nbrStart[v], n = nbrCount[v];
        if (n == 0) continue;
        F3 avg = f3s(0);
        for (uint32_t k = s0; k < s0 + n; k++) avg += xyz(velRead[nbrList[k]]);
        avg = avg / (float)n;
        F3 vel = xyz(velRead[v]);
        velLin[v] = f4(vel + (avg - vel) * clothViscosity, 0.0f);
    }
}

// ==========================================================================
// Stamps and dual (40_solver.metal:1088-1153, :1236-1359, :1689-1727)
// ==========================================================================
void Solver::stamp_membrane(const MembraneGPU& mb, uint32_t self, Accum& acc) const {
    F3 x0 = xyz(posLin[mb.ids.x]), x1 = xyz(posLin[mb.ids.y]), x2 = xyz(posLin[mb.ids.z]);
    float muA = mb.mat.x, lamA = mb.mat.y;
    F3 d0 = x1 - x0, d1 = x2 - x0;
    float a = mb.dm.x, b = mb.dm.y, c = mb.dm.z, d = mb.dm.w;
    F3 f1 = d0 * a + d1 * b;
    F3 f2 = d0 * c + d1 * d;
    float E11 = 0.5f * (dot(f1, f1) - 1.0f);
    float E22 = 0.5f * (dot(f2, f2) - 1.0f);
    float E12 = 0.5f * dot(f1, f2);
    float trE = E11 + E22;
    float S11 = 2.0f * muA * E11 + lamA * trE;
    float S22 = 2.0f * muA * E22 + lamA * trE;
    float S12 = 2.0f * muA * E12;
    F3 p1 = f1 * S11 + f2 * S12;
    F3 p2 = f1 * S12 + f2 * S22;
    float wx, wy;
    if (self == mb.ids.y) { wx = a; wy = c; }
    else if (self == mb.ids.z) { wx = b; wy = d; }
    else { wx = -a - b; wy = -c - d; }
    acc.rhsLin += p1 * wx + p2 * wy;
    F3 g11 = f1 * wx, g22 = f2 * wy;
    F3 g12 = (f2 * wx + f1 * wy) * 0.5f;
    F3 gtr = g11 + g22;
    acc.lhsLin = m3_add(acc.lhsLin, m3_scale(m3_outer(g11, g11), 2.0f * muA));
    acc.lhsLin = m3_add(acc.lhsLin, m3_scale(m3_outer(g22, g22), 2.0f * muA));
    acc.lhsLin = m3_add(acc.lhsLin, m3_scale(m3_outer(g12, g12), 4.0f * muA));
    acc.lhsLin = m3_add(acc.lhsLin, m3_scale(m3_outer(gtr, gtr), lamA));
}

void Solver::stamp_bend(const BendGPU& bd, uint32_t self, Accum& acc) const {
    float s = bd.mat.x;
    F3 m = xyz(posLin[bd.ids.x]) * bd.K.x + xyz(posLin[bd.ids.y]) * bd.K.y + xyz(posLin[bd.ids.z]) * bd.K.z +
           xyz(posLin[bd.ids.w]) * bd.K.w;
    float k;
    if (self == bd.ids.x) k = bd.K.x;
    else if (self == bd.ids.y) k = bd.K.y;
    else if (self == bd.ids.z) k = bd.K.z;
    else k = bd.K.w;
    acc.rhsLin += m * (s * k);
    acc.lhsLin = m3_add(acc.lhsLin, m3_diag(f3s(s * k * k)));
}

F3 Solver::soft_c(const SoftContactGPU& sc, F3& n, F3& t1, F3& t2, F3& rAW, bool& rigidA) const {
    uint32_t flags = fbits(sc.anchorA.w);
    rigidA = (flags & SCF_RIGID_A) != 0;
    bool roundA = (flags & SCF_ROUND_A) != 0;
    n = xyz(sc.normal);
    orthonormal(n, t1, t2);
    rAW = f3s(0);
    F3 C = xyz(sc.C0) * (1.0f - P.alpha);
    const uint32_t ids[4] = {sc.ids.x, sc.ids.y, sc.ids.z, sc.ids.w};
    const float ws[4] = {sc.weights.x, sc.weights.y, sc.weights.z, sc.weights.w};
    for (int k = 0; k < 4; k++) {
        uint32_t b = ids[k];
        if (b == WORLD_BODY) continue;
        float w = ws[k];
        F3 dq = xyz(posLin[b]) - xyz(initLin[b]);
        C += f3(dot(n, dq), dot(t1, dq), dot(t2, dq)) * w;
        if (k == 0 && rigidA) {
            rAW = roundA ? xyz(sc.anchorA) : q_rotate(posAng[b], xyz(sc.anchorA));
            F3 dqa = q_sub(posAng[b], initAng[b]);
            C += f3(dot(cross(rAW, n), dqa), dot(cross(rAW, t1), dqa), dot(cross(rAW, t2), dqa)) * w;
        }
    }
    return C;
}

void Solver::stamp_soft(const SoftContactGPU& sc, uint32_t self, Accum& acc) const {
    F3 n, t1, t2, rAW;
    bool rigidA;
    F3 C = soft_c(sc, n, t1, t2, rAW, rigidA);
    // softContactForce (40_solver.metal:1265-1312), barrier stage active
    F3 F = xyz(sc.penalty) * C + xyz(sc.lambda);
    float kN = sc.penalty.x;
    float rT = sc.anchorA.x;
    uint32_t kindB = (fbits(sc.anchorA.w) >> SCF_KIND_SHIFT) & 3u;
    if (rT > 0.0f && kindB != SC_RT && C.x < -0.5f * rT) {
        float dsep = fmax_(C.x + rT, 0.02f * rT);
        float kp = 0.25f * rT * rT * sc.penalty.x;
        F.x = -kp / dsep + sc.lambda.x;
        kN = kp / (dsep * dsep);
    }
    F.x = fmin_(F.x, 0.0f);
    float bounds = std::fabs(F.x) * sc.normal.w;
    float fs = std::sqrt(F.y * F.y + F.z * F.z);
    if (fs > bounds && fs > 0.0f) {
        float r = bounds / fs;
        F.y *= r;
        F.z *= r;
    }
    int slot = -1;
    const uint32_t ids[4] = {sc.ids.x, sc.ids.y, sc.ids.z, sc.ids.w};
    for (int k = 0; k < 4; k++) if (ids[k] == self) { slot = k; break; }
    if (slot < 0) return;
    const float ws[4] = {sc.weights.x, sc.weights.y, sc.weights.z, sc.weights.w};
    float w = ws[slot];
    if (slot == 0 && rigidA) {
        M3 jLin = M3{n * w, t1 * w, t2 * w};
        M3 jAng = M3{cross(rAW, jLin.r0), cross(rAW, jLin.r1), cross(rAW, jLin.r2)};
        M3 K = m3_diag(f3(kN, sc.penalty.y, sc.penalty.z));
        M3 jLinT = m3_transpose(jLin), jAngT = m3_transpose(jAng);
        M3 jAngTk = m3_mulm(jAngT, K);
        acc.lhsLin = m3_add(acc.lhsLin, m3_mulm(m3_mulm(jLinT, K), jLin));
        acc.lhsAng = m3_add(acc.lhsAng, m3_mulm(jAngTk, jAng));
        acc.lhsCross = m3_add(acc.lhsCross, m3_mulm(jAngTk, jLin));
        acc.rhsLin += m3_mul(jLinT, F);
        acc.rhsAng += m3_mul(jAngT, F);
    } else {
        float w2 = w * w;
        acc.lhsLin = m3_add(acc.lhsLin, m3_scale(m3_outer(n, n), kN * w2));
        acc.lhsLin = m3_add(acc.lhsLin, m3_scale(m3_outer(t1, t1), sc.penalty.y * w2));
        acc.lhsLin = m3_add(acc.lhsLin, m3_scale(m3_outer(t2, t2), sc.penalty.z * w2));
        acc.rhsLin += (n * F.x + t1 * F.y + t2 * F.z) * w;
    }
}

void Solver::dual_soft(uint32_t i) {
    SoftContactGPU& sc = soft[i];
    F3 n, t1, t2, rAW;
    bool rigidA;
    F3 C = soft_c(sc, n, t1, t2, rAW, rigidA);
    F3 F = xyz(sc.penalty) * C + xyz(sc.lambda);
    F.x = fmin_(F.x, 0.0f);
    float bnd = std::fabs(F.x) * sc.normal.w;
    float fs = std::sqrt(F.y * F.y + F.z * F.z);
    if (fs > bnd && fs > 0.0f) {
        float r = bnd / fs;
        F.y *= r;
        F.z *= r;
    }
    F.x = fmax_(F.x, -sc.C0.w);
    sc.lambda = f4(F, sc.lambda.w);
    F3 pen = xyz(sc.penalty);
    if (F.x < 0.0f) pen.x = fmin_(pen.x + P.betaLin * std::fabs(C.x), PENALTY_MAX_T);
    if (fs <= bnd) {
        pen.y = fmin_(pen.y + P.betaLin * std::fabs(C.y), PENALTY_MAX_T);
        pen.z = fmin_(pen.z + P.betaLin * std::fabs(C.z), PENALTY_MAX_T);
    }
    sc.penalty = f4(pen, sc.penalty.w);
}

}  // namespace oracle

// ==========================================================================
// Isotropic OGC (25_cloth.metal:147-267 isotropic cover, :347-931)
// ==========================================================================
namespace oracle {

static const uint32_t NONE = 0xFFFFFFFFu;
static const float FBIG = 3.402823466e38f;

struct Best4 {
    uint32_t id[4] = {NONE, NONE, NONE, NONE};
    float d2[4] = {FBIG, FBIG, FBIG, FBIG};
    bool has(uint32_t t) const { return id[0] == t || id[1] == t || id[2] == t || id[3] == t; }
    void insert(uint32_t t, float d) {
        if (d >= d2[3]) return;
        int i = 3;
        for (; i > 0 && d2[i - 1] > d; i--) { id[i] = id[i - 1]; d2[i] = d2[i - 1]; }
        id[i] = t;
        d2[i] = d;
    }
};
static inline uint32_t u4_at(U4 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w)); }

// Tracker topology (GPUSolver.swift:1338-1460): edge-adjacent triangles
// (edges in ascending key order), incident contact edges per vertex, sorted
// 1-ring-plus-2-ring sets, cloth-vertex flags.
void Solver::ogc_topology(const std::vector<std::array<int, 3>>& coll, const std::vector<std::vector<uint32_t>>& ring) {
    std::map<uint64_t, std::pair<int, int>> et;
    for (uint32_t ti = 0; ti < numTris; ti++) {
        const int a = coll[ti][0], b = coll[ti][1], c = coll[ti][2];
        const int pr[3][2] = {{a, b}, {b, c}, {a, c}};
        for (auto& e : pr) {
            uint64_t key = (uint64_t)std::min(e[0], e[1]) << 32 | (uint64_t)std::max(e[0], e[1]);
            auto it = et.find(key);
            if (it == et.end()) et.emplace(key, std::make_pair((int)ti, -1));
            else it->second.second = (int)ti;
        }
    }
    triAdj.assign(std::max<uint32_t>(1, numTris), U4{NONE, NONE, NONE, NONE});
    std::vector<int> fill(std::max<uint32_t>(1, numTris), 0);
    auto put = [&](int t, int o) {
        if (fill[t] >= 3) return;
        uint32_t* sl = &triAdj[t].x;
        sl[fill[t]++] = (uint32_t)o;
    };
    for (auto& kv : et) {
        if (kv.second.second < 0) continue;
        put(kv.second.first, kv.second.second);
        put(kv.second.second, kv.second.first);
    }
    std::vector<std::vector<uint32_t>> ve(nb);
    for (uint32_t i = 0; i < numEdges; i++) { ve[edges[2 * i]].push_back(i); ve[edges[2 * i + 1]].push_back(i); }
    vertEdgeStart.assign(nb, 0); vertEdgeCount.assign(nb, 0); vertEdgeList.clear();
    for (uint32_t i = 0; i < nb; i++) {
        vertEdgeStart[i] = (uint32_t)vertEdgeList.size();
        vertEdgeCount[i] = (uint32_t)ve[i].size();
        vertEdgeList.insert(vertEdgeList.end(), ve[i].begin(), ve[i].end());
    }
    nbr2Start.assign(nb, 0); nbr2Count.assign(nb, 0); nbr2List.clear();
    std::vector<uint32_t> mark(nb, NONE), two;
    for (uint32_t i = 0; i < nb; i++) {
        nbr2Start[i] = (uint32_t)nbr2List.size();
        if (ring[i].empty()) continue;
        two.clear();
        mark[i] = i;
        for (uint32_t n1 : ring[i]) {
            if (mark[n1] != i) { mark[n1] = i; two.push_back(n1); }
            for (uint32_t n2 : ring[n1]) if (mark[n2] != i) { mark[n2] = i; two.push_back(n2); }
        }
        std::sort(two.begin(), two.end());
        nbr2Count[i] = (uint32_t)two.size();
        nbr2List.insert(nbr2List.end(), two.begin(), two.end());
    }
    clothVert.assign(nb, 0);
    for (uint32_t i = 0; i < numAuthoredTris; i++) {
        clothVert[tris[i].x] = 1; clothVert[tris[i].y] = 1; clothVert[tris[i].z] = 1;
    }
    vtTrack.assign(nb, U4{NONE, NONE, NONE, NONE});
    vtTrackPrev = vtTrack;
    eeTrack.assign(std::max<uint32_t>(1, numEdges), U4{NONE, NONE, NONE, NONE});
    eeTrackPrev = eeTrack;
}

// Element grid, isotropic cover: skin radius + margin padding, at most
// 3x3x3 cells; triangles and authored contact edges in separate buckets.
void Solver::ogc_grid() {
    isoTriCells.assign(elemHashSize, {});
    isoEdgeCells.assign(elemHashSize, {});
    const float cs = surfaceCellSize;
    const uint32_t total = numTris + numSurfaceEdges;
    for (uint32_t gid = 0; gid < total; gid++) {
        F3 lo, hi;
        if (gid < numTris) {
            U4 t = tris[gid];
            F3 a = xyz(posLin[t.x]), b = xyz(posLin[t.y]), c = xyz(posLin[t.z]);
            float pad = fmax_(std::fabs(shape[t.x].w), fmax_(std::fabs(shape[t.y].w), std::fabs(shape[t.z].w))) + elemMargin;
            lo = vmin3(vmin3(a, b), c) - f3s(pad);
            hi = vmax3(vmax3(a, b), c) + f3s(pad);
        } else {
            uint32_t e = gid - numTris;
            F3 a = xyz(posLin[edges[2 * e]]), b = xyz(posLin[edges[2 * e + 1]]);
            float pad = fmax_(std::fabs(shape[edges[2 * e]].w), std::fabs(shape[edges[2 * e + 1]].w)) + elemMargin;
            lo = vmin3(a, b) - f3s(pad);
            hi = vmax3(a, b) + f3s(pad);
        }
        if (!finite3(lo) || !finite3(hi)) continue;
        I3 c0 = cell_of(lo, cs), r1 = cell_of(hi, cs);
        I3 c1{std::min(r1.x, c0.x + 2), std::min(r1.y, c0.y + 2), std::min(r1.z, c0.z + 2)};
        uint32_t seen[27];
        uint32_t ns = 0;
        for (int z = c0.z; z <= c1.z; z++)
            for (int y = c0.y; y <= c1.y; y++)
                for (int x = c0.x; x <= c1.x; x++) {
                    uint32_t h = elem_hash(I3{x, y, z}, elemHashSize);
                    bool dup = false;
                    for (uint32_t i = 0; i < ns; i++) dup = dup || seen[i] == h;
                    if (dup) continue;
                    seen[ns++] = h;
                    if (gid < numTris) isoTriCells[h].push_back(gid);
                    else isoEdgeCells[h].push_back(gid - numTris);
                }
    }
}

static inline void bound_min(std::vector<uint32_t>& b, uint32_t i, uint32_t bits) { if (bits < b[i]) b[i] = bits; }

// vt_emit tracking half (25_cloth.metal:391-529)
void Solver::ogc_track_vt(uint32_t gid) {
    const uint32_t v = particleIdx[gid];
    const F3 pv = xyz(posLin[v]);
    const F3 velV = xyz(velLin[v]);
    const uint32_t ns = nbrStart[v], ne = ns + nbrCount[v];
    const uint32_t gv = clothGroup[v];
    const bool solidV = gv != 0u && clothVert[v] == 0u;
    const uint32_t n2s = nbr2Start[v], n2e = n2s + nbr2Count[v];
    const float cap2 = surfaceCellSize * surfaceCellSize;
    float ownB2 = FBIG;
    Best4 best;
    auto consider = [&](uint32_t t) {
        if (t >= numTris || best.has(t)) return;
        U4 tid = tris[t];
        if (tid.x == v || tid.y == v || tid.z == v) return;
        if (solidV && clothGroup[tid.x] == gv && clothGroup[tid.y] == gv && clothGroup[tid.z] == gv &&
            clothVert[tid.x] == 0u && clothVert[tid.y] == 0u && clothVert[tid.z] == 0u)
            return;
        F3 bary;
        F3 q = closest_pt_triangle(pv, xyz(posLin[tid.x]), xyz(posLin[tid.y]), xyz(posLin[tid.z]), bary);
        F3 dd = pv - q;
        float d2 = dot(dd, dd);
        if (d2 < best.d2[3] && !nbr_contains(nbrList, ns, ne, tid.x) && !nbr_contains(nbrList, ns, ne, tid.y) &&
            !nbr_contains(nbrList, ns, ne, tid.z))
            best.insert(t, d2);
        if (d2 < cap2 && !nbr_contains(nbr2List, n2s, n2e, tid.x) && !nbr_contains(nbr2List, n2s, n2e, tid.y) &&
            !nbr_contains(nbr2List, n2s, n2e, tid.z)) {
            uint32_t db = fbits(d2);
            ownB2 = std::fmin(ownB2, d2);
            bound_min(boundsBits, tid.x, db);
            bound_min(boundsBits, tid.y, db);
            bound_min(boundsBits, tid.z, db);
        }
    };
    const U4 tracked = vtTrackPrev[v];
    for (int i = 0; i < 4; i++) consider(u4_at(tracked, i));
    if (tracked.x < numTris) {
        U4 adj = triAdj[tracked.x];
        for (int i = 0; i < 3; i++) consider(u4_at(adj, i));
    }
    for (uint32_t k = ns; k < ne && k < ns + 8; k++) consider(vtTrackPrev[nbrList[k]].x);
    F3 relV = velV;
    if (best.id[0] < numTris) {
        U4 bt = tris[best.id[0]];
        relV = relV - (xyz(velLin[bt.x]) + xyz(velLin[bt.y]) + xyz(velLin[bt.z])) / 3.0f;
    }
    const float vThresh = 0.25f * surfaceCellSize / fmax_(P.dt, 1e-6f);
    const uint32_t period = dot(relV, relV) > vThresh * vThresh ? 1u : 7u;
    const bool missing = best.id[0] == NONE;
    const bool reseed = ((v + P.frame) & period) == 0u || (missing && !solidV) ||
                        (missing && solidV && ((v + P.frame) & 3u) == 0u);
    if (reseed) {
        I3 cc = cell_of(pv, surfaceCellSize);
        for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    uint32_t h = elem_hash(I3{cc.x + dx, cc.y + dy, cc.z + dz}, elemHashSize);
                    for (uint32_t t : isoTriCells[h]) consider(t);
                }
    }
    vtTrack[v] = U4{best.id[0], best.id[1], best.id[2], best.id[3]};
    if (ownB2 < FBIG) bound_min(boundsBits, v, fbits(ownB2));
}

// vt_emit emission half (25_cloth.metal:531-613)
bool Solver::vt_contact(uint32_t v, uint32_t t, bool emit) {
    const F4 plv = posLin[v];
    const F3 pv = xyz(plv);
    const float massV = plv.w;
    const float rv = std::fabs(shape[v].w);
    const F3 velV = xyz(velLin[v]);
    const U4 tid = tris[t];
    const F3 a = xyz(posLin[tid.x]), b = xyz(posLin[tid.y]), c = xyz(posLin[tid.z]);
    F3 bary;
    const F3 q = closest_pt_triangle(pv, a, b, c, bary);
    const F3 dv = pv - q;
    const float dist2 = dot(dv, dv);
    const float rt = fmax_(std::fabs(shape[tid.x].w), fmax_(std::fabs(shape[tid.y].w), std::fabs(shape[tid.z].w)));
    const float hSum = rv + rt;
    const F3 velT = (xyz(velLin[tid.x]) + xyz(velLin[tid.y]) + xyz(velLin[tid.z])) / 3.0f;
    const float inflate = fmin_(length(velV - velT) * P.dt, 0.3f * surfaceCellSize);
    const float detect = hSum + elemMargin + inflate;
    if (dist2 > detect * detect) return false;
    const float dist = std::sqrt(dist2);
    F3 triN = cross(b - a, c - a);
    const float tnLen = length(triN);
    if (tnLen < 1e-12f) return false;
    triN = triN / tnLen;
    float minMass = massV > 0.0f ? massV : FBIG;
    const uint32_t others[3] = {tid.x, tid.y, tid.z};
    for (int k = 0; k < 3; k++) {
        if (others[k] == WORLD_BODY) continue;
        float m = posLin[others[k]].w;
        if (m > 0.0f) minMass = fmin_(minMass, m);
    }
    if (minMass == FBIG) return false;
    if (emit) {
        const uint32_t keyB = t, keyA = (SC_VT << 28) | v;
        const float side = dot(dv, triN) >= 0.0f ? 1.0f : -1.0f;
        const bool deep = bary.x > 0.02f && bary.y > 0.02f && bary.z > 0.02f;
        const float sMem = deep ? soft_prev_side(keyA, keyB, side) : side;
        F3 n;
        float g;
        if (dist > 1e-7f && side == sMem) { n = dv / dist; g = dist; }
        else { n = triN * sMem; g = -dist; }
        const float fricT = props[tid.x].w * bary.x + props[tid.y].w * bary.y + props[tid.z].w * bary.z;
        const float friction = std::sqrt(fmax_(props[v].w * fricT, 0.0f));
        soft_emit(U4{v, tid.x, tid.y, tid.z}, f4(1.0f, -bary.x, -bary.y, -bary.z), n, friction, f3s(0),
                  g - hSum + elemMargin, hSum - elemMargin, soft_lambda_cap(P, minMass), minMass, SC_VT, false, false,
                  sMem < 0.0f, keyA, keyB);
    }
    return true;
}

// ee_emit tracking half (25_cloth.metal:654-790)
void Solver::ogc_track_ee(uint32_t gid) {
    const uint32_t ax = edges[2 * gid], ay = edges[2 * gid + 1];
    const F3 a0 = xyz(posLin[ax]), a1 = xyz(posLin[ay]);
    const F3 velA = (xyz(velLin[ax]) + xyz(velLin[ay])) * 0.5f;
    const uint32_t nsx = nbrStart[ax], nex = nsx + nbrCount[ax];
    const uint32_t nsy = nbrStart[ay], ney = nsy + nbrCount[ay];
    const uint32_t gA = clothGroup[ax];
    const bool solidA = gA != 0u && clothGroup[ay] == gA && clothVert[ax] == 0u && clothVert[ay] == 0u;
    const uint32_t n2sx = nbr2Start[ax], n2ex = n2sx + nbr2Count[ax];
    const float cap2 = surfaceCellSize * surfaceCellSize;
    float ownB2 = FBIG;
    Best4 best;
    auto consider = [&](uint32_t e) {
        if (e >= numSurfaceEdges || e == gid || best.has(e)) return;
        const uint32_t bx = edges[2 * e], by = edges[2 * e + 1];
        if (bx == ax || bx == ay || by == ax || by == ay) return;
        if (solidA && clothGroup[bx] == gA && clothGroup[by] == gA && clothVert[bx] == 0u && clothVert[by] == 0u) return;
        float s, t;
        const F3 b0 = xyz(posLin[bx]), b1 = xyz(posLin[by]);
        closest_seg_seg_st(a0, a1, b0, b1, s, t);
        const F3 cA = a0 + (a1 - a0) * s;
        const F3 cB = b0 + (b1 - b0) * t;
        const F3 dd = cA - cB;
        const float d2 = dot(dd, dd);
        if (d2 < best.d2[3] && !nbr_contains(nbrList, nsx, nex, bx) && !nbr_contains(nbrList, nsx, nex, by) &&
            !nbr_contains(nbrList, nsy, ney, bx) && !nbr_contains(nbrList, nsy, ney, by))
            best.insert(e, d2);
        if (d2 < cap2 && !nbr_contains(nbr2List, n2sx, n2ex, bx) && !nbr_contains(nbr2List, n2sx, n2ex, by)) {
            uint32_t db = fbits(d2);
            ownB2 = std::fmin(ownB2, d2);
            bound_min(boundsBits, bx, db);
            bound_min(boundsBits, by, db);
        }
    };
    const U4 tracked = eeTrackPrev[gid];
    for (int i = 0; i < 4; i++) consider(u4_at(tracked, i));
    for (int side = 0; side < 2; side++) {
        const uint32_t vv = side == 0 ? ax : ay;
        const uint32_t es = vertEdgeStart[vv], ec = std::min(vertEdgeCount[vv], 6u);
        for (uint32_t k = es; k < es + ec; k++) consider(eeTrackPrev[vertEdgeList[k]].x);
    }
    F3 relV = velA;
    if (best.id[0] < numSurfaceEdges) {
        const uint32_t bx = edges[2 * best.id[0]], by = edges[2 * best.id[0] + 1];
        relV = relV - (xyz(velLin[bx]) + xyz(velLin[by])) * 0.5f;
    }
    const float vThresh = 0.25f * surfaceCellSize / fmax_(P.dt, 1e-6f);
    const uint32_t period = dot(relV, relV) > vThresh * vThresh ? 1u : 7u;
    const bool missing = best.id[0] == NONE;
    const bool reseed = ((gid + P.frame) & period) == 0u || (missing && !solidA) ||
                        (missing && solidA && ((gid + P.frame) & 3u) == 0u);
    if (reseed) {
        I3 cc = cell_of((a0 + a1) * 0.5f, surfaceCellSize);
        for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    uint32_t h = elem_hash(I3{cc.x + dx, cc.y + dy, cc.z + dz}, elemHashSize);
                    for (uint32_t e : isoEdgeCells[h]) consider(e);
                }
    }
    eeTrack[gid] = U4{best.id[0], best.id[1], best.id[2], best.id[3]};
    if (ownB2 < FBIG) {
        bound_min(boundsBits, ax, fbits(ownB2));
        bound_min(boundsBits, ay, fbits(ownB2));
    }
}

// ee_emit emission half (25_cloth.metal:792-854)
bool Solver::ee_contact(uint32_t gid, uint32_t eBi, bool emit) {
    const uint32_t ax = edges[2 * gid], ay = edges[2 * gid + 1], bx = edges[2 * eBi], by = edges[2 * eBi + 1];
    const F3 a0 = xyz(posLin[ax]), a1 = xyz(posLin[ay]);
    const F3 b0 = xyz(posLin[bx]), b1 = xyz(posLin[by]);
    float s, t;
    closest_seg_seg_st(a0, a1, b0, b1, s, t);
    const float EPS = 0.02f;
    if (s < EPS || s > 1.0f - EPS || t < EPS || t > 1.0f - EPS) return false;
    const F3 cA = a0 + (a1 - a0) * s;
    const F3 cB = b0 + (b1 - b0) * t;
    const F3 dv = cA - cB;
    const float dist = length(dv);
    const float rA = fmax_(std::fabs(shape[ax].w), std::fabs(shape[ay].w));
    const float rB = fmax_(std::fabs(shape[bx].w), std::fabs(shape[by].w));
    const float hSum = rA + rB;
    const F3 velA = (xyz(velLin[ax]) + xyz(velLin[ay])) * 0.5f;
    const F3 velB = (xyz(velLin[bx]) + xyz(velLin[by])) * 0.5f;
    const float inflate = fmin_(length(velA - velB) * P.dt, 0.3f * surfaceCellSize);
    if (dist - hSum > elemMargin + inflate) return false;
    if (dist < 1e-7f) return false;
    float minMass = FBIG;
    const uint32_t ids[4] = {ax, ay, bx, by};
    for (int j = 0; j < 4; j++) {
        float m = posLin[ids[j]].w;
        if (m > 0.0f) minMass = fmin_(minMass, m);
    }
    if (minMass == FBIG) return false;
    if (emit) {
        const F3 nGeo = dv / dist;
        const uint32_t keyA = (SC_EE << 28) | gid, keyB = eBi;
        F3 n = nGeo;
        float g = dist;
        int prev = soft_map_find(keyA, keyB);
        if (prev >= 0 && dot(nGeo, xyz(prevSoft[prev].normal)) < 0.0f) { n = nGeo * -1.0f; g = -dist; }
        const float fric = std::sqrt(fmax_((props[ax].w + props[ay].w) * 0.5f * (props[bx].w + props[by].w) * 0.5f, 0.0f));
        soft_emit(U4{ax, ay, bx, by}, f4(1.0f - s, s, -(1.0f - t), -t), n, fric, f3s(0), g - hSum + elemMargin,
                  hSum - elemMargin, soft_lambda_cap(P, minMass), minMass, SC_EE, false, false, false, keyA, keyB);
    }
    return true;
}

// Detection of one frame: grid, trackers and bounds, rigid-triangle records,
// then V-T records by particle and E-E records by edge, then the soft map.
void Solver::ogc_detect() {
    ogc_grid();
    for (uint32_t g = 0; g < numParticles; g++) ogc_track_vt(g);
    for (uint32_t g = 0; g < numSurfaceEdges; g++) ogc_track_ee(g);
    rt_emit();
    numSoftRT = softRaw;
    for (uint32_t g = 0; g < numParticles; g++) {
        const uint32_t v = particleIdx[g];
        const U4 best = vtTrack[v];
        for (int bi = 0; bi < 4; bi++) {
            const uint32_t t = u4_at(best, bi);
            if (t >= numTris) break;
            vt_contact(v, t, true);
        }
    }
    numSoftVT = softRaw - numSoftRT;
    for (uint32_t g = 0; g < numSurfaceEdges; g++) {
        const U4 best = eeTrack[g];
        for (int bi = 0; bi < 4; bi++) {
            const uint32_t e = u4_at(best, bi);
            if (e >= numSurfaceEdges) break;
            if (e <= g) continue;
            ee_contact(g, e, true);
        }
    }
    numSoftEE = softRaw - numSoftRT - numSoftVT;
    soft_map_rebuild();
}

// ogc_bounds_refresh (25_cloth.metal:879-931)
void Solver::ogc_refresh() {
    for (uint32_t g = 0; g < numParticles; g++) {
        const uint32_t v = particleIdx[g];
        const F3 pv = xyz(posLin[v]);
        const uint32_t n2s = nbr2Start[v], n2e = n2s + nbr2Count[v];
        float dmin2 = 3.0e38f;
        const U4 tracked = vtTrack[v];
        for (int i = 0; i < 4; i++) {
            const uint32_t t = u4_at(tracked, i);
            if (t >= numTris) break;
            U4 tid = tris[t];
            if (nbr_contains(nbr2List, n2s, n2e, tid.x) || nbr_contains(nbr2List, n2s, n2e, tid.y) ||
                nbr_contains(nbr2List, n2s, n2e, tid.z))
                continue;
            F3 bary;
            F3 q = closest_pt_triangle(pv, xyz(posLin[tid.x]), xyz(posLin[tid.y]), xyz(posLin[tid.z]), bary);
            F3 dd = pv - q;
            dmin2 = std::fmin(dmin2, dot(dd, dd));
        }
        const uint32_t es = vertEdgeStart[v], ec = std::min(vertEdgeCount[v], 6u);
        for (uint32_t k = es; k < es + ec; k++) {
            const uint32_t myE = vertEdgeList[k];
            const uint32_t other = eeTrack[myE].x;
            if (other >= numSurfaceEdges) continue;
            const uint32_t ox = edges[2 * other], oy = edges[2 * other + 1];
            if (nbr_contains(nbr2List, n2s, n2e, ox) || nbr_contains(nbr2List, n2s, n2e, oy)) continue;
            const F3 a0 = xyz(posLin[edges[2 * myE]]), a1 = xyz(posLin[edges[2 * myE + 1]]);
            const F3 b0 = xyz(posLin[ox]), b1 = xyz(posLin[oy]);
            float s, t;
            closest_seg_seg_st(a0, a1, b0, b1, s, t);
            const F3 dd = (a0 + (a1 - a0) * s) - (b0 + (b1 - b0) * t);
            dmin2 = std::fmin(dmin2, dot(dd, dd));
        }
        boundsBits[v] = fbits(dmin2);
        ogcPrev[v] = posLin[v];
    }
}

// Color-Jacobi commit of one color
void Solver::publish_color(uint32_t c) {
    for (uint32_t i = colorStart[c]; i < colorStart[c + 1]; i++) {
        const uint32_t v = colorList[i];
        posLin[v] = f4(xyz(posNext[v]), posLin[v].w);
        if (shape[v].w >= 0.0f) posAng[v] = angNext[v];
    }
}

}  // namespace oracle
