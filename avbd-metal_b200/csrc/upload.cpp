// upload.cpp — scene upload on the host (GPUSolver.swift:338-638, :901-2081).
//
// Computes per-body mass/inertia/radius, collider partition and cell size,
// the joint/spring/tet records, the sorted collision-exclusion list, the tet
// boundary surface groups, the static topology palette for soft scenes and
// the static part of the per-body adjacency.  Compiled with
// -ffp-contract=off so every float matches a plain float32 evaluation.
#include "upload.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <set>
#include <unordered_set>

namespace avbd {
namespace {

struct V3 { float x, y, z; };
inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 add(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 mul(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
inline V3 divs(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float length(V3 a) { return std::sqrt(dot(a, a)); }
inline float fmin_(float a, float b) { return a < b ? a : b; }
inline float fmax_(float a, float b) { return a > b ? a : b; }
inline V3 from(const float* p) { return V3{p[0], p[1], p[2]}; }

inline f4 qmul(f4 a, f4 b) {
    return f4{a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
              a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
              a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w,
              a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
inline float dot4(f4 a, f4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
inline f4 qinv(f4 q) { float d = dot4(q, q); return f4{-q.x / d, -q.y / d, -q.z / d, q.w / d}; }
inline V3 qrot(f4 q, V3 v) {
    V3 u{q.x, q.y, q.z};
    V3 c = cross(u, v);
    V3 t{2.0f * c.x, 2.0f * c.y, 2.0f * c.z};
    V3 wt{q.w * t.x, q.w * t.y, q.w * t.z};
    return add(add(v, wt), cross(u, t));
}

uint32_t next_pow2(uint32_t v) { uint32_t p = 1; while (p < v) p <<= 1; return p; }

bool desc_dynamic(const avbd_body_desc& b) {
    return b.has_explicit_mass ? b.mass > 0.0f : b.density > 0.0f;
}

// Bounding radius of a collider about its origin (GPUSolver.swift:993-1002):
// the farthest hull vertex for a convex hull.
float collider_radius(const avbd_scene_desc* s, const avbd_collider_desc& c) {
    if (c.hull_count > 0) {
        float r = 0.0f;
        for (uint32_t k = 0; k < c.hull_count; k++) {
            const float* v = s->hull_vertices + 3 * (size_t)(c.hull_offset + k);
            r = std::max(r, length(V3{v[0], v[1], v[2]}));
        }
        return r;
    }
    V3 sz = from(c.size);
    if (c.shape == AVBD_SHAPE_SPHERE) return sz.x / 2.0f;
    if (c.shape == AVBD_SHAPE_TORUS) return sz.x + sz.y;
    if (c.shape == AVBD_SHAPE_CAPSULE) return sz.x / 2.0f + sz.y;
    return length(mul(sz, 0.5f));
}

// Faces owned by exactly one tet, wound outward, in sorted order
// (GPUSolver.swift:875-897).
std::vector<std::array<int, 3>> boundary_faces(const avbd_scene_desc* s) {
    std::vector<std::array<int, 3>> out;
    if (s->num_tets == 0) return out;
    struct Face { std::array<int, 3> tri; int opp; int count; };
    std::map<std::array<int, 3>, Face> faces;
    static const int order[4][4] = {{0, 1, 2, 3}, {0, 1, 3, 2}, {0, 2, 3, 1}, {1, 2, 3, 0}};
    for (uint32_t t = 0; t < s->num_tets; t++) {
        const int32_t* ids = s->tets[t].ids;
        for (const auto& f : order) {
            std::array<int, 3> tri{ids[f[0]], ids[f[1]], ids[f[2]]};
            std::array<int, 3> key = tri;
            std::sort(key.begin(), key.end());
            auto it = faces.find(key);
            if (it != faces.end()) it->second.count++;
            else faces.emplace(key, Face{tri, ids[f[3]], 1});
        }
    }
    for (const auto& kv : faces) {
        if (kv.second.count != 1) continue;
        int a = kv.second.tri[0], b = kv.second.tri[1], c = kv.second.tri[2];
        V3 A = from(s->bodies[a].position), B = from(s->bodies[b].position), Cp = from(s->bodies[c].position);
        V3 n = cross(sub(B, A), sub(Cp, A));
        if (dot(n, sub(from(s->bodies[kv.second.opp].position), A)) > 0.0f) std::swap(b, c);
        out.push_back({a, b, c});
    }
    std::sort(out.begin(), out.end());
    return out;
}

inline float dist(V3 a, V3 b) { return length(sub(a, b)); }
inline V3 unit(V3 a) { return mul(a, 1.0f / std::sqrt(dot(a, a))); }
inline uint64_t edge_key(int a, int b) { return (uint64_t)std::min(a, b) << 32 | (uint64_t)std::max(a, b); }

// Cloth topology, membranes, bends and element-contact parameters
// (GPUSolver.swift:1289-1680).  Bends are numbered by ascending edge key.
void upload_cloth(const avbd_scene_desc* s, const std::vector<std::array<int, 3>>& boundary, HostScene& H) {
    const uint32_t nb = s->num_bodies;
    const uint32_t authored = s->num_tris;
    std::vector<std::array<int, 3>> coll;
    coll.reserve(authored + boundary.size());
    for (uint32_t i = 0; i < authored; i++) coll.push_back({s->tris[i].ids[0], s->tris[i].ids[1], s->tris[i].ids[2]});
    coll.insert(coll.end(), boundary.begin(), boundary.end());
    H.numTris = (uint32_t)coll.size();
    auto P = [&](int i) { return from(s->bodies[i].position); };
    auto SX = [&](int i) { return s->bodies[i].size[0]; };

    std::unordered_set<uint64_t> topoSeen, contactSeen;
    std::vector<uint64_t> topo, contact;
    float maxElemR = 0.0f, maxCollR = 0.0f;
    H.tris.resize(H.numTris);
    for (uint32_t i = 0; i < H.numTris; i++) {
        const int a = coll[i][0], b = coll[i][1], c = coll[i][2];
        H.tris[i] = u4{(uint32_t)a, (uint32_t)b, (uint32_t)c, 0u};
        const int ends[3][2] = {{a, b}, {b, c}, {a, c}};
        for (const auto& e : ends) {
            const uint64_t key = edge_key(e[0], e[1]);
            if (topoSeen.insert(key).second) topo.push_back(key);
            if (i < authored && contactSeen.insert(key).second) contact.push_back(key);
        }
        const V3 pa = P(a), pb = P(b), pc = P(c);
        const V3 m = divs(add(add(pa, pb), pc), 3.0f);
        const float thick = fmax_(SX(a), fmax_(SX(b), SX(c))) / 2.0f;
        maxCollR = fmax_(maxCollR, thick);
        maxElemR = fmax_(maxElemR, fmax_(dist(m, pa), fmax_(dist(m, pb), dist(m, pc))) + thick);
    }
    H.numSurfaceEdges = (uint32_t)contact.size();
    for (uint64_t key : topo)
        if (contactSeen.insert(key).second) contact.push_back(key);
    H.numEdges = (uint32_t)contact.size();
    std::vector<std::vector<uint32_t>> ring(nb);
    for (uint64_t key : topo) {
        const uint32_t a = (uint32_t)(key >> 32), b = (uint32_t)key;
        ring[a].push_back(b);
        ring[b].push_back(a);
    }
    H.edges.clear();
    H.edges.reserve(2 * contact.size());
    for (uint64_t key : contact) {
        const int a = (int)(key >> 32), b = (int)(uint32_t)key;
        H.edges.push_back((uint32_t)a);
        H.edges.push_back((uint32_t)b);
        maxElemR = fmax_(maxElemR, dist(P(a), P(b)) / 2.0f + fmax_(SX(a), SX(b)) / 2.0f);
    }
    H.nbrStart.assign(nb, 0);
    H.nbrCount.assign(nb, 0);
    H.nbrList.clear();
    for (uint32_t i = 0; i < nb; i++) {
        std::sort(ring[i].begin(), ring[i].end());
        H.nbrStart[i] = (uint32_t)H.nbrList.size();
        H.nbrCount[i] = (uint32_t)ring[i].size();
        H.nbrList.insert(H.nbrList.end(), ring[i].begin(), ring[i].end());
    }

    // connected surface components and self-collision flags
    H.selfCollision.assign(nb, 0);
    std::vector<uint8_t> onSurface(nb, 0);
    std::vector<int> parent(nb, -1);
    auto root = [&](int x) {
        int r = x;
        while (parent[r] >= 0 && parent[r] != r) r = parent[r];
        int c = x;
        while (parent[c] >= 0 && parent[c] != r) { const int n = parent[c]; parent[c] = r; c = n; }
        if (parent[r] < 0) parent[r] = r;
        return r;
    };
    for (const auto& f : coll) { const int r = root(f[0]); parent[root(f[1])] = r; parent[root(f[2])] = r; }
    std::set<int> selfRoots;
    for (uint32_t i = 0; i < authored; i++) selfRoots.insert(root(s->tris[i].ids[0]));
    for (uint32_t i = 0; i < s->num_tets; i++)
        if (s->tets[i].self_collision)
            for (int k = 0; k < 4; k++)
                if (parent[s->tets[i].ids[k]] >= 0) selfRoots.insert(root(s->tets[i].ids[k]));
    std::map<int, uint32_t> groupOf;
    for (const auto& f : coll) {
        const int r = root(f[0]);
        auto it = groupOf.find(r);
        const uint32_t g = it == groupOf.end() ? groupOf.emplace(r, (uint32_t)groupOf.size() + 1).first->second
                                               : it->second;
        const uint32_t self = selfRoots.count(r) ? 1u : 0u;
        for (int k = 0; k < 3; k++)
            if (s->bodies[f[k]].is_particle) { H.clothGroup[f[k]] = g; H.selfCollision[f[k]] = self; onSurface[f[k]] = 1; }
    }
    H.particleIdx.clear();
    for (uint32_t i = 0; i < nb; i++) if (onSurface[i]) H.particleIdx.push_back(i);
    H.numParticles = H.numTris == 0 ? 0u : (uint32_t)H.particleIdx.size();

    // StVK membranes and Bergou hinges over interior edges
    struct Flap { int opp; float k; };
    std::map<uint64_t, std::vector<Flap>> hinge;
    H.membranes.clear();
    for (uint32_t ti = 0; ti < authored; ti++) {
        const avbd_tri_desc& t = s->tris[ti];
        if (!(t.mu > 0.0f)) continue;
        const int i0 = t.ids[0], i1 = t.ids[1], i2 = t.ids[2];
        const V3 x0 = P(i0), d1 = sub(P(i1), x0), d2 = sub(P(i2), x0);
        const V3 nrm = cross(d1, d2);
        const float area = length(nrm) / 2.0f;
        if (!(area > 1e-10f)) continue;
        const V3 e1 = unit(d1);
        const V3 e2 = unit(cross(unit(nrm), e1));
        const float a = dot(d1, e1), b = dot(d1, e2), c = dot(d2, e1), dd = dot(d2, e2);
        const float det = a * dd - b * c;
        if (!(std::fabs(det) > 1e-12f)) continue;
        MembraneGPU m{};
        m.ids = u4{(uint32_t)i0, (uint32_t)i1, (uint32_t)i2, 0u};
        m.dm = f4{dd / det, -b / det, -c / det, a / det};
        m.mat = f4{t.mu * area, t.lambda * area, area, 0.0f};
        H.membranes.push_back(m);
        if (t.bend > 0.0f) {
            hinge[edge_key(i0, i1)].push_back(Flap{i2, t.bend});
            hinge[edge_key(i1, i2)].push_back(Flap{i0, t.bend});
            hinge[edge_key(i0, i2)].push_back(Flap{i1, t.bend});
        }
    }
    H.bends.clear();
    for (const auto& kv : hinge) {
        if (kv.second.size() != 2) continue;
        const int v0 = (int)(kv.first >> 32), v1 = (int)(uint32_t)kv.first;
        const V3 p0 = P(v0), p1 = P(v1);
        const float L = dist(p0, p1);
        if (!(L > 1e-9f)) continue;
        // unfold both flaps into the hinge plane from rest edge lengths
        float qx[4] = {0.0f, L, 0.0f, 0.0f}, qy[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        bool ok = true;
        for (int f = 0; f < 2 && ok; f++) {
            const V3 po = P(kv.second[f].opp);
            const float l0 = dist(po, p0), l1 = dist(po, p1);
            const float ax = (L * L + l0 * l0 - l1 * l1) / (2.0f * L);
            const float h2 = l0 * l0 - ax * ax;
            if (!(h2 > 1e-12f)) { ok = false; break; }
            qx[2 + f] = ax;
            qy[2 + f] = (f == 0 ? 1.0f : -1.0f) * std::sqrt(h2);
        }
        if (!ok) continue;
        // K spans the null space of {1, x, y} over the four stencil points
        auto minor3 = [&](int c0, int c1, int c2) {
            const V3 a = v3(1.0f, qx[c0], qy[c0]), b = v3(1.0f, qx[c1], qy[c1]), c = v3(1.0f, qx[c2], qy[c2]);
            return dot(a, cross(b, c));
        };
        f4 K{minor3(1, 2, 3), -minor3(0, 2, 3), minor3(0, 1, 3), -minor3(0, 1, 2)};
        auto cot = [&](int apex, int i, int j) {
            const float ux = qx[i] - qx[apex], uy = qy[i] - qy[apex];
            const float vx = qx[j] - qx[apex], vy = qy[j] - qy[apex];
            const float cr = ux * vy - uy * vx;
            return std::fabs(cr) > 1e-12f ? (ux * vx + uy * vy) / std::fabs(cr) : 0.0f;
        };
        const float want = cot(0, 1, 2) + cot(1, 0, 2);
        if (!(std::fabs(K.z) > 1e-12f)) continue;
        const float sc = want / K.z;
        K = f4{K.x * sc, K.y * sc, K.z * sc, K.w * sc};
        const float a1 = std::fabs((qx[1] - qx[0]) * qy[2]) / 2.0f;
        const float a2 = std::fabs((qx[1] - qx[0]) * qy[3]) / 2.0f;
        BendGPU bd{};
        bd.ids = u4{(uint32_t)v0, (uint32_t)v1, (uint32_t)kv.second[0].opp, (uint32_t)kv.second[1].opp};
        bd.K = K;
        bd.mat = f4{3.0f * (kv.second[0].k + kv.second[1].k) / 2.0f / fmax_(a1 + a2, 1e-9f), 0.0f, 0.0f, 0.0f};
        H.bends.push_back(bd);
    }

    // element-contact radii and cells
    float maxPartR = maxCollR, edgeSum = 0.0f;
    for (uint64_t key : topo) {
        const int a = (int)(key >> 32), b = (int)(uint32_t)key;
        maxPartR = fmax_(maxPartR, fmax_(SX(a), SX(b)) / 2.0f);
        edgeSum += dist(P(a), P(b));
    }
    const float meanEdge = topo.empty() ? 0.2f : edgeSum / (float)topo.size();
    H.elemMargin = fmin_(0.01f, fmax_(0.002f, 0.5f * maxPartR));
    const float forceReach = 2.0f * maxPartR + H.elemMargin;
    H.queryRadius = fmax_(1.5f * forceReach, 0.75f * meanEdge);
    const float reach = (2.0f * maxPartR + H.elemMargin) / 0.7f;
    H.surfaceCellSize = fmax_(0.02f, fmax_(fmax_(reach, meanEdge * 1.05f), maxElemR + maxPartR + H.elemMargin));
    H.elemCellSize = fmax_(0.02f, fmax_(fmax_(reach, meanEdge * 1.05f), 2.0f * maxElemR + H.queryRadius));

    // isotropic-OGC topology (GPUSolver.swift:1338-1460): edge-adjacent
    // triangles (edges visited in ascending key order), the incident contact
    // edges of every vertex, and the sorted 1-ring-plus-2-ring sets.
    std::map<uint64_t, std::pair<int, int>> edgeTris;
    for (uint32_t ti = 0; ti < H.numTris; ti++) {
        const int a = coll[ti][0], b = coll[ti][1], c = coll[ti][2];
        const int ends[3][2] = {{a, b}, {b, c}, {a, c}};
        for (const auto& e : ends) {
            auto it = edgeTris.find(edge_key(e[0], e[1]));
            if (it == edgeTris.end()) edgeTris.emplace(edge_key(e[0], e[1]), std::make_pair((int)ti, -1));
            else it->second.second = (int)ti;
        }
    }
    H.triAdj.assign(std::max<uint32_t>(1, H.numTris), u4{0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu});
    std::vector<int> fill(std::max<uint32_t>(1, H.numTris), 0);
    auto put = [&](int t, int other) {
        if (fill[t] >= 3) return;
        uint32_t* slots = &H.triAdj[t].x;
        slots[fill[t]++] = (uint32_t)other;
    };
    for (const auto& kv : edgeTris) {
        if (kv.second.second < 0) continue;
        put(kv.second.first, kv.second.second);
        put(kv.second.second, kv.second.first);
    }
    std::vector<std::vector<uint32_t>> vertEdges(nb);
    for (uint32_t i = 0; i < H.numEdges; i++) {
        vertEdges[H.edges[2 * i]].push_back(i);
        vertEdges[H.edges[2 * i + 1]].push_back(i);
    }
    H.vertEdgeStart.assign(nb, 0);
    H.vertEdgeCount.assign(nb, 0);
    H.vertEdgeList.clear();
    for (uint32_t i = 0; i < nb; i++) {
        H.vertEdgeStart[i] = (uint32_t)H.vertEdgeList.size();
        H.vertEdgeCount[i] = (uint32_t)vertEdges[i].size();
        H.vertEdgeList.insert(H.vertEdgeList.end(), vertEdges[i].begin(), vertEdges[i].end());
    }
    H.nbr2Start.assign(nb, 0);
    H.nbr2Count.assign(nb, 0);
    H.nbr2List.clear();
    std::vector<uint32_t> mark(nb, 0xFFFFFFFFu), two;
    for (uint32_t i = 0; i < nb; i++) {
        H.nbr2Start[i] = (uint32_t)H.nbr2List.size();
        if (ring[i].empty()) continue;
        two.clear();
        mark[i] = i;
        for (uint32_t n1 : ring[i]) {
            if (mark[n1] != i) { mark[n1] = i; two.push_back(n1); }
            for (uint32_t n2 : ring[n1])
                if (mark[n2] != i) { mark[n2] = i; two.push_back(n2); }
        }
        std::sort(two.begin(), two.end());
        H.nbr2Count[i] = (uint32_t)two.size();
        H.nbr2List.insert(H.nbr2List.end(), two.begin(), two.end());
    }
    H.clothVert.assign(nb, 0);
    for (uint32_t i = 0; i < authored; i++)
        for (int k = 0; k < 3; k++) H.clothVert[s->tris[i].ids[k]] = 1;

    // capacities (GPUSolver.swift:395-443)
    const uint64_t surf = H.particleIdx.size();
    const uint64_t pairsCap = std::max<uint64_t>(1, 64ull * surf + 128ull * topo.size());
    const uint64_t budget = std::min<uint64_t>(pairsCap, 8ull * surf + 8ull * topo.size());
    H.maxDatPairs = (uint32_t)std::min<uint64_t>(pairsCap, 0xFFFFFFFFull);
    H.maxSoft = (uint32_t)std::max<uint64_t>(1, 4ull * H.numTris + budget);
    H.softMapCapacity = next_pow2(std::max<uint32_t>(64u, 2u * H.maxSoft));
    H.elemHashSize = next_pow2(std::max<uint32_t>(64u, 2u * 4u * H.numTris));
    const uint64_t iso = std::max<uint64_t>(1, 4ull * surf + 4ull * H.numTris + 4ull * H.numSurfaceEdges);
    H.maxSoftIso = (uint32_t)std::min<uint64_t>(iso, 0x7FFFFFFFull);
    H.softMapCapacityIso = next_pow2(std::max<uint32_t>(64u, 2u * H.maxSoftIso));
}

}  // namespace

int upload_scene(const avbd_scene_desc* s, HostScene& H, std::string& err) {
    if (!s || s->abi_version != AVBD_ABI_VERSION) { err = "bad scene descriptor or ABI version"; return AVBD_ERR_INVALID_ARGUMENT; }
    if (s->num_bodies > 0 && !s->bodies) { err = "null body array"; return AVBD_ERR_INVALID_ARGUMENT; }
    if (!(s->settings.dt > 0.0f) || s->settings.iterations < 0) { err = "dt must be positive and iterations non-negative"; return AVBD_ERR_INVALID_ARGUMENT; }
    const uint32_t nb = s->num_bodies, nc = s->num_colliders;
    for (uint32_t i = 0; i < nc; i++) {
        const avbd_collider_desc& c = s->colliders[i];
        if (c.body < 0 || (uint32_t)c.body >= nb) { err = "collider owner out of range"; return AVBD_ERR_INVALID_ARGUMENT; }
        if (c.shape > AVBD_SHAPE_CAPSULE) { err = "unknown collider shape"; return AVBD_ERR_INVALID_ARGUMENT; }
        if (c.hull_count > 0) {
            // GPUSolver.swift:1023-1024 and Scene.swift:656-657
            if (c.hull_count < 4 || c.hull_count > 64) { err = "a convex collider needs 4...64 hull vertices"; return AVBD_ERR_INVALID_ARGUMENT; }
            if (!s->hull_vertices || (uint64_t)c.hull_offset + c.hull_count > s->num_hull_vertices) { err = "hull vertex range out of range"; return AVBD_ERR_INVALID_ARGUMENT; }
            for (uint32_t k = 0; k < 3 * c.hull_count; k++)
                if (!std::isfinite(s->hull_vertices[3 * (size_t)c.hull_offset + k])) { err = "convex collider vertices must be finite"; return AVBD_ERR_INVALID_ARGUMENT; }
        }
    }
    for (uint32_t i = 0; i < nb; i++)
        if (s->bodies[i].shape > AVBD_SHAPE_CAPSULE) { err = "unknown body shape"; return AVBD_ERR_INVALID_ARGUMENT; }
    for (uint32_t i = 0; i < s->num_tris; i++)
        for (int k = 0; k < 3; k++)
            if (s->tris[i].ids[k] < 0 || (uint32_t)s->tris[i].ids[k] >= nb) { err = "triangle vertex out of range"; return AVBD_ERR_INVALID_ARGUMENT; }
    for (uint32_t i = 0; i < s->num_joints; i++) {
        const avbd_joint_desc& j = s->joints[i];
        if (j.body_b < 0 || (uint32_t)j.body_b >= nb || j.body_a >= (int32_t)nb || j.body_a < -1) { err = "joint body out of range"; return AVBD_ERR_INVALID_ARGUMENT; }
        if (j.motor_torque > 0.0f && !j.has_hinge) { err = "a powered joint must define a hinge axis"; return AVBD_ERR_INVALID_ARGUMENT; }
    }
    for (uint32_t i = 0; i < s->num_springs; i++) {
        const avbd_spring_desc& p = s->springs[i];
        if (p.body_a < 0 || p.body_b < 0 || (uint32_t)p.body_a >= nb || (uint32_t)p.body_b >= nb) { err = "spring body out of range"; return AVBD_ERR_INVALID_ARGUMENT; }
    }
    for (uint32_t i = 0; i < s->num_tets; i++)
        for (int k = 0; k < 4; k++)
            if (s->tets[i].ids[k] < 0 || (uint32_t)s->tets[i].ids[k] >= nb) { err = "tet vertex out of range"; return AVBD_ERR_INVALID_ARGUMENT; }

    H.numBodies = nb;
    H.numColliders = nc;
    uint32_t enabled = 0;
    for (uint32_t i = 0; i < nc; i++) enabled += s->colliders[i].collision_enabled ? 1u : 0u;
    const uint32_t mppb = s->max_pairs_per_body ? s->max_pairs_per_body : 16u;
    H.maxPairs = std::max<uint32_t>(4096u, enabled * mppb);
    H.mapCapacity = next_pow2(2 * H.maxPairs);
    H.gridHashSize = next_pow2(std::max<uint32_t>(64u, 2u * std::max<uint32_t>(1u, enabled)));
    std::vector<std::array<int, 3>> boundary = boundary_faces(s);
    H.numTris = (uint32_t)boundary.size() + s->num_tris;

    // ---- bodies (GPUSolver.swift:915-969)
    H.posLin.assign(nb, f4{}); H.posAng.assign(nb, f4{}); H.velLin.assign(nb, f4{});
    H.velAng.assign(nb, f4{}); H.prevVelLin.assign(nb, f4{}); H.props.assign(nb, f4{});
    H.shape.assign(nb, f4{}); H.spinVel.assign(nb, f4{});
    H.gravityScale.assign(nb, 1.0f); H.shapeType.assign(nb, 0); H.clothGroup.assign(nb, 0);
    H.isDynamic.assign(nb, 0);
    const float PI = 3.14159265358979323846f;
    H.numDynamicBodies = 0;
    for (uint32_t i = 0; i < nb; i++) {
        const avbd_body_desc& b = s->bodies[i];
        V3 size = from(b.size);
        float mass, radius;
        V3 moment;
        if (b.shape == AVBD_SHAPE_BOX) {
            mass = b.density > 0.0f ? size.x * size.y * size.z * b.density : 0.0f;
            moment = V3{(size.y * size.y + size.z * size.z) / 12.0f * mass,
                        (size.x * size.x + size.z * size.z) / 12.0f * mass,
                        (size.x * size.x + size.y * size.y) / 12.0f * mass};
            radius = length(mul(size, 0.5f));
        } else if (b.shape == AVBD_SHAPE_SPHERE) {
            float r = size.x / 2.0f;
            mass = b.density > 0.0f ? 4.0f / 3.0f * PI * r * r * r * b.density : 0.0f;
            float m = 0.4f * mass * r * r;
            moment = V3{m, m, m};
            radius = r;
        } else if (b.shape == AVBD_SHAPE_TORUS) {
            float R = size.x, r = size.y;
            mass = b.density > 0.0f ? 2.0f * PI * PI * R * r * r * b.density : 0.0f;
            float iDia = mass * (R * R / 2.0f + 5.0f * r * r / 8.0f);
            float iAxis = mass * (R * R + 3.0f * r * r / 4.0f);
            moment = V3{iDia, iDia, iAxis};
            radius = R + r;
        } else {
            float L = size.x, r = size.y;
            mass = b.density > 0.0f ? PI * r * r * (L + 4.0f * r / 3.0f) * b.density : 0.0f;
            float iAxis = 0.5f * mass * r * r;
            float iPerp = mass * (L * L / 12.0f + r * r / 4.0f);
            moment = V3{iPerp, iPerp, iAxis};
            radius = L / 2.0f + r;
        }
        if (b.has_explicit_mass) { mass = b.mass; moment = from(b.diagonal_inertia); }
        H.posLin[i] = f4{b.position[0], b.position[1], b.position[2], mass};
        H.posAng[i] = f4{b.rotation[0], b.rotation[1], b.rotation[2], b.rotation[3]};
        H.velLin[i] = f4{b.velocity[0], b.velocity[1], b.velocity[2], 0.0f};
        H.prevVelLin[i] = H.velLin[i];
        H.props[i] = f4{moment.x, moment.y, moment.z, b.friction};
        H.shape[i] = f4{size.x, size.y, size.z, b.is_particle ? -radius : radius};
        H.gravityScale[i] = b.gravity_scale;
        H.shapeType[i] = b.shape;
        H.isDynamic[i] = desc_dynamic(b) ? 1 : 0;
        if (mass > 0.0f) H.numDynamicBodies++;
    }

    // ---- colliders and broadphase partition (GPUSolver.swift:971-1089)
    H.colOwner.assign(nc, 0); H.colShapeType.assign(nc, 0); H.colGroup.assign(nc, 0);
    H.colShared.assign(nc, 0); H.colShape.assign(nc, f4{}); H.colLocalPos.assign(nc, f4{});
    H.colLocalRot.assign(nc, f4{}); H.colFriction.assign(2 * nc, 0.0f);
    H.colHullRange.assign(2 * nc, 0u);
    H.hullVerts.clear();
    std::vector<float> radii;
    for (uint32_t i = 0; i < nc; i++) {
        const avbd_collider_desc& c = s->colliders[i];
        float r = collider_radius(s, c);
        bool particle = s->bodies[c.body].is_particle != 0;
        H.colOwner[i] = (uint32_t)c.body;
        H.colGroup[i] = c.collision_group;
        H.colShared[i] = c.collides_with_shared ? 1u : 0u;
        H.colShape[i] = f4{c.size[0], c.size[1], c.size[2], particle ? -r : r};
        H.colLocalPos[i] = f4{c.local_position[0], c.local_position[1], c.local_position[2], c.friction};
        H.colLocalRot[i] = f4{c.local_rotation[0], c.local_rotation[1], c.local_rotation[2], c.local_rotation[3]};
        H.colFriction[2 * i] = c.friction;
        H.colFriction[2 * i + 1] = c.dynamic_friction;
        uint32_t flags = c.shape;
        if (c.hull_count > 0) {
            // hulls are packed in collider order (GPUSolver.swift:1020-1032)
            H.colHullRange[2 * i] = (uint32_t)H.hullVerts.size();
            H.colHullRange[2 * i + 1] = c.hull_count;
            for (uint32_t k = 0; k < c.hull_count; k++) {
                const float* v = s->hull_vertices + 3 * (size_t)(c.hull_offset + k);
                H.hullVerts.push_back(f4{v[0], v[1], v[2], 0.0f});
            }
            flags = 4u;
        }
        if (particle) flags |= SHAPE_PARTICLE;
        if (c.world_round_anchor) flags |= COLLIDER_WORLD_ROUND_ANCHOR;
        H.colShapeType[i] = flags;
        if (c.collision_enabled && H.isDynamic[c.body]) radii.push_back(r);
    }
    std::vector<float> sorted = radii;
    std::sort(sorted.begin(), sorted.end());
    const float median = sorted.empty() ? 0.5f : sorted[sorted.size() / 2];
    const float threshold = median * 4.0f;
    bool isolated = false;
    for (uint32_t i = 0; i < nc; i++)
        if (s->colliders[i].collision_enabled && s->colliders[i].collision_group != 0) isolated = true;
    for (uint32_t i = 0; i < nc; i++) {
        const avbd_collider_desc& c = s->colliders[i];
        if (!c.collision_enabled) continue;
        if (collider_radius(s, c) > threshold || (isolated && c.collision_group == 0)) H.globalIdx.push_back(i);
        else H.hashedIdx.push_back(i);
    }
    float maxHashedRadius = 0.05f, maxParticleRadius = 0.0f;
    uint32_t numHashedRigid = 0, numHashedParticles = 0;
    for (uint32_t i : H.hashedIdx) {
        maxHashedRadius = fmax_(maxHashedRadius, std::fabs(H.colShape[i].w));
        if (H.colShape[i].w >= 0.0f) numHashedRigid++;
        else { numHashedParticles++; maxParticleRadius = fmax_(maxParticleRadius, std::fabs(H.colShape[i].w)); }
    }

    // ---- joints (GPUSolver.swift:1092-1195)
    const uint32_t nj = s->num_joints;
    H.joints.assign(nj, JointGPU{});
    const float dt = s->settings.dt;
    for (uint32_t i = 0; i < nj; i++) {
        const avbd_joint_desc& j = s->joints[i];
        JointGPU g{};
        uint32_t aIdx = j.body_a >= 0 ? (uint32_t)j.body_a : WORLD_BODY;
        uint32_t flags = 0;
        if (std::isinf(j.stiffness_lin)) flags |= 1;
        if (std::isinf(j.stiffness_ang)) flags |= 2;
        if (std::isfinite(j.fracture)) flags |= 4;
        if (j.fracture_linear) flags |= 8;
        g.header = u4{aIdx, (uint32_t)j.body_b, 0, flags};
        const float bigK = 3.0e10f;
        g.rA = f4{j.r_a[0], j.r_a[1], j.r_a[2], fmin_(j.stiffness_lin, bigK)};
        g.rB = f4{j.r_b[0], j.r_b[1], j.r_b[2], fmin_(j.stiffness_ang, bigK)};
        V3 sizeA = j.body_a >= 0 ? from(s->bodies[j.body_a].size) : V3{0, 0, 0};
        V3 ss = add(sizeA, from(s->bodies[j.body_b].size));
        g.C0Lin = f4{0, 0, 0, dot(ss, ss)};
        g.C0Ang = f4{0, 0, 0, fmin_(j.fracture, 3.0e18f)};
        f4 qA0 = j.body_a >= 0 ? H.posAng[j.body_a] : f4{0, 0, 0, 1};
        f4 rel = qmul(qinv(qA0), H.posAng[j.body_b]);
        float rl = std::sqrt(dot4(rel, rel));
        g.restRel = f4{rel.x / rl, rel.y / rl, rel.z / rl, rel.w / rl};
        if (j.has_hinge) {
            g.hingeAxis = f4{j.hinge_axis[0], j.hinge_axis[1], j.hinge_axis[2], 1.0f};
            g.dynamics.x = j.armature;
            if (j.motor_torque > 0.0f) {
                g.motor = f4{j.motor_target, j.motor_torque, 0.0f, j.motor_stiffness};
                g.limits = f4{j.limit_lo, j.limit_hi, j.motor_damping, 0.0f};
                if (j.motor_mode == AVBD_MOTOR_IMPLICIT_POSITION_PD) g.header.w |= MOTOR_IMPLICIT;
                else if (j.motor_mode == AVBD_MOTOR_EXPLICIT_TORQUE_PD) g.header.w |= MOTOR_EXPLICIT;
                else g.header.w |= MOTOR_VELOCITY;
                if (j.motor_rate != 0.0f) H.rateMotors.push_back({i, j.motor_rate});
            }
            if (j.limit_lo < j.limit_hi && j.motor_torque == 0.0f) g.limits = f4{j.limit_lo, j.limit_hi, 0.0f, 0.0f};
        }
        float massA = j.body_a >= 0 ? H.posLin[j.body_a].w : 0.0f;
        float massB = H.posLin[j.body_b].w;
        float eff = 0.0f;
        bool have = false;
        for (float m : {massA, massB}) if (m > 0.0f) { eff = have ? fmin_(eff, m) : m; have = true; }
        float floorK = fmin_(1.0e9f, fmax_(1.0f, eff / fmax_(dt * dt, 1.0e-12f)));
        if (std::isinf(j.stiffness_lin)) g.penaltyLin = f4{floorK, floorK, floorK, floorK};
        if (std::isinf(j.stiffness_ang)) g.penaltyAng = f4{floorK, floorK, floorK, floorK};
        if (j.stiffness_lin > 0.0f && std::isfinite(j.stiffness_lin)) { float k = fmin_(j.stiffness_lin, 1e9f); g.penaltyLin = f4{k, k, k, k}; }
        if (j.stiffness_ang > 0.0f && std::isfinite(j.stiffness_ang)) { float k = fmin_(j.stiffness_ang, 1e9f); g.penaltyAng = f4{k, k, k, k}; }
        H.joints[i] = g;
        // A joint with zero stiffness and no motor is an exclusion marker: no
        // stage ever reads it (adjacency skips it, its penalties warm-start
        // to zero so the dual is a no-op, and it is never breakable in effect).
        bool inert = g.rA.w == 0.0f && g.rB.w == 0.0f && g.motor.y == 0.0f;
        if (!inert) H.activeJoints.push_back(i);
    }
    H.initPenLin.resize(nj); H.initPenAng.resize(nj);
    for (uint32_t i = 0; i < nj; i++) { H.initPenLin[i] = H.joints[i].penaltyLin; H.initPenAng[i] = H.joints[i].penaltyAng; }

    // ---- springs (GPUSolver.swift:1197-1212)
    H.springs.assign(s->num_springs, SpringGPU{});
    for (uint32_t i = 0; i < s->num_springs; i++) {
        const avbd_spring_desc& sp = s->springs[i];
        SpringGPU g{};
        g.header = u4{(uint32_t)sp.body_a, (uint32_t)sp.body_b, sp.hard ? 1u : 0u, 0};
        float rest = sp.rest;
        if (rest < 0.0f) {
            V3 pA = add(qrot(H.posAng[sp.body_a], from(sp.r_a)), V3{H.posLin[sp.body_a].x, H.posLin[sp.body_a].y, H.posLin[sp.body_a].z});
            V3 pB = add(qrot(H.posAng[sp.body_b], from(sp.r_b)), V3{H.posLin[sp.body_b].x, H.posLin[sp.body_b].y, H.posLin[sp.body_b].z});
            rest = length(sub(pA, pB));
        }
        g.rA = f4{sp.r_a[0], sp.r_a[1], sp.r_a[2], sp.stiffness};
        g.rB = f4{sp.r_b[0], sp.r_b[1], sp.r_b[2], rest};
        H.springs[i] = g;
        if (sp.hard) H.hardSprings.push_back(i);
    }

    // ---- tets (GPUSolver.swift:1214-1235): rows of Dm^-1 via the adjugate
    H.tets.assign(s->num_tets, TetGPU{});
    for (uint32_t i = 0; i < s->num_tets; i++) {
        const avbd_tet_desc& t = s->tets[i];
        auto P3 = [&](int id) { return V3{H.posLin[id].x, H.posLin[id].y, H.posLin[id].z}; };
        V3 x0 = P3(t.ids[0]);
        V3 d0 = sub(P3(t.ids[1]), x0), d1 = sub(P3(t.ids[2]), x0), d2 = sub(P3(t.ids[3]), x0);
        float six = dot(d0, cross(d1, d2));
        float vol = std::fabs(six) / 6.0f;
        V3 r0 = divs(cross(d1, d2), six), r1 = divs(cross(d2, d0), six), r2 = divs(cross(d0, d1), six);
        TetGPU g{};
        g.ids = u4{(uint32_t)t.ids[0], (uint32_t)t.ids[1], (uint32_t)t.ids[2], (uint32_t)t.ids[3]};
        g.r0 = f4{r0.x, r0.y, r0.z, six};
        g.r1 = f4{r1.x, r1.y, r1.z, t.mu * vol};
        g.r2 = f4{r2.x, r2.y, r2.z, t.lambda * vol};
        H.tets[i] = g;
    }

    // ---- collision exclusions (GPUSolver.swift:1265-1287)
    std::vector<uint64_t> ex;
    auto key = [](int a, int b) { return ((uint64_t)std::min(a, b) << 32) | (uint64_t)std::max(a, b); };
    for (uint32_t i = 0; i < nj; i++) if (s->joints[i].body_a >= 0) ex.push_back(key(s->joints[i].body_a, s->joints[i].body_b));
    for (uint32_t i = 0; i < s->num_springs; i++) ex.push_back(key(s->springs[i].body_a, s->springs[i].body_b));
    for (uint32_t i = 0; i < s->num_exclusions; i++) ex.push_back(key(s->exclusions[i].body_a, s->exclusions[i].body_b));
    std::sort(ex.begin(), ex.end());
    ex.erase(std::unique(ex.begin(), ex.end()), ex.end());
    for (uint64_t k : ex) { H.exclusions.push_back((uint32_t)(k >> 32)); H.exclusions.push_back((uint32_t)k); }

    // ---- cloth topology and elements (GPUSolver.swift:1289-1680)
    H.cloth = s->num_tris > 0;
    if (H.numTris > 0) {
        upload_cloth(s, boundary, H);
        // Element contacts (V-T, E-E, rigid feature vs triangle) can arise
        // unless the scene has a single closed soft surface, no authored
        // triangles, no self-collision and no rigid collider other than
        // large static ground slabs whose corners lie far outside the scene:
        // then the isotropic-OGC stages would produce nothing and are skipped.
        std::set<uint32_t> groups;
        bool self = false;
        for (uint32_t v : H.particleIdx) { groups.insert(H.clothGroup[v]); self = self || H.selfCollision[v] != 0; }
        bool rigidReach = false;
        for (uint32_t i = 0; i < nc; i++) {
            const avbd_collider_desc& c = s->colliders[i];
            if (!c.collision_enabled || s->bodies[c.body].is_particle) continue;
            const bool slab = !H.isDynamic[c.body] && c.shape == AVBD_SHAPE_BOX && c.hull_count == 0 && c.size[0] >= 20.0f && c.size[1] >= 20.0f;
            rigidReach = rigidReach || !slab;
        }
        H.ogc = H.cloth || groups.size() > 1 || self || rigidReach;
    }

    // ---- static palette for soft scenes (GPUSolver.swift:1956-2049)
    H.dynamicColoring = (H.numTris == 0 && s->num_tets == 0);
    H.colors.assign(nb, 0);
    for (uint32_t i = 0; i < nb; i++) H.colors[i] = i % MAX_COLORS;
    H.colorStart.assign(MAX_COLORS + 2, 0);
    H.colorCounts.assign(MAX_COLORS, 0);
    if (!H.dynamicColoring) {
        std::vector<std::vector<uint32_t>> adj(nb);
        auto link2 = [&](int a, int b) {
            if (a < 0 || b < 0) return;
            if (H.isDynamic[a] && H.isDynamic[b]) { adj[a].push_back((uint32_t)b); adj[b].push_back((uint32_t)a); }
        };
        for (uint32_t i = 0; i < nj; i++) {
            const avbd_joint_desc& j = s->joints[i];
            if (j.stiffness_lin != 0.0f || j.stiffness_ang != 0.0f || j.motor_torque != 0.0f) link2(j.body_a, j.body_b);
        }
        for (uint32_t i = 0; i < s->num_springs; i++) link2(s->springs[i].body_a, s->springs[i].body_b);
        for (uint32_t i = 0; i < s->num_tets; i++)
            for (int a = 0; a < 4; a++) for (int b = a + 1; b < 4; b++) link2(s->tets[i].ids[a], s->tets[i].ids[b]);
        uint32_t maxColor = 0;
        std::vector<uint32_t> colors(nb, 0);
        for (uint32_t v = 0; v < nb; v++) {
            if (!H.isDynamic[v]) continue;
            uint64_t used = 0;
            for (uint32_t n : adj[v]) if (n < v && colors[n] < 64) used |= 1ull << colors[n];
            if (used == ~0ull) { err = "static coloring needs more than 64 colors"; return AVBD_ERR_RUNTIME_FAILURE; }
            uint32_t c = 0;
            while (used & (1ull << c)) c++;
            colors[v] = c;
            maxColor = std::max(maxColor, c);
        }
        H.staticUsedColors = maxColor + 1;
        std::vector<std::vector<uint32_t>> buckets(MAX_COLORS);
        for (uint32_t v = 0; v < nb; v++) if (H.isDynamic[v]) buckets[colors[v]].push_back(v);
        for (int c = 0; c < MAX_COLORS; c++) {
            H.colorStart[c] = (uint32_t)H.colorList.size();
            H.colorCounts[c] = (uint32_t)buckets[c].size();
            H.colorList.insert(H.colorList.end(), buckets[c].begin(), buckets[c].end());
        }
        H.colorStart[MAX_COLORS] = (uint32_t)H.colorList.size();
        H.colorStart[MAX_COLORS + 1] = H.staticUsedColors;
        for (uint32_t v = 0; v < nb; v++) H.colors[v] = colors[v];
    }

    // ---- static adjacency segments (40_solver.metal:27-243, static kinds)
    std::vector<std::vector<uint32_t>> pre(nb), post(nb);
    auto dyn = [&](uint32_t b) { return b != WORLD_BODY && H.posLin[b].w > 0.0f; };
    for (uint32_t g : H.activeJoints) {
        uint32_t e = (FK_JOINT << ADJ_KIND_SHIFT) | g;
        if (dyn(H.joints[g].header.x)) pre[H.joints[g].header.x].push_back(e);
        if (dyn(H.joints[g].header.y)) pre[H.joints[g].header.y].push_back(e);
    }
    for (uint32_t i = 0; i < H.springs.size(); i++) {
        uint32_t e = (FK_SPRING << ADJ_KIND_SHIFT) | i;
        if (dyn(H.springs[i].header.x)) pre[H.springs[i].header.x].push_back(e);
        if (dyn(H.springs[i].header.y)) pre[H.springs[i].header.y].push_back(e);
    }
    for (uint32_t t = 0; t < H.tets.size(); t++) {
        uint32_t e = (FK_TET << ADJ_KIND_SHIFT) | t;
        for (uint32_t v : {H.tets[t].ids.x, H.tets[t].ids.y, H.tets[t].ids.z, H.tets[t].ids.w})
            if (dyn(v)) post[v].push_back(e);
    }
    for (uint32_t m = 0; m < H.membranes.size(); m++) {
        const uint32_t e = (FK_MEMBRANE << ADJ_KIND_SHIFT) | m;
        for (uint32_t v : {H.membranes[m].ids.x, H.membranes[m].ids.y, H.membranes[m].ids.z})
            if (dyn(v)) post[v].push_back(e);
    }
    for (uint32_t b = 0; b < H.bends.size(); b++) {
        const uint32_t e = (FK_BEND << ADJ_KIND_SHIFT) | b;
        for (uint32_t v : {H.bends[b].ids.x, H.bends[b].ids.y, H.bends[b].ids.z, H.bends[b].ids.w})
            if (dyn(v)) post[v].push_back(e);
    }
    // The warp-per-particle primal may drop its generic stamp path when no
    // dynamic body is rigid and no particle carries a joint or spring entry
    // (sphere contacts always have exactly one contact point).
    H.particleFastPath = !H.cloth && !H.ogc;
    for (uint32_t b = 0; b < nb && H.particleFastPath; b++) {
        if (!(H.posLin[b].w > 0.0f)) continue;
        if (H.shape[b].w >= 0.0f || !pre[b].empty()) { H.particleFastPath = false; break; }
    }
    // lanes per body for each static color: enough for the largest static
    // adjacency plus one contact entry in a single pass
    H.colorLanes.assign(MAX_COLORS, 8);
    if (!H.dynamicColoring) {
        for (int c = 0; c < MAX_COLORS; c++) {
            size_t mx = 0;
            for (uint32_t i = H.colorStart[c]; i < H.colorStart[c + 1]; i++) {
                const uint32_t b = H.colorList[i];
                mx = std::max(mx, pre[b].size() + post[b].size() + 1);
            }
            H.colorLanes[c] = mx <= 8 ? 8u : (mx <= 16 ? 16u : 32u);
        }
    }
    // launch order of each static color: lean particles, then the rest
    // (bodies are independent within a color, so the order only decides
    // which kernel instance takes a body)
    H.colorLaunch.clear();
    H.colorLean.assign(MAX_COLORS, 0);
    if (!H.dynamicColoring) {
        const bool clothKinds = H.cloth || H.ogc;
        auto lean = [&](uint32_t b) {
            if (H.shape[b].w >= 0.0f) return false;                       // rigid
            for (uint32_t e : pre[b])
                if (!clothKinds || (e >> ADJ_KIND_SHIFT) != FK_SPRING) return false;
            if (!clothKinds)
                for (uint32_t e : post[b])
                    if ((e >> ADJ_KIND_SHIFT) != FK_TET) return false;
            return true;
        };
        H.colorLaunch.reserve(H.colorList.size());
        for (int c = 0; c < MAX_COLORS; c++) {
            const uint32_t s0 = H.colorStart[c], s1 = H.colorStart[c + 1];
            for (uint32_t i = s0; i < s1; i++)
                if (lean(H.colorList[i])) H.colorLaunch.push_back(H.colorList[i]);
            H.colorLean[c] = (uint32_t)H.colorLaunch.size() - s0;
            for (uint32_t i = s0; i < s1; i++)
                if (!lean(H.colorList[i])) H.colorLaunch.push_back(H.colorList[i]);
        }
    }
    H.staticSeg.assign(nb, u4{});
    H.postTets.assign(nb, 0);
    for (uint32_t b = 0; b < nb; b++) {
        std::sort(pre[b].begin(), pre[b].end());
        std::sort(post[b].begin(), post[b].end());
        for (uint32_t e : post[b]) H.postTets[b] += (e >> ADJ_KIND_SHIFT) == FK_TET ? 1u : 0u;
        H.staticSeg[b] = u4{(uint32_t)H.preList.size(), (uint32_t)pre[b].size(),
                            (uint32_t)H.postList.size(), (uint32_t)post[b].size()};
        H.preList.insert(H.preList.end(), pre[b].begin(), pre[b].end());
        H.postList.insert(H.postList.end(), post[b].begin(), post[b].end());
    }
    // tet records in incidence order: a vertex's lanes read its tets'
    // records contiguously instead of following each entry to the record.
    // Kept only while the copy stays small beside the 126 MB L2 (measured:
    // soft cube, 15.6 MB, 0.767 -> 0.745 ms per frame; mixed scene, 60 MB,
    // 5.34 -> 5.58 ms, its working set no longer fits)
    H.tetInc.clear();
    if (!H.tets.empty() && H.postList.size() * sizeof(TetGPU) <= (32u << 20)) {
        H.tetInc.assign(H.postList.size(), TetGPU{});
        for (uint32_t b = 0; b < nb; b++)
            for (uint32_t i = 0; i < H.postTets[b]; i++) {
                const uint32_t q = H.staticSeg[b].z + i;
                H.tetInc[q] = H.tets[H.postList[q] & ADJ_INDEX_MASK];
            }
    }

    // learned warm start rows: every dynamic particle, then every dynamic
    // rigid body (3-DOF and 6-DOF corrections)
    H.learnIdx.clear();
    for (uint32_t b = 0; b < nb; b++)
        if (s->bodies[b].is_particle && H.posLin[b].w > 0.0f) H.learnIdx.push_back(b);
    H.P.learnParticles = (uint32_t)H.learnIdx.size();
    for (uint32_t b = 0; b < nb; b++)
        if (!s->bodies[b].is_particle && H.posLin[b].w > 0.0f) H.learnIdx.push_back(b);
    H.P.learnRigid = 0;

    // ---- spinners and parameters (GPUSolver.swift:630-637, :2052-2080)
    H.spinners.assign(s->spinners, s->spinners + s->num_spinners);
    for (const auto& sp : H.spinners) {
        if (sp.body < 0 || (uint32_t)sp.body >= nb) { err = "spinner body out of range"; return AVBD_ERR_INVALID_ARGUMENT; }
        H.spinVel[sp.body] = f4{sp.axis[0] * sp.omega, sp.axis[1] * sp.omega, sp.axis[2] * sp.omega, 1.0f};
    }
    Params& P = H.P;
    P.numBodies = nb;
    P.numJoints = nj;
    P.numSprings = (uint32_t)H.springs.size();
    P.numTets = (uint32_t)H.tets.size();
    P.mapCapacity = H.mapCapacity;
    P.maxPairs = H.maxPairs;
    P.cellSize = maxHashedRadius * 2.0f;
    P.gridHashSize = H.gridHashSize;
    P.numHashed = (uint32_t)H.hashedIdx.size();
    P.numGlobals = (uint32_t)H.globalIdx.size();
    P.numHashedRigid = numHashedRigid;
    P.roundShapes = 0u;
    for (uint32_t i = 0; i < nc; i++)
        if ((H.colShapeType[i] & SHAPE_KIND_MASK) >= 2u) P.roundShapes = 1u;
    // Particle grid: when the coarse cells (twice the largest hashed radius,
    // at least 0.1 m) are well above the particles, particle candidates come
    // from cells just above twice the largest particle radius (two
    // overlapping particles always lie in neighbouring fine cells) instead of
    // the coarse buckets; the pair kernel keeps exactly the candidates the
    // coarse scan accepts.
    P.fineCellSize = 2.02f * maxParticleRadius;
    P.fineBP = (numHashedParticles > 0 && P.fineCellSize > 0.0f && P.cellSize >= 2.0f * P.fineCellSize) ? 1u : 0u;
    P.fineHashSize = std::min<uint32_t>(next_pow2(std::max<uint32_t>(64u, 2u * numHashedParticles)), 1u << 20);
    P.numTris = H.numTris;
    P.numParticles = H.numTris == 0 ? 0 : H.numParticles;
    P.maxSpeed = fmax_(30.0f, 1.5f * P.cellSize / dt * 0.5f);
    // effectiveSurfaceTruncationMode (GPUSolver.swift:93-101)
    P.surfaceTruncationMode = 0;
    if (P.numParticles > 0) {
        bool volumetricSelf = false;
        for (uint32_t i = 0; i < s->num_tets; i++) volumetricSelf = volumetricSelf || s->tets[i].self_collision;
        const uint32_t automatic = (volumetricSelf || (s->num_tris > 0 && s->num_tets == 0)) ? 2u : 1u;
        P.surfaceTruncationMode = s->truncation_selection == AVBD_TRUNCATION_AUTOMATIC ? automatic : s->truncation_selection;
    }
    if (P.surfaceTruncationMode == 2u && s->num_tets > 0) { err = "Planar-DAT truncation of tet surfaces is not supported by this library"; return AVBD_ERR_UNSUPPORTED; }
    P.cloth = (H.cloth && P.surfaceTruncationMode == 2u) ? 1u : 0u;
    H.ogc = H.ogc && P.surfaceTruncationMode == 1u;
    P.ogc = H.ogc ? 1u : 0u;
    // Element contacts couple bodies that share a static color: those scenes
    // solve a color against its pre-color pose and publish it afterwards.
    P.colorJacobi = (P.cloth || P.ogc) ? 1u : 0u;
    P.numEdges = H.numEdges;
    P.numSurfaceEdges = H.numSurfaceEdges;
    P.elemHashSize = H.elemHashSize;
    P.maxDatPairs = H.maxDatPairs;
    P.maxSoft = H.maxSoft;
    P.softMapCapacity = H.softMapCapacity;
    P.numMembranes = (uint32_t)H.membranes.size();
    P.numBends = (uint32_t)H.bends.size();
    P.elemMargin = H.elemMargin;
    P.queryRadius = H.queryRadius;
    P.elemCellSize = H.elemCellSize;
    P.surfaceCellSize = H.surfaceCellSize;
    P.clothViscosity = s->settings.cloth_viscosity;
    P.tetInversionPreventionEnabled = 0;
    P.planarDATRelaxation = 0.85f;
    P.numExclusions = (uint32_t)(H.exclusions.size() / 2);
    if (P.ogc) {
        // isotropic element contacts: detection-radius cells, authored
        // contact edges only, the isotropic soft-contact budget
        // (GPUSolver.swift:2117-2133)
        P.elemCellSize = H.surfaceCellSize;
        P.numEdges = H.numSurfaceEdges;
        P.maxSoft = H.maxSoftIso;
        P.softMapCapacity = H.softMapCapacityIso;
    }
    return AVBD_OK;
}

}  // namespace avbd
