// oracle_solver.h — record layouts and the Solver state of the CPU oracle.
//
// TEST INFRASTRUCTURE, NOT PRODUCT CODE (see avbd_oracle.cpp).
#pragma once
#include "oracle_math.h"
#include "../include/avbd.h"

#include <algorithm>
#include <array>
#include <cfloat>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <set>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace oracle {

static const float PENALTY_MIN = 1.0f;
static const float PENALTY_MAX = 1.0e10f;
static const float PENALTY_MAX_T = 1.0e6f;
static const float STICK_THRESH = 0.00001f;
static const int MAX_COLORS = 64;
static const uint32_t WORLD_BODY = 0xFFFFFFFFu;
static const uint32_t FK_JOINT = 0, FK_SPRING = 1, FK_MANIFOLD = 2, FK_TET = 3,
                      FK_SOFT = 4, FK_MEMBRANE = 5, FK_BEND = 6;
static const int ADJ_KIND_SHIFT = 28;
static const uint32_t ADJ_INDEX_MASK = 0x0FFFFFFFu;
static const int MAX_CONTACTS = 8;
static const uint32_t MOTOR_MODE_MASK = 3u << 4, MOTOR_IMPLICIT = 1u << 4,
                      MOTOR_EXPLICIT = 2u << 4, MOTOR_VELOCITY = 3u << 4;

// ---- GPU record layouts (00_common.metal:330-431) ------------------------
struct JointGPU {
    U4 header;  // bodyA, bodyB, broken, flags
    F4 rA, rB, C0Lin, C0Ang, lambdaLin, lambdaAng, penaltyLin, penaltyAng,
        restRel, hingeAxis, motor, limits, dynamics;
};
struct SpringGPU { U4 header; F4 rA, rB, dual; };
struct TetGPU { U4 ids; F4 r0, r1, r2; };
struct ContactGPU { F4 rA, rB, C0, lambda, penalty; };
struct ManifoldGPU {
    U4 header;  // bodyA, bodyB, numContacts, flags (1 active, 2 roundA, 4 roundB)
    U4 colliderPair;
    F4 basisN, basisT1;
    ContactGPU contacts[MAX_CONTACTS];
};
static_assert(sizeof(JointGPU) == 224, "JointGPU layout");
static_assert(sizeof(SpringGPU) == 64, "SpringGPU layout");
static_assert(sizeof(TetGPU) == 64, "TetGPU layout");
static_assert(sizeof(ManifoldGPU) == 704, "ManifoldGPU layout");

// Cloth element records (00_common.metal:387-421).
struct MembraneGPU { U4 ids; F4 dm, mat; };      // StVK triangle: DmInv (a, b, c, d), (mu A, lambda A, A)
struct BendGPU { U4 ids; F4 K, mat; };           // Bergou hinge: cotangent K, 3 kappa / (A1 + A2)
struct SoftContactGPU {                          // 4-slot element contact
    U4 ids;
    F4 normal, anchorA, weights, C0, lambda, penalty;
};
static_assert(sizeof(MembraneGPU) == 48, "MembraneGPU layout");
static_assert(sizeof(BendGPU) == 48, "BendGPU layout");
static_assert(sizeof(SoftContactGPU) == 112, "SoftContactGPU layout");

static const uint32_t SC_VT = 1, SC_RT = 2, SC_EE = 3;
static const uint32_t SCF_RIGID_A = 1, SCF_SIDE_NEG = 2, SCF_KIND_SHIFT = 2, SCF_ROUND_A = 32;
static const uint32_t DAT_PAIR_VT = 0, DAT_PAIR_EE = 1, DAT_PAIR_TRUNCATE = 1, DAT_PAIR_CONTACT = 2;
static const uint32_t ELEM_EDGE_BIT = 0x80000000u;
static const float EE_INTERIOR_EPS = 0.02f;
static const float DAT_GEOMETRY_EPS = 1.0e-8f;
static const float DAT_TIME_MARGIN = 1.0e-3f;
static const uint32_t RT_MAX_PER_TRI = 4;

struct Params {
    float dt, gravity, alpha, betaLin, betaAng, gamma;
    uint32_t numBodies, numJoints, numSprings, mapCapacity, maxPairs;
    float cellSize;
    uint32_t gridHashSize, numHashed, numGlobals;
    float maxSpeed, lambdaMax;
    uint32_t iterations, numTets, numTris, numParticles;
    float rodDecayPow, particleDamping;
    uint32_t numHashedRigid, frame, frictionCombineMode;
    float collisionMargin, rigidLinearDamping, rigidAngularDamping;
    uint32_t surfaceTruncationMode, tetInversionPreventionEnabled;
    float planarDATRelaxation;
};

static uint32_t next_pow2(uint32_t v) {
    uint32_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

// Hash of an integer cell (20_broadphase.metal:16-28).
static inline uint32_t cell_hash(int cx, int cy, int cz, uint32_t group, uint32_t size) {
    uint32_t h = ((uint32_t)cx * 92837111u) ^ ((uint32_t)cy * 689287499u)
               ^ ((uint32_t)cz * 283923481u);
    h ^= group * 0x9e3779b9u;
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    return h & (size - 1u);
}
static inline void cell_coord(F3 p, float cs, int& x, int& y, int& z) {
    x = (int)std::floor(p.x / cs);
    y = (int)std::floor(p.y / cs);
    z = (int)std::floor(p.z / cs);
}
// Manifold persistence-map hash (20_broadphase.metal:547-553).
static inline uint32_t pair_map_hash(uint32_t a, uint32_t b, uint32_t cap) {
    uint32_t h = (a * 73856093u) ^ (b * 19349663u);
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    return h & (cap - 1u);
}
static inline bool groups_compatible(uint32_t a, uint32_t b) { return a == 0u || b == 0u || a == b; }
static inline bool domains_compatible(uint32_t ga, uint32_t gb, uint32_t sa, uint32_t sb) {
    if (!groups_compatible(ga, gb)) return false;
    if (ga == 0u && gb != 0u) return sb != 0u;
    if (gb == 0u && ga != 0u) return sa != 0u;
    return true;
}

struct Accum { M3 lhsLin, lhsAng, lhsCross; F3 rhsLin, rhsAng; };
static inline Accum accum_zero() { return Accum{m3_zero(), m3_zero(), m3_zero(), f3s(0), f3s(0)}; }
static inline Accum accum_add(const Accum& a, const Accum& b) {
    return Accum{m3_add(a.lhsLin, b.lhsLin), m3_add(a.lhsAng, b.lhsAng),
                 m3_add(a.lhsCross, b.lhsCross), a.rhsLin + b.rhsLin, a.rhsAng + b.rhsAng};
}

struct Solver {
    avbd_settings settings{};
    Params P{};
    uint32_t nb = 0, nc = 0;
    uint64_t frameIndex = 0;
    std::string error;
    int failure = AVBD_FAIL_NONE;
    int threads = 1;

    // bodies
    std::vector<F4> posLin, posAng, initLin, initAng, inertLin, inertAng, velLin, velAng,
        prevVelLin, props, shape, spinVel, ogcPrev;
    std::vector<float> gravityScale;
    std::vector<uint32_t> shapeType, boundsBits, clothGroup, clothVert;
    std::vector<uint8_t> isDynamic, isParticle;
    // colliders
    std::vector<uint32_t> colOwner, colShapeType, colGroup, colShared;
    std::vector<F4> colShape, colLocalPos, colLocalRot;
    std::vector<float> colFrictionS, colFrictionD;
    std::vector<uint32_t> colHullFirst, colHullCount;  // convex hull vertex range per collider
    std::vector<F3> hullVerts;
    std::vector<F4> scenePos;  // body positions of the scene description (skin rest poses)
    // skin bindings: ids, weights, rest normal, rows of Dm^-1
    struct Skin { U4 ids; F4 weights; F3 restNormal, inv0, inv1, inv2; };
    std::vector<Skin> skins;
    std::vector<uint32_t> hashedIdx, globalIdx, hashedRigidIdx;
    // constraints
    std::vector<JointGPU> joints;
    std::vector<F4> initPenLin, initPenAng;
    std::vector<SpringGPU> springs;
    std::vector<TetGPU> tets;
    std::vector<uint32_t> exclusions;  // (a, b) pairs, sorted
    std::vector<avbd_spinner_desc> spinners;
    struct RateMotor { uint32_t joint; float rate; };
    std::vector<RateMotor> rateMotors;
    // capacities
    uint32_t maxPairs = 0, mapCapacity = 0, gridHashSize = 0;
    uint32_t numTris = 0, numParticles = 0;
    bool dynamicColoring = true;
    uint32_t staticUsedColors = 1;
    // per-frame
    std::vector<uint32_t> cellCount, cellStart, cellBodies, cellRigid, bodyCellSlot;
    std::vector<uint32_t> pairCount, pairStart, pairs;
    std::vector<ManifoldGPU> manifolds, prevManifolds;
    std::vector<uint32_t> mapKeyA, mapKeyB, mapVal;
    std::vector<uint32_t> adjStart, adjCount, adjList;
    std::vector<uint32_t> colorsA, colorsB, colorStart, colorList;
    uint32_t numPairs = 0, pairCandidates = 0, colorConflicts = 0, ogcExceeded = 0;
    uint32_t colorCounts[MAX_COLORS] = {};

    // ---- cloth: element topology, contacts and Planar-DAT (25_cloth.metal,
    // 27_planar_dat.metal, upload GPUSolver.swift:1289-1680)
    bool cloth = false;                 // authored triangles present
    bool colorJacobi = false;           // same-color reads see the pre-color pose
    uint32_t numAuthoredTris = 0, numEdges = 0, numSurfaceEdges = 0;
    uint32_t elemHashSize = 64, maxDatPairs = 1, maxSoft = 1, softMapCapacity = 64;
    float elemMargin = 0.0f, queryRadius = 0.0f, elemCellSize = 1.0f, surfaceCellSize = 1.0f;
    float clothViscosity = 0.0f;
    std::vector<U4> tris;
    std::vector<uint32_t> edges;        // (a, b) per edge, a < b
    std::vector<uint32_t> nbrStart, nbrCount, nbrList, particleIdx, selfCollision;
    std::vector<MembraneGPU> membranes;
    std::vector<BendGPU> bends;
    std::vector<uint32_t> elemCellStart, elemCellCount, elemCells;
    std::vector<U4> datPairs;
    uint32_t datRaw = 0, datVT = 0, datEE = 0;
    std::vector<SoftContactGPU> soft, prevSoft;
    uint32_t softRaw = 0, numSoft = 0;
    std::vector<uint32_t> softKeyA, softKeyB, softVal;
    std::vector<uint32_t> truncBits;
    std::vector<F4> posNext, angNext;
    // isotropic OGC (25_cloth.metal:347-931): tracker topology, tracked sets
    // of this frame and the previous one, the exceeder count of the pass
    bool ogc = false;
    uint32_t maxSoftIso = 1, softMapCapacityIso = 64;
    std::vector<U4> triAdj, vtTrack, vtTrackPrev, eeTrack, eeTrackPrev;
    std::vector<uint32_t> nbr2Start, nbr2Count, nbr2List, vertEdgeStart, vertEdgeCount, vertEdgeList;
    std::vector<std::vector<uint32_t>> isoTriCells, isoEdgeCells;   // per bucket, ascending element index
    uint32_t ogcPass = 0;
    uint32_t numSoftRT = 0, numSoftVT = 0, numSoftEE = 0;
    struct DatCounters {
        uint32_t pairsPeak, vtPeak, eePeak, gridOverflow, invalidAnchor, truncations,
            vtDegenerate, eeDegenerate, nonfinite, tetDegenerate, softCandidates;
    } dat{};

    bool body_dynamic(uint32_t b) const { return b != WORLD_BODY && posLin[b].w > 0.0f; }
    // binary search of the sorted (lo, hi) exclusion pairs (20_broadphase.metal:134-147)
    bool pair_excluded_bodies(uint32_t a, uint32_t b) const {
        uint32_t lo = 0, hi = (uint32_t)(exclusions.size() / 2), count = hi;
        while (lo < hi) {
            uint32_t mid = (lo + hi) >> 1;
            uint32_t ex = exclusions[2 * mid], ey = exclusions[2 * mid + 1];
            if (ex < a || (ex == a && ey < b)) lo = mid + 1; else hi = mid;
        }
        return lo < count && exclusions[2 * lo] == a && exclusions[2 * lo + 1] == b;
    }

    // ---------------------------------------------------------------- upload
    int create(const avbd_scene_desc* s);
    void sync_params();
    void step();
    // stages
    void broadphase();
    uint32_t process_producer(uint32_t producer, bool emit, uint32_t base);
    void narrowphase();
    void narrow_one(uint32_t gid);
    void map_rebuild();
    int map_find(uint32_t a, uint32_t b) const;
    void warmstart_joints();
    void warmstart_bodies();
    void adjacency();
    void dynamic_coloring();
    void neighbor_colors(uint32_t entry, uint32_t self, uint32_t myColor,
                         const std::vector<uint32_t>& colorsIn, uint32_t& maskLo,
                         uint32_t& maskHi, uint32_t& allLo, uint32_t& allHi,
                         bool& conflict) const;
    void primal_color(uint32_t c);
    void primal_body(uint32_t body);
    void stamp_entry(uint32_t entry, uint32_t body, Accum& acc) const;
    void stamp_joint(const JointGPU& j, uint32_t self, Accum& acc) const;
    void stamp_spring(const SpringGPU& sp, uint32_t self, Accum& acc) const;
    void stamp_tet(const TetGPU& t, uint32_t self, Accum& acc) const;
    void stamp_manifold(const ManifoldGPU& m, uint32_t self, Accum& acc) const;
    void stamp_membrane(const MembraneGPU& m, uint32_t self, Accum& acc) const;
    void stamp_bend(const BendGPU& b, uint32_t self, Accum& acc) const;
    void stamp_soft(const SoftContactGPU& sc, uint32_t self, Accum& acc) const;
    F3 soft_c(const SoftContactGPU& sc, F3& n, F3& t1, F3& t2, F3& rAW, bool& rigidA) const;
    void dual_soft(uint32_t i);
    // cloth stages
    int cloth_upload(const avbd_scene_desc* s, const std::vector<std::array<int, 3>>& boundary);
    void elem_bounds(uint32_t e, F3& lo, F3& hi) const;
    void elem_grid();
    void dat_build_pairs();
    void rt_emit();
    void dat_emit_contacts();
    void soft_emit(U4 ids, F4 weights, F3 n, float friction, F3 anchorA, float C0n, float restT,
                   float lamCap, float minMass, uint32_t kind, bool rigidA, bool roundA, bool sideNeg,
                   uint32_t keyA, uint32_t keyB);
    int soft_map_find(uint32_t keyA, uint32_t keyB) const;
    float soft_prev_side(uint32_t keyA, uint32_t keyB, float proposed) const;
    void soft_map_rebuild();
    bool dat_unsafe() const;
    F3 cur_pos(uint32_t b, uint32_t activeColor) const;
    void dat_reduce(uint32_t activeColor);
    void dat_apply_particles();
    void dat_apply_color(uint32_t c);
    void dat_restore_failed_surface();
    void smooth_particle_velocities();
    // isotropic OGC stages
    void ogc_topology(const std::vector<std::array<int, 3>>& coll, const std::vector<std::vector<uint32_t>>& ring);
    void ogc_grid();
    void ogc_detect();
    void ogc_track_vt(uint32_t gid);
    void ogc_track_ee(uint32_t gid);
    bool vt_contact(uint32_t v, uint32_t t, bool emit);
    bool ee_contact(uint32_t gid, uint32_t e, bool emit);
    void ogc_refresh();
    void publish_color(uint32_t c);
    void dual_all();
    void dual_joint(uint32_t gid);
    void dual_spring(uint32_t si);
    void dual_manifold(uint32_t mi);
    void finalize();
    void advance_spinners();
    float max_constraint_error() const;
    // AL residual: per body the squared norm of the primal's right-hand side
    // (the gradient of the augmented-Lagrangian objective), summed in double
    float body_residual_sq(uint32_t body) const;
    double residual() const;
    // Stage observer for the pinning harness (oracle/ref_pin.cpp): called
    // before (after = 0) and after (after = 1) every stage of a frame.
    enum Stage { ST_BROADPHASE, ST_NARROWPHASE, ST_MAP, ST_WARM_JOINTS, ST_WARM_BODIES, ST_ADJACENCY,
                 ST_COLORING, ST_PRIMAL, ST_DUAL, ST_FINALIZE, ST_COUNT_ };
    typedef void (*StageHook)(Solver* s, int stage, int arg, int after, void* ctx);
    StageHook stageHook = nullptr;
    void* stageCtx = nullptr;
    void hook(int stage, int arg, int after) { if (stageHook) stageHook(this, stage, arg, after, stageCtx); }
    bool traceEnabled = false;
    std::vector<double> trace;   // [0] warm start (plain), [1] warm start used, [2 + k] after iteration k
};

}  // namespace oracle
