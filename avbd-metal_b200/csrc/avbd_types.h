// avbd_types.h — device-resident records of the solver step, shared by host
// and CUDA code.
//
// Layouts are float4/uint4-granular and match the reference's GPU record ABI
// field for field (Sources/PhysicsAVBD/Shaders/00_common.metal:233-468), so a
// record read back with avbd_debug_read() can be compared byte-for-byte with
// the reference's definition.  The parameter block below is the subset of
// `SimParams` the implemented stages consume.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define AVBD_HD __host__ __device__
#else
#define AVBD_HD
#endif

namespace avbd {

struct alignas(16) f4 { float x, y, z, w; };
struct alignas(16) u4 { uint32_t x, y, z, w; };

constexpr float PENALTY_MIN = 1.0f;
constexpr float PENALTY_MAX = 1.0e10f;
constexpr float PENALTY_MAX_T = 1.0e6f;
constexpr float STICK_THRESH = 0.00001f;
constexpr int MAX_COLORS = 64;
constexpr int MAX_CONTACTS = 8;
constexpr uint32_t WORLD_BODY = 0xFFFFFFFFu;
constexpr uint32_t FK_JOINT = 0, FK_SPRING = 1, FK_MANIFOLD = 2, FK_TET = 3, FK_SOFT = 4,
                   FK_MEMBRANE = 5, FK_BEND = 6;
constexpr int ADJ_KIND_SHIFT = 28;
constexpr uint32_t ADJ_INDEX_MASK = 0x0FFFFFFFu;
constexpr uint32_t MOTOR_MODE_MASK = 3u << 4;
constexpr uint32_t MOTOR_IMPLICIT = 1u << 4;
constexpr uint32_t MOTOR_EXPLICIT = 2u << 4;
constexpr uint32_t MOTOR_VELOCITY = 3u << 4;
constexpr uint32_t SHAPE_KIND_MASK = 0xFu;
constexpr uint32_t SHAPE_PARTICLE = 0x10u;
constexpr uint32_t COLLIDER_WORLD_ROUND_ANCHOR = 0x20u;

struct JointGPU {
    u4 header;      // bodyA (WORLD_BODY = world), bodyB, broken, flags
    f4 rA;          // w = stiffnessLin
    f4 rB;          // w = stiffnessAng
    f4 C0Lin;       // w = torqueArm
    f4 C0Ang;       // w = fracture
    f4 lambdaLin, lambdaAng, penaltyLin, penaltyAng;
    f4 restRel;     // rest relative rotation qA^-1 qB
    f4 hingeAxis;   // xyz axis in B local; w != 0 -> hinge
    f4 motor;       // target, effort limit, pad, kp
    f4 limits;      // lo, hi, kd, pad
    f4 dynamics;    // armature, predicted twist, explicit effort
};
struct SpringGPU { u4 header; f4 rA, rB, dual; };      // dual: lambda, penalty, C0
struct TetGPU { u4 ids; f4 r0, r1, r2; };               // DmInv rows; w: 6V, muV, lamV
struct ContactGPU { f4 rA, rB, C0, lambda, penalty; };  // rA.w feature, rB.w stick
struct ManifoldGPU {
    u4 header;        // bodyA, bodyB, numContacts, flags (1 active, 2 roundA, 4 roundB)
    u4 colliderPair;
    f4 basisN;        // w = dynamic friction
    f4 basisT1;       // w = static friction
    ContactGPU contacts[MAX_CONTACTS];
};
static_assert(sizeof(JointGPU) == 224, "JointGPU layout");
static_assert(sizeof(SpringGPU) == 64, "SpringGPU layout");
static_assert(sizeof(TetGPU) == 64, "TetGPU layout");
static_assert(sizeof(ManifoldGPU) == 704, "ManifoldGPU layout");

// Cloth element records (00_common.metal:387-421).
struct MembraneGPU { u4 ids; f4 dm, mat; };   // StVK: DmInv (a, b, c, d); (mu A, lambda A, A)
struct BendGPU { u4 ids; f4 K, mat; };        // Bergou hinge: cotangent K; 3 kappa / (A1 + A2)
struct SoftContactGPU {                       // element contact on a 4-slot stencil
    u4 ids;       // WORLD_BODY = unused slot
    f4 normal;    // w = friction
    f4 anchorA;   // rigid slot-0 local anchor, or (restT, 0, 0); w = flag bits
    f4 weights;
    f4 C0;        // x = normal gap at step start; w = lambda cap
    f4 lambda;    // w = persistence key A (bits)
    f4 penalty;   // w = persistence key B (bits)
};
static_assert(sizeof(MembraneGPU) == 48, "MembraneGPU layout");
static_assert(sizeof(BendGPU) == 48, "BendGPU layout");
static_assert(sizeof(SoftContactGPU) == 112, "SoftContactGPU layout");

constexpr uint32_t SC_VT = 1, SC_RT = 2, SC_EE = 3;
constexpr uint32_t SCF_RIGID_A = 1, SCF_SIDE_NEG = 2, SCF_KIND_SHIFT = 2, SCF_ROUND_A = 32;
constexpr uint32_t DAT_PAIR_VT = 0, DAT_PAIR_EE = 1, DAT_PAIR_TRUNCATE = 1, DAT_PAIR_CONTACT = 2;
constexpr uint32_t ELEM_EDGE_BIT = 0x80000000u;
constexpr uint32_t RT_MAX_PER_TRI = 4;
constexpr uint32_t FULL_PASS = 0xFFFFFFFFu;

// Per-frame parameters (SimParams, 00_common.metal:233-288), passed by value.
struct Params {
    float dt, gravity, alpha, betaLin, betaAng, gamma;
    uint32_t numBodies, numJoints, numSprings, mapCapacity, maxPairs;
    float cellSize;
    uint32_t gridHashSize, numHashed, numGlobals;
    float maxSpeed, lambdaMax;
    uint32_t iterations, numTets, numTris, numParticles;
    float rodDecayPow, particleDamping;
    uint32_t numHashedRigid, frictionCombineMode;
    float collisionMargin, rigidLinearDamping, rigidAngularDamping;
    uint32_t surfaceTruncationMode, tetInversionPreventionEnabled;
    float planarDATRelaxation;
    uint32_t numExclusions;
    // cloth element pipeline (Planar-DAT)
    uint32_t cloth;                   // authored triangles: element contacts + Planar-DAT
    uint32_t colorJacobi;             // the primal writes posNext; a commit pass publishes it
    uint32_t numEdges, numSurfaceEdges, elemHashSize;
    uint32_t maxDatPairs, maxSoft, softMapCapacity, numMembranes, numBends;
    float elemMargin, queryRadius, elemCellSize, surfaceCellSize, clothViscosity;
    // isotropic OGC element contacts (tet surfaces, mixed scenes)
    uint32_t ogc;
    // particle grid of the broadphase (rigid colliders much larger than the
    // particles): cell size and hash size
    uint32_t fineBP, fineHashSize;
    float fineCellSize;
    // the scene has torus, capsule or convex-hull colliders (second
    // narrowphase pass)
    uint32_t roundShapes;
    // learned warm start: particle rows lead the learned list, dynamic rigid
    // bodies follow; learnRigid = the model predicts rigid corrections too
    uint32_t learnParticles, learnRigid;
};

// Device counters of one frame (the reference's CTR_* layout, trimmed).
struct Counters {
    uint32_t numPairs;
    uint32_t pairCandidates;
    uint32_t colorConflicts;
    uint32_t ogcExceeded;
    uint32_t usedColors;
    uint32_t waitTimeouts;
    uint32_t pad[2];
    uint32_t colorCount[MAX_COLORS];
    uint32_t colorStart[MAX_COLORS + 2];
    uint32_t changed[32];
    // element contacts and Planar-DAT (CTR_SOFT .. CTR_DAT_TET_DEGENERATE)
    uint32_t numSoftRT;       // rigid-triangle records at the head of the soft list
    uint32_t softRaw;         // soft demand before capacity clipping
    uint32_t numSoft;         // stored soft records
    uint32_t datRaw, datStored, datVT, datEE;   // current pair stream
    uint32_t datPairsPeak, datVTPeak, datEEPeak;
    uint32_t datGridOverflow, datInvalidAnchor, datTruncations;
    uint32_t datVTDegenerate, datEEDegenerate, datNonfinite, datTetDegenerate;
    // isotropic OGC bound exceeders: [0], [1] alternate over the iterations
    // (the refresh after iteration k reads slot k & 1 and clears the other);
    // [2], [3] count the plain and predicted trial sweeps of the learned warm
    // start
    uint32_t ogcSlots[4];
    uint32_t numSoftVT, numSoftEE;   // isotropic element contacts of this frame
    uint32_t ogcQueue;               // trackers that reseed from the grid this frame
    uint32_t adjLong;                // bodies whose contact segment is sorted by a block
};

}  // namespace avbd
