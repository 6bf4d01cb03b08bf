// upload.h — host-side scene upload: turns an avbd_scene_desc into the
// device-ready arrays of one solver (GPUSolver.swift:338-638, :901-2081).
#pragma once
#include <string>
#include <vector>

#include "../../include/avbd.h"
#include "avbd_types.h"

namespace avbd {

struct HostScene {
    // capacities
    uint32_t numBodies = 0, numColliders = 0;
    uint32_t maxPairs = 0, mapCapacity = 0, gridHashSize = 0;
    uint32_t numTris = 0, numParticles = 0;
    bool dynamicColoring = true;
    uint32_t staticUsedColors = 1;
    uint32_t numDynamicBodies = 0;
    bool particleFastPath = false;   // all dynamic bodies are particles without joints/springs
    Params P{};

    // bodies (SoA float4)
    std::vector<f4> posLin, posAng, velLin, velAng, prevVelLin, props, shape, spinVel;
    std::vector<float> gravityScale;
    std::vector<uint32_t> shapeType, clothGroup;
    std::vector<uint8_t> isDynamic;

    // colliders
    std::vector<uint32_t> colOwner, colShapeType, colGroup, colShared;
    std::vector<f4> colShape, colLocalPos, colLocalRot;
    std::vector<float> colFriction;  // (static, dynamic) pairs
    std::vector<uint32_t> colHullRange;  // (first vertex, vertex count) pairs
    std::vector<f4> hullVerts;
    std::vector<uint32_t> hashedIdx, globalIdx;

    // constraints
    std::vector<JointGPU> joints;
    std::vector<f4> initPenLin, initPenAng;
    std::vector<uint32_t> activeJoints;   // non-inert joints: the only ones any stage reads
    std::vector<SpringGPU> springs;
    std::vector<uint32_t> hardSprings;
    std::vector<TetGPU> tets;
    std::vector<uint32_t> exclusions;     // sorted (lo, hi) pairs, flattened
    std::vector<avbd_spinner_desc> spinners;
    std::vector<std::pair<uint32_t, float>> rateMotors;

    // static palette (soft scenes) in final form
    std::vector<uint32_t> colors, colorStart, colorList, colorCounts;
    std::vector<uint32_t> colorLanes;      // lanes per body for each static color
    // Primal launch order of each static color: the color's "lean"
    // particles first (every adjacency entry one of the particle term kinds:
    // tets, one-point manifolds, and with cloth or OGC also springs,
    // membranes, bends and element contacts), then the rest (rigid bodies,
    // particles with joints).  colorLean[c] counts the lean ones.
    std::vector<uint32_t> colorLaunch, colorLean;

    // Static per-body adjacency, split around the per-frame contact entries:
    // pre = joints + springs (kinds 0, 1), post = tets (kind 3), each sorted.
    // The solver walks pre, then this frame's manifolds (kind 2), then post,
    // which is exactly the ascending (kind << 28 | index) order.
    std::vector<uint32_t> preList, postList;
    std::vector<u4> staticSeg;            // preStart, preCount, postStart, postCount
    // tets (kind 3) at the head of each post segment: element contacts
    // (kind 4) go between them and the membranes / bends (kinds 5, 6)
    std::vector<uint32_t> postTets;
    // every tet record once per incident vertex, at the position of its entry
    // in postList (tets lead each body's static post segment)
    std::vector<TetGPU> tetInc;

    // cloth (authored triangles): element topology and elements.  In cloth
    // scenes the post segment holds membranes and bends (kinds 5, 6) and the
    // per-frame segment manifolds and element contacts (kinds 2, 4), which
    // keeps the walk in ascending order.
    bool cloth = false;
    uint32_t numEdges = 0, numSurfaceEdges = 0, elemHashSize = 64;
    uint32_t maxDatPairs = 1, maxSoft = 1, softMapCapacity = 64;
    float elemMargin = 0.0f, queryRadius = 0.0f, elemCellSize = 1.0f, surfaceCellSize = 1.0f;
    std::vector<u4> tris;
    std::vector<uint32_t> edges;          // (a, b) per edge
    std::vector<uint32_t> nbrStart, nbrCount, nbrList, particleIdx, selfCollision;
    std::vector<MembraneGPU> membranes;
    std::vector<BendGPU> bends;

    // isotropic OGC (25_cloth.metal:347-931): tracker propagation topology
    // and the 2-ring exclusion sets of the conservative bounds.  `ogc` is set
    // when element contacts can arise (several surfaces, authored triangles,
    // self-collision or rigid colliders that may reach a surface).
    bool ogc = false;
    std::vector<u4> triAdj;               // up to 3 edge-adjacent triangles per triangle
    std::vector<uint32_t> nbr2Start, nbr2Count, nbr2List;
    std::vector<uint32_t> vertEdgeStart, vertEdgeCount, vertEdgeList;
    std::vector<uint32_t> clothVert;      // 1 for vertices of authored triangles
    uint32_t maxSoftIso = 1, softMapCapacityIso = 64;

    // dynamic particles whose warm start the learned model may predict
    std::vector<uint32_t> learnIdx;
};

// Returns an AVBD_* status; on failure `err` holds a message.
int upload_scene(const avbd_scene_desc* s, HostScene& out, std::string& err);

}  // namespace avbd
