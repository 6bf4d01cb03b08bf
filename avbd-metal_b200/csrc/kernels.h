// kernels.h — device buffers of one solver and the host launchers of every
// stage kernel.  All launches go to the solver's stream, so one frame is a
// fixed launch sequence that the runtime captures into a CUDA graph.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "avbd_types.h"

namespace avbd {

struct DevPtrs {
    // bodies
    float4 *posLin, *posAng, *initLin, *initAng, *inertLin, *inertAng;
    float4 *velLin, *velAng, *prevVelLin, *props, *shape, *spinVel;
    float* gravityScale;
    uint32_t* clothGroup;
    uint32_t* bodyShape;                  // AVBD_SHAPE_* of each body
    // colliders
    uint32_t *colOwner, *colShapeType, *colGroup, *colShared;
    float4 *colShape, *colLocalPos, *colLocalRot;
    float2* colFriction;
    uint2* colHullRange;                  // (first vertex, vertex count); count 0 = analytic shape
    float4* hullVerts;                    // convex hull vertices in the collider frame
    uint32_t *hashedIdx, *globalIdx;
    uint32_t* exclusions;                 // uint2 pairs
    // broadphase
    uint32_t *cellCount, *cellStart, *cellBodies, *cellRigid;
    uint32_t* cellTmp;                    // bucket contents before the per-bucket sort
    uint32_t* colBucket;                  // bucket of every hashed collider this frame
    uint32_t *rigidStart, *rigidCells;    // rigid colliders of each bucket, in bucket order
    // particle grid (P.fineBP): particle colliders in cells of twice the
    // largest particle radius
    uint32_t *fineCount, *fineStart, *fineTmp, *fineCells;
    uint2* fineSlot;
    uint32_t* heavyProducers;             // producer indices of hashed rigid colliders (particle grid on)
    // per chunk of 32 consecutive global colliders (more than 32 globals):
    // box of their collider spheres (lo, hi) and of their bodies' bounding
    // spheres (lo, hi), this frame
    float4* globalChunk;
    // per global collider g: its owner body (set at upload) and, rewritten
    // by the chunk pass every frame, the owner's pose and shape in one place:
    // [3g] position + bounding radius (shape.w), [3g+1] rotation,
    // [3g+2] shape.xyz + AVBD_SHAPE_* kind (as float bits)
    uint32_t* globalOwner;
    float4* globalRec;
    uint2* bodyCellSlot;
    uint32_t *pairCount, *pairStart, *pairLaneCount;
    uint2* pairs;
    float4* colCenter;                    // per frame: world center xyz, |radius|
    uint4* colMeta;                       // owner, group, shared | dynamic << 1, clothGroup(owner)
    // contacts (current frame and previous frame)
    ManifoldGPU *manifolds, *prevManifolds;
    uint32_t *mapKeyA, *mapKeyB, *mapVal;
    // constraints
    JointGPU* joints;
    uint32_t* activeJoints;
    SpringGPU* springs;
    uint32_t* hardSprings;
    TetGPU* tets;
    // adjacency: static segments + per-frame contact segment
    uint4* staticSeg;
    uint32_t *preList, *postList;
    uint32_t *dynCount, *dynStart, *dynCursor, *dynList;
    uint32_t* dynSplit;                   // manifold entries at the head of each sorted dyn segment
    uint32_t* adjLongQueue;               // bodies with long contact segments this frame
    uint32_t* postTets;                   // tet entries at the head of each static post segment
    const TetGPU* tetInc;                 // tet records in postList order (null without tets)
    // coloring
    uint32_t *colorsA, *colorsB, *colorList, *bodySlot;
    uint32_t* colorLaunch;                // static palette: primal launch order per color
    // control
    Counters* counters;
    uint32_t* scanScratch;                // block sums of the exclusive scans
    float* diag;
    uint32_t *colorStart;                 // static palette or counters->colorStart
    float4 *initPenLin, *initPenAng;      // authored joint penalties (state resets)
    uint32_t* resetFlags;                 // body flags for set_body_states
    // kinematic drivers advanced at frame end
    uint32_t* spinnerBody;
    float4* spinnerAxisOmega;             // xyz axis, w omega
    uint32_t* rateJoint;
    float* rateValue;
    uint32_t numSpinners, numRateMotors;
    uint32_t* failureLatch;               // [0] kind, [1] frame, [2] detail
    uint32_t* frameCounter;
    // cloth: element topology (static)
    uint4* tris;                          // collision triangles (authored, then tet faces)
    uint2* edges;                         // unique edges, authored prefix first
    uint32_t *nbrStart, *nbrCount, *nbrList;   // sorted one-ring per vertex
    uint32_t *particleIdx, *selfCollision;
    MembraneGPU* membranes;
    BendGPU* bends;
    // cloth: per frame
    uint32_t *elemCellCount, *elemCellStart, *elemCursor, *elemCells;   // 2H buckets: triangles, edges
    float4* elemBox;                            // tight AABB per element (lo, hi)
    int4* elemRange;                            // binned cell range per element: first cell,
                                                // w = extents (x | y << 2 | z << 4, each 0..3)
    uint32_t *datOwnerCount, *datOwnerStart;    // pairs per query owner (particles, edges)
    uint4* datPairs;                            // (kind, owner, other, flags)
    uint2* datCache;                            // first pairs of each owner from the counting pass (other, flags)
    uint32_t *rtCount, *rtStart;                // rigid-triangle records per triangle
    uint2* rtCand;                              // (body, feature) of each record, RT_MAX_PER_TRI per triangle
    uint32_t *datEmit, *datEmitStart;           // element contacts per query owner
    SoftContactGPU *soft, *prevSoft;
    uint32_t *softKeyA, *softKeyB, *softVal;
    uint32_t* truncBits;                        // Planar-DAT step fraction per body (float bits)
    float4 *ogcPrev, *posNext, *angNext;
    uint32_t* bigScanScratch;
    // isotropic OGC (tet surfaces, mixed scenes): tracker topology (static),
    // tracked closest elements (this frame / previous frame), conservative
    // bounds (squared distances as float bits), the bound-exceeder count the
    // primal of this pass adds to
    uint4 *triAdj;
    uint32_t *nbr2Start, *nbr2Count, *nbr2List;
    uint32_t *vertEdgeStart, *vertEdgeCount, *vertEdgeList;
    uint32_t* clothVert;
    uint4 *vtTrack, *vtTrackPrev, *eeTrack, *eeTrackPrev;
    uint32_t* ogcBounds;
    uint32_t* ogcExceed;                        // one of counters->ogcSlots
    uint32_t* elemCellsTmp;                     // bucket contents before the per-bucket sort
    float4* ogcPartial;                         // per query owner: tracked set so far, its distances, own bound
    // learned warm start
    uint32_t* learnIdx;                         // dynamic particles the model predicts
    float *learnFeat, *learnPred, *learnTarget; // [n][32], [n][3], [n][3]
    float4 *learnSaveLin, *learnSaveAng;        // the plain warm start
    float4 *learnSweptLin, *learnSweptAng;      // pose buffers of the predicted trial branch
    uint32_t* learnSlot;                        // body -> index in learnIdx (or 0xFFFFFFFF)
    float4* learnStat;                          // per learned vertex: summed contact normal, contact count
    float *learnGap, *learnStiff, *learnRingN;  // closest contact gap; static stiffness sum and ring size
    uint32_t* learnRingStart;                   // 1-ring CSR over learned vertices: (slot, multiplicity)
    uint2* learnRing;
    float *learnPrm, *learnNorm, *learnResidBodies;
    float* learnResidBodies2;                   // per-body residual scratch of the predicted branch
    float4 *learnNextLin, *learnNextAng;        // pending solves of the predicted branch (color-Jacobi scenes)
    void* learnHalf;                            // BF16 weight image of the inference kernel (UMMA layout)
    double* learnResid;                         // [0] plain, [1] predicted, [2] scratch
    double* learnTrace;                         // residual trace of the last frame
    uint32_t* learnAccepted;                    // frames whose prediction was kept (running)
};

struct Sizes {
    uint32_t numBodies, numColliders, numActiveJoints, numHardSprings, numTets;
    uint32_t maxPairs, producers, numDynamicBodies;
    uint32_t scanScratchWords;
    bool dynamicColoring;
    bool particleFastPath;   // every dynamic body a particle with only tet/contact entries
    // cloth
    uint32_t numTris, numParticles, numEdges, numMembranes, numBends;
    uint32_t maxDatPairs, maxSoft, elemHashSize;
    uint32_t numLearn;        // learned rows in use (particles, plus rigid bodies with learnRigid)
    uint32_t numLearnAll;     // learned rows allocated: every dynamic particle and rigid body
    uint32_t numDynamicRigid;
    uint32_t numHeavyProducers;
    // static palette on the host (null with dynamic coloring)
    const uint32_t* colorCounts;
    const uint32_t* colorLanes;
    const uint32_t* colorLean;            // lean particles at the head of each color's launch order
    const uint32_t* colorStartHost;       // static palette: each color's start in the list
    // dynamic coloring: block shape of the rigid primal's grid-stride launch
    // (blocks, threads per block), chosen by the runtime's autotuner
    uint32_t dynBlocks, dynThreads;
};

// exclusive scan of n words (n <= 1024 * 1024); out may not alias in
void launch_exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* scratch,
                           cudaStream_t st);

void launch_broadphase(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);
void launch_narrowphase(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);
void launch_map_rebuild(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);
void launch_warmstart(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);
void launch_adjacency(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);
void launch_dynamic_coloring(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);
// one color of the block-descent primal; `count` is the color's body count
// when known on the host (static palette), else 0xFFFFFFFF (read on device);
// `lanes` is 8, 16 or 32 lanes per body (grouped kernel) or
// AVBD_PRIMAL_STAGED (staged kernel: block-wide term evaluation, then an
// 8-lane fold per body), every choice computing the same floats
// With a side stream and two events, the color's non-lean bodies (a block
// each) run on the side stream beside the lean particles (a fork and a join
// on `st`; in a captured frame, two parallel graph branches).
constexpr uint32_t NO_HOST_START = 0xFFFFFFFFu;   // a color start the kernel reads on the device
constexpr uint32_t AVBD_PRIMAL_STAGED = 1;
void launch_primal_color(const Params& P, const DevPtrs& d, const Sizes& z, uint32_t color,
                         uint32_t count, uint32_t lanes, cudaStream_t st, cudaStream_t side = nullptr,
                         cudaEvent_t fork = nullptr, cudaEvent_t join = nullptr);
// squared AL-gradient norm of every dynamic body (perBody[numDynamicBodies])
// and their fixed-order sum (total)
void launch_residual(const Params& P, const DevPtrs& d, const Sizes& z, float* perBody, double* total,
                     cudaStream_t st);
// dynamic coloring: colors [first, 64) in one block, after the per-color launches
void launch_primal_tail(const Params& P, const DevPtrs& d, const Sizes& z, uint32_t first, cudaStream_t st);
// every iteration of a small scene in one thread block
void launch_solve_small(const Params& P, const DevPtrs& d, const Sizes& z, uint32_t colorBound,
                        cudaStream_t st);
void launch_dual(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);
void launch_finalize(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);
void launch_max_constraint_error(const Params& P, const DevPtrs& d, const Sizes& z,
                                 cudaStream_t st);
void launch_reset_bodies(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);

// ---- headless render and observation compute (render.cu)
// SkinBindingGPU (layout of avbd_skin_binding)
struct SkinBinding { uint4 ids; float4 weights, restNormal, inv0, inv1, inv2; };
// one Push-T environment with the goal heading's cos/sin
struct PushTDev { uint4 ids; float4 frame; float goalYaw, halfWin, goalCos, goalSin; };
static_assert(sizeof(SkinBinding) == 96, "SkinBinding layout");
static_assert(sizeof(PushTDev) == 48, "PushTDev layout");
// out: 24 floats per instance (avbd_render_instance)
void launch_build_instances(const DevPtrs& d, const uint32_t* ids, const float4* colors, uint32_t n,
                            uint32_t colorMode, float* out, cudaStream_t st);
void launch_soft_normals(const DevPtrs& d, uint32_t numTris, const uint32_t* surfVerts, const uint32_t* vtStart,
                         const uint32_t* vtCount, const uint32_t* vtList, uint32_t numSurf, float4* faceN,
                         float clothScale, float4* out, cudaStream_t st);
void launch_skin_deform(const float4* posLin, const SkinBinding* b, uint32_t n, float4* out, cudaStream_t st);
// shapes: 6 float4 of scratch per environment
void launch_pusht_obs(const float4* posLin, const float4* posAng, const PushTDev* envs, uint32_t numEnvs,
                      uint32_t res, float4* shapes, uint8_t* out, cudaStream_t st);
// spinners and legacy rate motors, then the end-of-frame failure check
void launch_frame_end(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);

// exclusive scan of any n < 2^30 words; scratch holds n/1024 + n/1024^2 + 64 words
void launch_exclusive_scan_large(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* scratch,
                                 cudaStream_t st);
size_t scan_large_scratch_words(uint32_t n);

// cloth element pipeline (cloth.cu)
// step-start detection: element grid, pair stream, rigid-triangle contacts
void launch_cloth_detect(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);
// after the predictor: predictor truncation, accepted-pose pair stream,
// element contacts, soft map, re-anchor
void launch_cloth_accept(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);
// per-color Planar-DAT pass that also publishes the color's solve
void launch_dat_color(const Params& P, const DevPtrs& d, const Sizes& z, uint32_t color, uint32_t count,
                      cudaStream_t st);
void launch_cloth_restore(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);
// rigid-feature-vs-triangle records at the head of the soft list
void launch_rt_emit(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);
// soft totals over `owners` query owners, then the soft persistence map
void launch_soft_map(const Params& P, const DevPtrs& d, const Sizes& z, uint32_t owners, cudaStream_t st);
// isotropic OGC: element grid, V-T / E-E trackers and bounds, rigid-triangle
// and element contact records, soft map (once per frame, before warm start)
void launch_ogc_detect(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);
// publish one color's solve (posNext -> posLin) in color-Jacobi scenes
// `start`: the color's start in the color list when known on the host
// (static palette), else NO_HOST_START (read on the device)
void launch_publish_color(const Params& P, const DevPtrs& d, uint32_t color, uint32_t count, uint32_t start,
                          cudaStream_t st);
// mid-solve OGC bound refresh when more than 1% of surface vertices hit their
// bound in the pass counted by `readSlot`; zeroes `zeroSlot` for the next pass
void launch_ogc_refresh(const Params& P, const DevPtrs& d, const Sizes& z, uint32_t* readSlot, uint32_t* zeroSlot,
                        cudaStream_t st);
void launch_cloth_smoothing(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);

// learned warm start (learned.cu)
void launch_learn_features(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);
void launch_learn_apply(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);
void launch_learn_select(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);
void launch_learn_branch(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);
void launch_learn_adopt(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);
void launch_learn_target(const Params& P, const DevPtrs& d, const Sizes& z, cudaStream_t st);
void launch_copy_double(const double* src, double* dst, cudaStream_t st);
void launch_mlp_infer(const void* halfW, const float* prm, const float* norm, const float* X, uint32_t n, float* Y,
                      uint32_t* status, cudaStream_t st);
void launch_mlp_mirror(const float* prm, void* halfW, cudaStream_t st);
uint32_t mlp_param_count();
uint32_t mlp_half_count();
uint32_t mlp_norm_count();

}  // namespace avbd
