// ref_pin.cpp — runs the reference's own solver kernels beside the oracle.
//
// TEST INFRASTRUCTURE, NOT PRODUCT CODE.  Built only where the reference's
// sources are present (oracle/_ref/build.sh): the shader files
// Sources/PhysicsAVBD/Shaders/*.metal are compiled, unchanged and where they
// lie, as C++ through the Metal stand-in header msl/metal_stdlib, inside
// namespace `ref`.  Nothing of them is copied into this repository.
//
// The oracle (avbd_oracle.cpp) calls a stage observer before and after every
// stage of a frame.  For each observed stage this file snapshots the stage's
// inputs, lets the oracle run its restatement, then runs the reference's
// kernel for the same stage on the snapshot — one kernel invocation per grid
// thread, in thread order — and compares the two outputs word for word.  The
// oracle's result then carries the frame on, so every frame of a scene is a
// fresh per-stage comparison on real data (no divergence builds up).
//
// Kernels that exchange values between SIMD lanes (simd_shuffle_xor in the
// 8-lane split primal, 40_solver.metal:1544-1686) run their lanes as
// cooperative contexts (ucontext): every lane runs to its next shuffle, the
// values are exchanged, and all lanes go on — the lockstep a SIMD group has.
//
// Stages and kernels:
//   warm start   warmstart_joints, warmstart_bodies   (40_solver.metal:546-724)
//   primal       primal_particles_split, per color     (40_solver.metal:1544-1686)
//   dual         dual_all                             (40_solver.metal:1850-1906)
//   finalize     finalize_velocities                  (40_solver.metal:2108-2150)
//   narrowphase  np_collide                           (30_narrowphase.metal:337-1322)
//   map          pm_clear + pm_insert                 (20_broadphase.metal:555-593)
//   adjacency    adj_clear_degrees, adj_count, adj_copy_cursor, adj_scatter,
//                adj_sort                             (40_solver.metal:18-248)
//   diagnostics  diag_error                           (40_solver.metal:2189-2229)
#include <ucontext.h>

#include <functional>
#include <memory>

#include "oracle_solver.h"

// after every system header: the stand-in defines the Metal address-space
// qualifiers as empty macros
#include <metal_stdlib>

namespace ref {
#include "00_common.metal"
#include "10_scan.metal"
#include "20_broadphase.metal"
#include "25_cloth.metal"
#include "27_planar_dat.metal"
#include "30_narrowphase.metal"
#include "40_solver.metal"
}  // namespace ref

thread_local msl_shim::LaneHooks msl_shim::tl_lanes{};
void msl_shim::unsupported(const char* what) {
    std::fprintf(stderr, "ref_pin: unsupported Metal construct: %s\n", what);
    std::abort();
}

static_assert(sizeof(ref::JointGPU) == sizeof(oracle::JointGPU), "JointGPU");
static_assert(sizeof(ref::SpringGPU) == sizeof(oracle::SpringGPU), "SpringGPU");
static_assert(sizeof(ref::TetGPU) == sizeof(oracle::TetGPU), "TetGPU");
static_assert(sizeof(ref::ManifoldGPU) == sizeof(oracle::ManifoldGPU), "ManifoldGPU");
static_assert(sizeof(ref::SoftContactGPU) == sizeof(oracle::SoftContactGPU), "SoftContactGPU");
static_assert(sizeof(ref::MembraneGPU) == sizeof(oracle::MembraneGPU), "MembraneGPU");
static_assert(sizeof(ref::BendGPU) == sizeof(oracle::BendGPU), "BendGPU");
static_assert(sizeof(float4) == 16 && sizeof(uint2) == 8 && sizeof(float2) == 8, "vector sizes");

namespace {

using oracle::Solver;

// ---------------------------------------------------------------------------
// Lanes of one SIMD group as cooperative contexts.
// ---------------------------------------------------------------------------
struct LaneGroup {
    static constexpr int kMaxLanes = 32;
    static constexpr size_t kStack = 256 * 1024;
    ucontext_t sched{}, lane[kMaxLanes]{};
    std::unique_ptr<char[]> stacks[kMaxLanes];
    bool done[kMaxLanes] = {};
    unsigned phase[kMaxLanes] = {};
    alignas(16) unsigned char slot[2][kMaxLanes][64];
    std::function<void(uint32_t)> body;
    int cur = -1;

    static thread_local LaneGroup* active;

    static void entry() {
        LaneGroup* g = active;
        const int l = g->cur;
        g->body((uint32_t)l);
        g->done[l] = true;       // returning resumes `sched` (uc_link)
    }
    static void exchange_hook(void* ctx, const void* mine, void* partner, unsigned bytes, unsigned mask) {
        static_cast<LaneGroup*>(ctx)->exchange(mine, partner, bytes, mask);
    }
    static void barrier_hook(void* ctx) {
        static_cast<LaneGroup*>(ctx)->exchange(nullptr, nullptr, 0, 0);
    }
    void exchange(const void* mine, void* partner, unsigned bytes, unsigned mask) {
        const int l = cur;
        const unsigned p = phase[l] & 1u;
        if (bytes > sizeof(slot[0][0])) msl_shim::unsupported("shuffle of more than 64 bytes");
        if (bytes) std::memcpy(slot[p][l], mine, bytes);
        phase[l]++;
        swapcontext(&lane[l], &sched);             // every live lane reaches this phase first
        if (bytes) std::memcpy(partner, slot[p][(unsigned)l ^ mask], bytes);
    }
    // Runs body(lane) for lanes 0..n-1 in lockstep between shuffles.
    void run(int n, std::function<void(uint32_t)> f) {
        body = std::move(f);
        active = this;
        msl_shim::LaneHooks saved = msl_shim::tl_lanes;
        msl_shim::tl_lanes = msl_shim::LaneHooks{&exchange_hook, &barrier_hook, this};
        for (int l = 0; l < n; l++) {
            if (!stacks[l]) stacks[l].reset(new char[kStack]);
            getcontext(&lane[l]);
            lane[l].uc_stack.ss_sp = stacks[l].get();
            lane[l].uc_stack.ss_size = kStack;
            lane[l].uc_link = &sched;
            makecontext(&lane[l], &LaneGroup::entry, 0);
            done[l] = false;
            phase[l] = 0;
        }
        bool live = true;
        while (live) {
            live = false;
            for (int l = 0; l < n; l++) {
                if (done[l]) continue;
                cur = l;
                swapcontext(&sched, &lane[l]);
                live = live || !done[l];
            }
        }
        msl_shim::tl_lanes = saved;
    }
};
thread_local LaneGroup* LaneGroup::active = nullptr;

// ---------------------------------------------------------------------------
// Comparison records
// ---------------------------------------------------------------------------
struct StageStats {
    double calls = 0, compared = 0, mismatched = 0, maxRel = 0;
    long long firstBadFrame = -1;
    long long firstBadIndex = -1;
};

static float as_f(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

struct Pin {
    Solver* S = nullptr;
    StageStats st[Solver::ST_COUNT_ + 1];   // last slot: diagnostics
    uint32_t primalEvery = 1;               // check the primal on every k-th iteration
    uint32_t iteration = 0;
    LaneGroup lanes;
    ref::SimParams P{};
    std::vector<uint32_t> counters;
    // snapshots
    std::vector<oracle::F4> posLin, posAng, initLin, initAng, inertLin, inertAng, velLin, velAng, prevVelLin,
        ogcPrev;
    std::vector<uint32_t> bounds;
    std::vector<oracle::JointGPU> joints;
    std::vector<oracle::SpringGPU> springs;
    std::vector<oracle::ManifoldGPU> manifolds;
    std::vector<oracle::SoftContactGPU> soft;
    bool primalActive = false;
    int dumps = 0;
    int perturbStage = -1;     // self-check: flip one input bit of this stage's reference run

    // Compare two arrays of 32-bit words record by record (words per record).
    void compare_words(int stage, const void* got, const void* want, size_t records, size_t words,
                       bool floats = true) {
        StageStats& s = st[stage];
        const uint32_t* a = static_cast<const uint32_t*>(got);
        const uint32_t* b = static_cast<const uint32_t*>(want);
        for (size_t r = 0; r < records; r++) {
            s.compared += 1;
            bool bad = false;
            for (size_t w = 0; w < words; w++) {
                const uint32_t x = a[r * words + w], y = b[r * words + w];
                if (x == y) continue;
                bad = true;
                if (floats) {
                    const double fx = as_f(x), fy = as_f(y);
                    const double rel = std::fabs(fx - fy) / std::max(1.0, std::fabs(fy));
                    s.maxRel = std::max(s.maxRel, std::isfinite(rel) ? rel : 1e30);
                } else {
                    s.maxRel = 1e30;
                }
            }
            if (bad) {
                s.mismatched += 1;
                if (s.firstBadFrame < 0) { s.firstBadFrame = (long long)S->frameIndex; s.firstBadIndex = (long long)r; }
            }
        }
    }

    // ref::SimParams from the oracle's state (GPUSolver.swift:2097-2150 syncParams)
    void sync_params() {
        const oracle::Params& Q = S->P;
        ref::SimParams p{};
        p.dt = Q.dt; p.gravity = Q.gravity; p.alpha = Q.alpha; p.betaLin = Q.betaLin; p.betaAng = Q.betaAng;
        p.gamma = Q.gamma; p.numBodies = Q.numBodies; p.numJoints = Q.numJoints; p.numSprings = Q.numSprings;
        p.mapCapacity = Q.mapCapacity; p.maxManifolds = Q.maxPairs; p.maxPairs = Q.maxPairs;
        p.cellSize = Q.cellSize; p.gridHashSize = Q.gridHashSize; p.numHashed = Q.numHashed;
        p.numGlobals = Q.numGlobals; p.maxSpeed = Q.maxSpeed; p.lambdaMax = Q.lambdaMax;
        p.iterations = Q.iterations; p.numTets = Q.numTets; p.numTris = Q.numTris; p.numEdges = S->numEdges;
        p.numParticles = Q.numParticles; p.maxSoft = S->maxSoft; p.softMapCapacity = S->softMapCapacity;
        p.numMembranes = (uint32_t)S->membranes.size(); p.numBends = (uint32_t)S->bends.size();
        p.elemCellSize = S->elemCellSize; p.elemHashSize = S->elemHashSize; p.rodDecayPow = Q.rodDecayPow;
        p.particleDamping = Q.particleDamping; p.numHashedRigid = Q.numHashedRigid; p.elemMargin = S->elemMargin;
        p.frame = Q.frame; p.frictionCombineMode = Q.frictionCombineMode; p.collisionMargin = Q.collisionMargin;
        p.rigidLinearDamping = Q.rigidLinearDamping; p.rigidAngularDamping = Q.rigidAngularDamping;
        p.surfaceTruncationMode = Q.surfaceTruncationMode; p.maxPlanarDATPairs = S->maxDatPairs;
        p.numSurfaceContactEdges = S->numSurfaceEdges; p.planarDATQueryRadius = S->queryRadius;
        p.planarDATRelaxation = Q.planarDATRelaxation; p.surfaceContactCellSize = S->surfaceCellSize;
        p.tetInversionPreventionEnabled = Q.tetInversionPreventionEnabled;
        P = p;
        counters.assign(CTR_TOTAL, 0u);
        counters[CTR_PAIRS] = S->numPairs;
        counters[CTR_SOFT] = S->numSoft;
    }

    template <class T> static T* cast(std::vector<oracle::F4>& v) { return reinterpret_cast<T*>(v.data()); }
    template <class T> static const T* ccast(const std::vector<oracle::F4>& v) {
        return reinterpret_cast<const T*>(v.data());
    }
    ::atomic_uint* ctr() { return reinterpret_cast<::atomic_uint*>(counters.data()); }

    void snap_bodies() {
        posLin = S->posLin; posAng = S->posAng; initLin = S->initLin; initAng = S->initAng;
        inertLin = S->inertLin; inertAng = S->inertAng; velLin = S->velLin; velAng = S->velAng;
        prevVelLin = S->prevVelLin; ogcPrev = S->ogcPrev; bounds = S->boundsBits;
    }

    // ---------------------------------------------------------------- stages
    void warm_joints(bool after) {
        if (!after) { snap_bodies(); joints = S->joints; springs = S->springs; return; }
        sync_params();
        const uint32_t n = (uint32_t)(joints.size() + springs.size());
        for (uint32_t gid = 0; gid < n; gid++)
            ref::warmstart_joints(cast<float4>(posLin), cast<float4>(posAng),
                                  reinterpret_cast<ref::JointGPU*>(joints.data()), P,
                                  reinterpret_cast<ref::SpringGPU*>(springs.data()), cast<float4>(velLin),
                                  cast<float4>(velAng), gid);
        st[Solver::ST_WARM_JOINTS].calls += 1;
        compare_words(Solver::ST_WARM_JOINTS, joints.data(), S->joints.data(), joints.size(), 56);
        compare_words(Solver::ST_WARM_JOINTS, springs.data(), S->springs.data(), springs.size(), 16);
    }

    void warm_bodies(bool after) {
        if (!after) { snap_bodies(); return; }
        sync_params();
        uint32_t mode = P.surfaceTruncationMode;
        std::vector<oracle::F4> shape = S->shape;
        for (uint32_t gid = 0; gid < S->nb; gid++)
            ref::warmstart_bodies(cast<float4>(posLin), cast<float4>(posAng), cast<float4>(initLin),
                                  cast<float4>(initAng), cast<float4>(inertLin), cast<float4>(inertAng),
                                  cast<float4>(velLin), cast<float4>(velAng), cast<float4>(prevVelLin), P,
                                  cast<float4>(ogcPrev), bounds.data(), mode, cast<float4>(shape),
                                  S->gravityScale.data(), gid);
        st[Solver::ST_WARM_BODIES].calls += 1;
        const int k = Solver::ST_WARM_BODIES;
        compare_words(k, posLin.data(), S->posLin.data(), S->nb, 4);
        compare_words(k, posAng.data(), S->posAng.data(), S->nb, 4);
        compare_words(k, initLin.data(), S->initLin.data(), S->nb, 4);
        compare_words(k, initAng.data(), S->initAng.data(), S->nb, 4);
        compare_words(k, inertLin.data(), S->inertLin.data(), S->nb, 4);
        compare_words(k, inertAng.data(), S->inertAng.data(), S->nb, 4);
    }

    // The split primal of one color (8 lanes per body).  Each body's group
    // runs on the pre-color pose (its result is recorded and the pose put
    // back), which is the color-Jacobi reading the oracle and the CUDA path
    // use; where a color has no same-color coupling it equals the in-place
    // sweep.
    void primal(int color, bool after) {
        if (!after) {
            primalActive = (iteration % primalEvery) == 0;
            if (primalActive) snap_bodies();
            return;
        }
        if (!primalActive) return;
        sync_params();
        const uint32_t s0 = S->colorStart[color], e0 = S->colorStart[color + 1];
        if (s0 == e0) return;
        std::vector<uint32_t> ctrs = counters;
        if (perturbStage == Solver::ST_PRIMAL) inertLin[S->colorList[s0]].x += 1e-3f;
        std::vector<oracle::F4> outLin(e0 - s0), outAng(e0 - s0);
        uint32_t colorIndex = (uint32_t)color;
        std::vector<oracle::F4> props = S->props, shape = S->shape;
        for (uint32_t slot = 0; slot < e0 - s0; slot++) {
            const uint32_t body = S->colorList[s0 + slot];
            const oracle::F4 keepLin = posLin[body], keepAng = posAng[body];
            lanes.run(8, [&](uint32_t lane) {
                ref::primal_particles_split(
                    cast<float4>(posLin), cast<float4>(posAng), ccast<float4>(initLin), ccast<float4>(initAng),
                    ccast<float4>(inertLin), ccast<float4>(inertAng), ccast<float4>(props),
                    reinterpret_cast<const ref::JointGPU*>(S->joints.data()),
                    reinterpret_cast<const ref::SpringGPU*>(S->springs.data()),
                    reinterpret_cast<const ref::ManifoldGPU*>(S->manifolds.data()), S->adjStart.data(),
                    S->adjCount.data(), S->adjList.data(), S->colorList.data(), S->colorStart.data(), colorIndex, P,
                    ccast<float4>(shape), reinterpret_cast<const ref::TetGPU*>(S->tets.data()),
                    reinterpret_cast<const ref::SoftContactGPU*>(S->soft.data()),
                    reinterpret_cast<const ref::MembraneGPU*>(S->membranes.data()),
                    reinterpret_cast<const ref::BendGPU*>(S->bends.data()), S->boundsBits.data(),
                    ccast<float4>(S->ogcPrev), reinterpret_cast<::atomic_uint*>(ctrs.data()), slot * 8u + lane);
            });
            outLin[slot] = posLin[body];
            outAng[slot] = posAng[body];
            posLin[body] = keepLin;
            posAng[body] = keepAng;
        }
        std::vector<oracle::F4> wantLin(e0 - s0), wantAng(e0 - s0);
        for (uint32_t slot = 0; slot < e0 - s0; slot++) {
            const uint32_t body = S->colorList[s0 + slot];
            wantLin[slot] = S->colorJacobi ? S->posNext[body] : S->posLin[body];
            wantAng[slot] = S->colorJacobi ? S->angNext[body] : S->posAng[body];
        }
        st[Solver::ST_PRIMAL].calls += 1;
        compare_words(Solver::ST_PRIMAL, outLin.data(), wantLin.data(), e0 - s0, 4);
        compare_words(Solver::ST_PRIMAL, outAng.data(), wantAng.data(), e0 - s0, 4);
    }

    void dual(bool after) {
        if (!after) {
            joints = S->joints; springs = S->springs;
            manifolds.assign(S->manifolds.begin(), S->manifolds.begin() + S->numPairs);
            soft.assign(S->soft.begin(), S->soft.begin() + std::min<size_t>(S->numSoft, S->soft.size()));
            return;
        }
        sync_params();
        manifolds.resize(std::max<size_t>(manifolds.size(), 1));
        soft.resize(std::max<size_t>(soft.size(), 1));
        const uint32_t n = (uint32_t)(S->joints.size() + S->springs.size()) + S->numPairs + S->numSoft;
        if (perturbStage == Solver::ST_DUAL && S->numPairs) manifolds[0].contacts[0].lambda.x += 1.0f;
        for (uint32_t gid = 0; gid < n; gid++)
            ref::dual_all(ccast<float4>(S->posLin), ccast<float4>(S->posAng), ccast<float4>(S->initLin),
                          ccast<float4>(S->initAng), reinterpret_cast<ref::JointGPU*>(joints.data()),
                          reinterpret_cast<ref::ManifoldGPU*>(manifolds.data()), ctr(), P,
                          reinterpret_cast<ref::SpringGPU*>(springs.data()),
                          reinterpret_cast<ref::SoftContactGPU*>(soft.data()), gid);
        const int k = Solver::ST_DUAL;
        st[k].calls += 1;
        compare_words(k, joints.data(), S->joints.data(), joints.size(), 56);
        compare_words(k, springs.data(), S->springs.data(), springs.size(), 16);
        compare_words(k, manifolds.data(), S->manifolds.data(), S->numPairs, 176);
        compare_words(k, soft.data(), S->soft.data(), S->numSoft, 28);
        iteration++;
    }

    void finalize(bool after) {
        if (!after) { snap_bodies(); return; }
        sync_params();
        std::vector<oracle::F4> shape = S->shape;
        for (uint32_t gid = 0; gid < S->nb; gid++)
            ref::finalize_velocities(ccast<float4>(S->posLin), ccast<float4>(S->posAng), ccast<float4>(S->initLin),
                                     ccast<float4>(S->initAng), cast<float4>(velLin), cast<float4>(velAng),
                                     cast<float4>(prevVelLin), P, ccast<float4>(shape), S->gravityScale.data(), gid);
        const int k = Solver::ST_FINALIZE;
        st[k].calls += 1;
        compare_words(k, velLin.data(), S->velLin.data(), S->nb, 4);
        compare_words(k, velAng.data(), S->velAng.data(), S->nb, 4);
        compare_words(k, prevVelLin.data(), S->prevVelLin.data(), S->nb, 4);
    }

    // Narrowphase: this frame's manifolds from the candidate pairs, warm
    // started from the previous frame's through the persistence map.
    void narrow(bool after) {
        if (!after) return;
        sync_params();
        const uint32_t nc = S->nc;
        std::vector<uint32_t> hullRange(2 * std::max<uint32_t>(nc, 1));
        for (uint32_t c = 0; c < nc; c++) {
            hullRange[2 * c] = S->colHullFirst.empty() ? 0u : S->colHullFirst[c];
            hullRange[2 * c + 1] = S->colHullCount.empty() ? 0u : S->colHullCount[c];
        }
        std::vector<float> hull(4 * std::max<size_t>(S->hullVerts.size(), 1), 0.0f);
        for (size_t i = 0; i < S->hullVerts.size(); i++) {
            hull[4 * i] = S->hullVerts[i].x; hull[4 * i + 1] = S->hullVerts[i].y; hull[4 * i + 2] = S->hullVerts[i].z;
        }
        std::vector<float> fric(2 * std::max<uint32_t>(nc, 1));
        for (uint32_t c = 0; c < nc; c++) { fric[2 * c] = S->colFrictionS[c]; fric[2 * c + 1] = S->colFrictionD[c]; }
        std::vector<oracle::ManifoldGPU> out(std::max<uint32_t>(S->numPairs, 1));
        std::memset(out.data(), 0, out.size() * sizeof(oracle::ManifoldGPU));
        std::vector<oracle::F4> colShape = S->colShape, props = S->props, spin = S->spinVel, lp = S->colLocalPos,
                                lr = S->colLocalRot;
        for (uint32_t gid = 0; gid < S->numPairs; gid++)
            ref::np_collide(ccast<float4>(S->posLin), ccast<float4>(S->posAng), ccast<float4>(colShape),
                            ccast<float4>(props), reinterpret_cast<const uint2*>(S->pairs.data()), ctr(),
                            reinterpret_cast<ref::ManifoldGPU*>(out.data()),
                            reinterpret_cast<const ref::ManifoldGPU*>(S->prevManifolds.data()),
                            reinterpret_cast<const ::atomic_uint*>(S->mapKeyA.data()), S->mapKeyB.data(),
                            S->mapVal.data(), P, S->colShapeType.data(), ccast<float4>(spin),
                            ccast<float4>(S->velLin), ccast<float4>(S->velAng), S->colOwner.data(), ccast<float4>(lp),
                            ccast<float4>(lr), reinterpret_cast<const uint2*>(hullRange.data()),
                            reinterpret_cast<const float4*>(hull.data()), reinterpret_cast<const float2*>(fric.data()),
                            gid);
        const int k = Solver::ST_NARROWPHASE;
        st[k].calls += 1;
        // the active part of every manifold: header, pair, basis, contacts
        for (uint32_t m = 0; m < S->numPairs; m++) {
            // a pair without contacts writes only its header and collider
            // pair (the reference leaves the rest of the record as it was)
            const uint32_t cnt = std::max(S->manifolds[m].header.z, out[m].header.z);
            const size_t words = cnt == 0 ? 8 : 16 + 20 * (size_t)std::min<uint32_t>(cnt, 8u);
            const double before = st[k].mismatched;
            compare_words(k, &out[m], &S->manifolds[m], 1, words);
            if (st[k].mismatched > before && std::getenv("REF_PIN_DUMP") && dumps++ < 3) {
                const uint32_t* a = reinterpret_cast<const uint32_t*>(&out[m]);
                const uint32_t* b = reinterpret_cast<const uint32_t*>(&S->manifolds[m]);
                std::fprintf(stderr, "frame %llu manifold %u (colliders %u %u):\n", (unsigned long long)S->frameIndex, m,
                             S->manifolds[m].colliderPair.x, S->manifolds[m].colliderPair.y);
                for (size_t w = 0; w < words; w++)
                    if (a[w] != b[w])
                        std::fprintf(stderr, "  word %zu: ref %08x (%g) oracle %08x (%g)\n", w, a[w], as_f(a[w]), b[w],
                                     as_f(b[w]));
            }
        }
    }

    // Persistence map: the same key -> manifold set (slot placement depends
    // on insertion order).
    void map(bool after) {
        if (!after) return;
        sync_params();
        std::vector<uint32_t> ka(S->mapCapacity), kb(S->mapCapacity), kv(S->mapCapacity);
        uint32_t cap = S->mapCapacity;
        for (uint32_t gid = 0; gid < cap; gid++)
            ref::pm_clear(reinterpret_cast<::atomic_uint*>(ka.data()), cap, gid);
        for (uint32_t gid = 0; gid < S->numPairs; gid++)
            ref::pm_insert(reinterpret_cast<const ref::ManifoldGPU*>(S->manifolds.data()),
                           reinterpret_cast<::atomic_uint*>(ka.data()), kb.data(), kv.data(), ctr(), P, gid);
        std::map<std::pair<uint32_t, uint32_t>, uint32_t> a, b;
        for (uint32_t i = 0; i < cap; i++) {
            if (ka[i]) a[{ka[i], kb[i]}] = kv[i];
            if (S->mapKeyA[i]) b[{S->mapKeyA[i], S->mapKeyB[i]}] = S->mapVal[i];
        }
        const int k = Solver::ST_MAP;
        st[k].calls += 1;
        st[k].compared += 1;
        if (a != b) {
            st[k].mismatched += 1;
            st[k].maxRel = 1e30;
            if (st[k].firstBadFrame < 0) st[k].firstBadFrame = (long long)S->frameIndex;
        }
    }

    // Adjacency: per body, the sorted list of (kind << 28 | index) entries.
    void adjacency(bool after) {
        if (!after) return;
        sync_params();
        uint32_t nb = S->nb;
        std::vector<uint32_t> deg(nb), start(nb), cursor(nb);
        auto* degA = reinterpret_cast<::atomic_uint*>(deg.data());
        for (uint32_t g = 0; g < nb; g++) ref::adj_clear_degrees(degA, nb, g);
        const uint32_t total = P.numJoints + P.numSprings + S->numPairs + P.numTets + S->numSoft + P.numMembranes +
                               P.numBends;
        auto* J = reinterpret_cast<const ref::JointGPU*>(S->joints.data());
        auto* Sp = reinterpret_cast<const ref::SpringGPU*>(S->springs.data());
        auto* M = reinterpret_cast<const ref::ManifoldGPU*>(S->manifolds.data());
        auto* T = reinterpret_cast<const ref::TetGPU*>(S->tets.data());
        auto* Sc = reinterpret_cast<const ref::SoftContactGPU*>(S->soft.data());
        auto* Mb = reinterpret_cast<const ref::MembraneGPU*>(S->membranes.data());
        auto* B = reinterpret_cast<const ref::BendGPU*>(S->bends.data());
        for (uint32_t g = 0; g < total; g++)
            ref::adj_count(ccast<float4>(S->posLin), J, Sp, M, degA, ctr(), P, T, Sc, Mb, B, g);
        uint32_t run = 0;
        for (uint32_t i = 0; i < nb; i++) { start[i] = run; run += deg[i]; }
        std::vector<uint32_t> list(std::max<uint32_t>(run, 1));
        auto* curA = reinterpret_cast<::atomic_uint*>(cursor.data());
        for (uint32_t g = 0; g < nb; g++) ref::adj_copy_cursor(start.data(), curA, nb, g);
        for (uint32_t g = 0; g < total; g++)
            ref::adj_scatter(ccast<float4>(S->posLin), J, Sp, M, curA, list.data(), ctr(), P, T, Sc, Mb, B, g);
        for (uint32_t g = 0; g < nb; g++)
            ref::adj_sort(start.data(), deg.data(), list.data(), nb, g);
        const int k = Solver::ST_ADJACENCY;
        st[k].calls += 1;
        for (uint32_t b = 0; b < nb; b++) {
            st[k].compared += 1;
            bool same = deg[b] == S->adjCount[b];
            for (uint32_t i = 0; same && i < deg[b]; i++)
                same = list[start[b] + i] == S->adjList[S->adjStart[b] + i];
            if (!same) {
                st[k].mismatched += 1;
                st[k].maxRel = 1e30;
                if (st[k].firstBadFrame < 0) { st[k].firstBadFrame = (long long)S->frameIndex; st[k].firstBadIndex = b; }
            }
        }
    }

    // Broadphase: counting-sort hash grid, then candidate pairs in producer
    // order (count, exclusive scan, emit) from the frame-start pose.
    void broadphase(bool after) {
        if (!after) return;
        sync_params();
        const uint32_t H = S->gridHashSize, nh = P.numHashed, producers = P.numHashed + P.numGlobals;
        std::vector<uint32_t> cellCount(H, 0u), cellStart(H), cellRigid(H, 0u), cellBodies(std::max(nh, 1u));
        std::vector<uint32_t> slot(2 * std::max(nh, 1u));
        std::vector<uint32_t> clothGroup = S->clothGroup;
        clothGroup.resize(std::max<size_t>(clothGroup.size(), S->nb), 0u);
        std::vector<oracle::F4> colShape = S->colShape, lp = S->colLocalPos;
        for (uint32_t g = 0; g < nh; g++)
            ref::bp_count(ccast<float4>(S->posLin), S->hashedIdx.data(), reinterpret_cast<::atomic_uint*>(cellCount.data()),
                          reinterpret_cast<uint2*>(slot.data()), P, ccast<float4>(colShape), cellRigid.data(),
                          S->colOwner.data(), ccast<float4>(lp), ccast<float4>(S->posAng), S->colGroup.data(), g);
        uint32_t run = 0;
        for (uint32_t i = 0; i < H; i++) { cellStart[i] = run; run += cellCount[i]; }
        for (uint32_t g = 0; g < nh; g++)
            ref::bp_scatter(S->hashedIdx.data(), reinterpret_cast<const uint2*>(slot.data()), cellStart.data(),
                            cellBodies.data(), P, g);
        uint32_t hs = H;
        for (uint32_t g = 0; g < H; g++) ref::bp_sort_cells(cellStart.data(), cellCount.data(), cellBodies.data(), hs, g);
        const int k = Solver::ST_BROADPHASE;
        st[k].calls += 1;
        compare_words(k, cellCount.data(), S->cellCount.data(), H, 1, false);
        compare_words(k, cellStart.data(), S->cellStart.data(), H, 1, false);
        compare_words(k, cellBodies.data(), S->cellBodies.data(), nh, 1, false);
        if (producers == 0) return;
        std::vector<uint32_t> excl = S->exclusions;
        if (excl.empty()) excl.assign(2, 0u);
        uint32_t nExcl = (uint32_t)(S->exclusions.size() / 2);
        std::vector<uint32_t> pairCount(producers), pairStart(producers);
        std::vector<uint32_t> pairs(2 * (size_t)std::max(S->maxPairs, 1u));
        for (uint32_t g = 0; g < producers; g++)
            ref::bp_count_pairs_deterministic(
                ccast<float4>(S->posLin), ccast<float4>(colShape), S->hashedIdx.data(), cellStart.data(),
                cellCount.data(), cellBodies.data(), S->globalIdx.data(), reinterpret_cast<const uint2*>(excl.data()),
                nExcl, pairCount.data(), reinterpret_cast<uint2*>(pairs.data()), P, clothGroup.data(), cellRigid.data(),
                S->colOwner.data(), ccast<float4>(lp), ccast<float4>(S->posAng), S->colGroup.data(),
                S->colShared.data(), g);
        run = 0;
        for (uint32_t i = 0; i < producers; i++) { pairStart[i] = run; run += pairCount[i]; }
        for (uint32_t g = 0; g < producers; g++)
            ref::bp_emit_pairs_deterministic(
                ccast<float4>(S->posLin), ccast<float4>(colShape), S->hashedIdx.data(), cellStart.data(),
                cellCount.data(), cellBodies.data(), S->globalIdx.data(), reinterpret_cast<const uint2*>(excl.data()),
                nExcl, pairStart.data(), reinterpret_cast<uint2*>(pairs.data()), P, clothGroup.data(), cellRigid.data(),
                S->colOwner.data(), ccast<float4>(lp), ccast<float4>(S->posAng), S->colGroup.data(),
                S->colShared.data(), g);
        std::vector<uint32_t> ctrs(CTR_TOTAL, 0u), args(9, 0u);
        ref::bp_finalize_deterministic_pairs(pairCount.data(), pairStart.data(),
                                             reinterpret_cast<::atomic_uint*>(ctrs.data()), args.data(), P);
        const uint32_t npairs = ctrs[CTR_PAIRS];
        std::vector<uint32_t> meta = {ctrs[CTR_PAIR_CANDIDATES], npairs}, want = {S->pairCandidates, S->numPairs};
        compare_words(k, meta.data(), want.data(), 1, 2, false);
        compare_words(k, pairs.data(), S->pairs.data(), std::min(npairs, S->numPairs), 2, false);
    }

    // Dynamic coloring of rigid-only scenes: 20 Jacobi passes over the
    // double-buffered colors, the serial repair, validation, then the
    // per-color counts, offsets (color_scan, a threadgroup kernel, restated
    // here as the serial scan it performs) and the color lists.
    std::vector<uint32_t> colA, colB;
    void coloring(bool after) {
        if (!after) { colA = S->colorsA; colB = S->colorsB; return; }
        sync_params();
        const uint32_t nb = S->nb;
        auto* J = reinterpret_cast<const ref::JointGPU*>(S->joints.data());
        auto* Sp = reinterpret_cast<const ref::SpringGPU*>(S->springs.data());
        auto* M = reinterpret_cast<const ref::ManifoldGPU*>(S->manifolds.data());
        auto* T = reinterpret_cast<const ref::TetGPU*>(S->tets.data());
        auto* Sc = reinterpret_cast<const ref::SoftContactGPU*>(S->soft.data());
        auto* Mb = reinterpret_cast<const ref::MembraneGPU*>(S->membranes.data());
        auto* B = reinterpret_cast<const ref::BendGPU*>(S->bends.data());
        std::vector<uint32_t> changed(64, 0u);
        auto* chg = reinterpret_cast<::atomic_uint*>(changed.data());
        std::vector<uint32_t>* src = &colA;
        std::vector<uint32_t>* dst = &colB;
        for (uint32_t pass = 0; pass < 20; pass++) {
            for (uint32_t g = 0; g < nb; g++)
                ref::color_iterate(ccast<float4>(S->posLin), J, Sp, M, S->adjStart.data(), S->adjCount.data(),
                                   S->adjList.data(), src->data(), dst->data(), chg, P, T, Sc, Mb, B, pass, g);
            std::swap(src, dst);
        }
        std::vector<uint32_t>& fin = *src;
        uint32_t finalPass = 19;
        ref::color_repair_greedy(ccast<float4>(S->posLin), J, Sp, M, S->adjStart.data(), S->adjCount.data(),
                                 S->adjList.data(), fin.data(), chg, P, T, Sc, Mb, B, finalPass, 0u);
        std::vector<uint32_t> ctrs(CTR_TOTAL, 0u), bodySlot(nb, 0u), colorStart(MAX_COLORS + 2, 0u);
        auto* ct = reinterpret_cast<::atomic_uint*>(ctrs.data());
        for (uint32_t g = 0; g < nb; g++)
            ref::color_validate(ccast<float4>(S->posLin), J, Sp, M, S->adjStart.data(), S->adjCount.data(),
                                S->adjList.data(), fin.data(), ct, P, T, Sc, Mb, B, g);
        for (uint32_t g = 0; g < nb; g++) ref::color_count(ccast<float4>(S->posLin), fin.data(), ct, bodySlot.data(), P, g);
        uint32_t run = 0, used = 0;
        for (uint32_t c = 0; c < MAX_COLORS; c++) {
            colorStart[c] = run;
            run += ctrs[CTR_COLOR_BASE + c];
            if (ctrs[CTR_COLOR_BASE + c] > 0) used = c + 1;
        }
        colorStart[MAX_COLORS] = run;
        colorStart[MAX_COLORS + 1] = used;
        std::vector<uint32_t> colorList(std::max(run, 1u), 0u);
        for (uint32_t g = 0; g < nb; g++)
            ref::color_scatter(ccast<float4>(S->posLin), fin.data(), bodySlot.data(), colorStart.data(),
                               colorList.data(), P, g);
        const int k = Solver::ST_COLORING;
        st[k].calls += 1;
        compare_words(k, fin.data(), S->colorsA.data(), nb, 1, false);
        compare_words(k, colorStart.data(), S->colorStart.data(), MAX_COLORS + 2, 1, false);
        compare_words(k, colorList.data(), S->colorList.data(), run, 1, false);
        std::vector<uint32_t> conf = {ctrs[CTR_COLOR_CONFLICTS]}, want = {S->colorConflicts};
        compare_words(k, conf.data(), want.data(), 1, 1, false);
    }

    void on_stage(int stage, int arg, int after) {
        switch (stage) {
            case Solver::ST_WARM_JOINTS: warm_joints(after); break;
            case Solver::ST_WARM_BODIES: warm_bodies(after); break;
            case Solver::ST_PRIMAL: primal(arg, after); break;
            case Solver::ST_DUAL: dual(after); break;
            case Solver::ST_FINALIZE: finalize(after); break;
            case Solver::ST_NARROWPHASE: narrow(after); break;
            case Solver::ST_MAP: map(after); break;
            case Solver::ST_ADJACENCY: adjacency(after); break;
            case Solver::ST_COLORING: coloring(after); break;
            case Solver::ST_BROADPHASE: if (!after) iteration = 0; broadphase(after); break;
            default: break;
        }
    }

    // diag_error on the last frame's manifolds (GPUSolver.swift:4829-4864)
    float diag() {
        sync_params();
        counters[CTR_PAIRS] = S->numPairs;
        std::vector<uint32_t> out(1, 0u);
        const uint32_t n = (uint32_t)S->joints.size() + S->numPairs;
        for (uint32_t gid = 0; gid < n; gid++)
            ref::diag_error(ccast<float4>(S->posLin), ccast<float4>(S->posAng),
                            reinterpret_cast<const ref::JointGPU*>(S->joints.data()),
                            reinterpret_cast<const ref::ManifoldGPU*>(S->prevManifolds.data()), ctr(),
                            reinterpret_cast<::atomic_uint*>(out.data()), P, gid);
        return as_f(out[0]);
    }
};

void stage_hook(Solver* s, int stage, int arg, int after, void* ctx) {
    Pin* p = static_cast<Pin*>(ctx);
    p->S = s;
    p->on_stage(stage, arg, after);
}

}  // namespace

extern "C" {

// Attach the reference kernels to an oracle solver (from oracle_create).
// primal_every: check the primal on every k-th iteration only (1 = all).
void* ref_pin_attach(void* oracle_handle, uint32_t primal_every) {
    Solver* s = static_cast<Solver*>(oracle_handle);
    Pin* p = new Pin();
    p->S = s;
    p->primalEvery = primal_every ? primal_every : 1u;
    s->stageHook = &stage_hook;
    s->stageCtx = p;
    return p;
}

void ref_pin_detach(void* oracle_handle, void* pin) {
    Solver* s = static_cast<Solver*>(oracle_handle);
    if (s->stageCtx == pin) { s->stageHook = nullptr; s->stageCtx = nullptr; }
    delete static_cast<Pin*>(pin);
}

// out[stage * 6 + {0..5}] = calls, records compared, records mismatched,
// largest relative error of a mismatched float, first bad frame, first bad
// record index; stages in Solver::Stage order.
int ref_pin_stats(void* pin, double* out, uint32_t n) {
    Pin* p = static_cast<Pin*>(pin);
    for (uint32_t k = 0; k < (uint32_t)Solver::ST_COUNT_ && 6 * k + 5 < n; k++) {
        const StageStats& s = p->st[k];
        out[6 * k + 0] = s.calls;
        out[6 * k + 1] = s.compared;
        out[6 * k + 2] = s.mismatched;
        out[6 * k + 3] = s.maxRel;
        out[6 * k + 4] = (double)s.firstBadFrame;
        out[6 * k + 5] = (double)s.firstBadIndex;
    }
    return 0;
}

// Self-check of the harness: perturb one input of the given stage's
// reference run (the primal's inertial target of the first body of each
// color, the first contact's dual of the dual stage), so that comparison
// must report mismatches.
void ref_pin_perturb_for_testing(void* pin, int stage) { static_cast<Pin*>(pin)->perturbStage = stage; }

// The reference's diag_error on the oracle's current state.
float ref_pin_diag_error(void* pin) { return static_cast<Pin*>(pin)->diag(); }

}  // extern "C"
