// runtime.cu — the solver object behind the C ABI of include/avbd.h.
//
// Owns every device buffer (GPUSolver.swift:445-608), builds one CUDA graph
// per manifold-buffer parity for the whole frame (GPUSolver.swift:3138-4375
// encodes the same stage order into one Metal command buffer), replays it per
// frame, latches the first runtime failure (GPUSolver.swift:2800-2922) and
// serves state reads and writes.
#include <cuda_runtime.h>

#include <array>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/avbd.h"
#include "dmath.cuh"
#include "kernels.h"
#include "upload.h"

using namespace avbd;

namespace {
thread_local std::string g_last_error;
}  // namespace

namespace avbd {
// Message for avbd_last_error(NULL, ...) from entry points without a solver.
void set_thread_error(const char* msg) { g_last_error = msg; }
}  // namespace avbd

namespace {

__global__ void k_set_positions(float4* posLin, const float* xyz, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = posLin[i];
    posLin[i] = make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], p.w);
}

__global__ void k_set_states(DevPtrs d, const uint32_t* ids, const avbd_body_state* st, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t b = ids ? ids[i] : i;
    const avbd_body_state s = st[i];
    const float w = d.posLin[b].w;
    d.posLin[b] = make_float4(s.position[0], s.position[1], s.position[2], w);
    d.posAng[b] = make_float4(s.rotation[0], s.rotation[1], s.rotation[2], s.rotation[3]);
    d.velLin[b] = make_float4(s.velocity[0], s.velocity[1], s.velocity[2], 0.0f);
    d.velAng[b] = make_float4(s.angular_velocity[0], s.angular_velocity[1], s.angular_velocity[2], 0.0f);
    d.prevVelLin[b] = d.velLin[b];
    d.resetFlags[b] = 1u;
}

__global__ void k_set_motor_targets(JointGPU* joints, const uint32_t* ids, const float* targets, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    JointGPU& j = joints[ids[i]];
    if ((j.header.w & MOTOR_MODE_MASK) == 0u) return;   // welded/disabled: a no-op
    j.motor.x = targets[i];
}

// World anchors (rA.xyz), velocity commands (motor.x) and effort limits
// (motor.y) of listed joints; the host has validated every entry.
__global__ void k_set_joint_anchors(JointGPU* joints, const uint32_t* ids, const float* xyz, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    JointGPU& j = joints[ids[i]];
    j.rA.x = xyz[3 * i];
    j.rA.y = xyz[3 * i + 1];
    j.rA.z = xyz[3 * i + 2];
}
__global__ void k_set_motor_field(JointGPU* joints, const uint32_t* ids, const float* v, uint32_t n, int torque) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    JointGPU& j = joints[ids[i]];
    if (torque) j.motor.y = v[i];
    else j.motor.x = v[i];
}

// Hinge twist angle of child against parent and the twist rate about the
// child's hinge axis (GPUSolver.swift:2606-2637).
__global__ void k_motor_states(const JointGPU* joints, const float4* posAng, const float4* velAng,
                               const uint32_t* ids, uint32_t n, float* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const JointGPU& j = joints[ids[i]];
    const uint32_t a = j.header.x, b = j.header.y;
    const float4 qB = posAng[b];
    const float4 qA = a == WORLD_BODY ? make_float4(0, 0, 0, 1) : posAng[a];
    float4 r = q_mul(q_inv(q_mul(qA, tof(j.restRel))), qB);
    if (r.w < 0.0f) r = neg4(r);
    const float3 axis = xyz(tof(j.hingeAxis));
    out[2 * i] = 2.0f * atan2_series(dot(xyz(r), axis), r.w);
    const float3 wB = xyz(velAng[b]);
    const float3 wA = a == WORLD_BODY ? s3(0) : xyz(velAng[a]);
    out[2 * i + 1] = dot(wB - wA, q_rotate(qB, axis));
}
}  // namespace

struct avbd_snapshot {
    std::vector<std::vector<uint8_t>> blobs;
    uint64_t frame;
};

struct avbd_solver {
    HostScene H;
    DevPtrs d{};
    Sizes z{};
    Params P{};
    avbd_settings settings{};
    int device = 0;
    cudaStream_t stream = nullptr;       // the solver's own stream (graph capture)
    cudaStream_t launch = nullptr;       // where frames run: own or caller's stream
    // the learned warm start's predicted trial branch runs beside the plain
    // one on this stream (fork / join by events inside the frame)
    cudaStream_t branchStream = nullptr;
    cudaEvent_t forkEvent = nullptr, joinEvent = nullptr;
    cudaEvent_t wideFork = nullptr, wideJoin = nullptr;   // per-color side branch of the primal
    // per-stage profiling: events at stage boundaries inside the frame graph
    bool profiling = false;
    std::vector<cudaEvent_t> events;
    std::vector<int> intervalStage;
    int usedEvents = 0;
    avbd_profile prof{};
    uint64_t kernelsPerFrame = 0;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    bool graphsValid = false;
    // Dynamic coloring: the frame graph launches this many colors one by one
    // and a single-block tail kernel takes the rest.  It grows (and the graphs
    // are re-captured) when a retired frame used more colors.
    uint32_t colorLaunchBound = 8;
    bool colorBoundFitted = false;
    // batched worlds (avbd_create_batched): ragged body ranges, the bodies'
    // and motors' state at creation, the motorized joints of every world
    std::vector<uint32_t> worldOffsets;
    std::vector<avbd_body_state> initialStates;
    std::vector<float> initialMotorTargets;
    std::vector<std::vector<uint32_t>> worldMotors;
    // learned warm start
    static constexpr uint32_t kTraceLength = 2 + 256;
    int learnMode = AVBD_WARM_START_PLAIN;
    bool modelSet = false, learnCapture = false, residualTrace = false;
    uint32_t learnTrials = 1;

    // per-color launches are needed by the learned warm start's trial sweeps
    // and by the per-iteration residual trace
    void update_small_solve() {
        smallSolve = z.numDynamicBodies <= 512 && !P.cloth && !P.ogc && learnMode == AVBD_WARM_START_PLAIN && !learnCapture &&
                     !residualTrace;
        if (smallSolve) tuneStage = -1;
    }
    uint64_t frame = 0;
    int failure = AVBD_FAIL_NONE;
    std::string error;
    bool smallSolve = false;
    std::vector<void*> allocations;
    struct StateBuf { void* ptr; size_t bytes; };
    std::vector<StateBuf> state;       // buffers captured by snapshots
    // staging for host-side writes
    void* stage = nullptr;
    size_t stageBytes = 0;
    uint32_t* hostLatch = nullptr;     // pinned copy of the failure latch
    // render surface (built on the first smooth-normals call): surface
    // vertices, their incident triangles, face normals
    bool renderSurfaceReady = false;
    uint32_t numSurfVerts = 0;
    uint32_t *surfVerts = nullptr, *surfVtStart = nullptr, *surfVtCount = nullptr, *surfVtList = nullptr;
    uint32_t* surfClothVert = nullptr;
    float4* faceNormals = nullptr;
    // skin bindings (replaced by each upload)
    SkinBinding* skin = nullptr;
    uint32_t numSkin = 0;
    // the last Push-T environment table, kept on the device while the
    // caller passes the same records
    std::vector<avbd_pusht_env> pushtHost;
    PushTDev* pushtDev = nullptr;
    float4* pushtShapes = nullptr;  // 6 float4 per environment
    size_t pushtCap = 0;

    ~avbd_solver() {
        if (launch) cudaStreamSynchronize(launch);
        if (stream) cudaStreamSynchronize(stream);
        for (auto& g : graph) if (g) cudaGraphExecDestroy(g);
        for (auto& e : events) cudaEventDestroy(e);
        for (auto& e : tuneEvents) cudaEventDestroy(e);
        for (void* p : allocations) cudaFree(p);
        if (stage) cudaFree(stage);
        if (skin) cudaFree(skin);
        if (pushtDev) cudaFree(pushtDev);
        if (pushtShapes) cudaFree(pushtShapes);
        if (hostLatch) cudaFreeHost(hostLatch);
        if (forkEvent) cudaEventDestroy(forkEvent);
        if (joinEvent) cudaEventDestroy(joinEvent);
        if (wideFork) cudaEventDestroy(wideFork);
        if (wideJoin) cudaEventDestroy(wideJoin);
        if (branchStream) cudaStreamDestroy(branchStream);
        if (stream) cudaStreamDestroy(stream);
    }

    bool check(cudaError_t e, const char* what) {
        if (e == cudaSuccess) return true;
        if (failure == AVBD_FAIL_NONE) {
            failure = AVBD_FAIL_COMMAND_EXECUTION;
            error = std::string(what) + ": " + cudaGetErrorString(e);
        }
        return false;
    }

    template <typename T>
    bool alloc(T*& ptr, size_t count, const char* label, bool snapshot = false) {
        size_t bytes = sizeof(T) * (count ? count : 1);
        void* p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            error = std::string("allocation failed: ") + label;
            return false;
        }
        cudaMemset(p, 0, bytes);
        allocations.push_back(p);
        ptr = static_cast<T*>(p);
        if (snapshot) state.push_back({p, bytes});
        return true;
    }
    template <typename T>
    bool upload(T*& ptr, const std::vector<T>& host, const char* label, bool snapshot = false) {
        if (!alloc(ptr, host.size(), label, snapshot)) return false;
        if (!host.empty() && cudaMemcpy(ptr, host.data(), sizeof(T) * host.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
            error = std::string("upload failed: ") + label;
            return false;
        }
        return true;
    }

    void sync_params() {
        P.dt = settings.dt;
        P.gravity = settings.gravity;
        P.alpha = settings.alpha;
        P.betaLin = settings.beta_lin;
        P.betaAng = settings.beta_ang;
        P.gamma = settings.gamma;
        P.lambdaMax = settings.lambda_max;
        P.iterations = (uint32_t)(settings.iterations < 0 ? 0 : settings.iterations);
        P.rodDecayPow = settings.rod_decay_pow;
        P.particleDamping = settings.particle_damping;
        P.frictionCombineMode = settings.friction_combine_mode;
        P.collisionMargin = settings.collision_margin > 0.0f ? settings.collision_margin : 0.0f;
        P.rigidLinearDamping = settings.rigid_linear_damping > 0.0f ? settings.rigid_linear_damping : 0.0f;
        P.rigidAngularDamping = settings.rigid_angular_damping > 0.0f ? settings.rigid_angular_damping : 0.0f;
        P.clothViscosity = settings.cloth_viscosity;
    }

    // One frame, in the reference's stage order.  `parity` selects which
    // manifold buffer is "current" (the buffers swap after every frame).
    // With profiling on, an event is recorded at every stage boundary.
    void encode_frame(int parity) { encode_frame_on(parity, stream, nullptr, nullptr); }

    // One frame on stream `st`.  `lanes` overrides the per-color lane width
    // and `primalEvents` (2 per primal launch, in launch order) brackets every
    // primal launch; both are used by the autotuner's eager frames.
    void encode_frame_on(int parity, cudaStream_t st, const uint32_t* lanes, cudaEvent_t* primalEvents) {
        DevPtrs f = d;
        if (parity) {
            std::swap(f.manifolds, f.prevManifolds);
            std::swap(f.soft, f.prevSoft);
            std::swap(f.vtTrack, f.vtTrackPrev);
            std::swap(f.eeTrack, f.eeTrackPrev);
        }
        uint32_t* ogcSlots = d.counters ? reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(d.counters) +
                                                                      offsetof(Counters, ogcSlots))
                                        : nullptr;
        f.ogcExceed = ogcSlots;
        usedEvents = 0;
        uint32_t primalLaunch = 0;
        auto mark = [&](int stage) {
            if (!profiling || primalEvents) return;
            cudaEventRecordWithFlags(events[usedEvents], st, cudaEventRecordExternal);
            intervalStage[usedEvents] = stage;
            usedEvents++;
        };
        mark(AVBD_STAGE_BROADPHASE);
        cudaMemsetAsync(f.counters, 0, sizeof(Counters), st);
        launch_broadphase(P, f, z, st);
        mark(AVBD_STAGE_NARROWPHASE);
        launch_narrowphase(P, f, z, st);
        mark(AVBD_STAGE_PERSISTENCE_MAP);
        launch_map_rebuild(P, f, z, st);
        if (P.cloth) {
            mark(AVBD_STAGE_ELEMENT_CONTACTS);
            launch_cloth_detect(P, f, z, st);
        } else if (P.ogc) {
            mark(AVBD_STAGE_ELEMENT_CONTACTS);
            launch_ogc_detect(P, f, z, st);
        }
        mark(AVBD_STAGE_WARMSTART);
        launch_warmstart(P, f, z, st);
        if (P.cloth) {
            mark(AVBD_STAGE_ELEMENT_CONTACTS);
            launch_cloth_accept(P, f, z, st);
        }
        mark(AVBD_STAGE_ADJACENCY);
        launch_adjacency(P, f, z, st);
        if (z.dynamicColoring) {
            mark(AVBD_STAGE_COLORING);
            launch_dynamic_coloring(P, f, z, st);
        }
        const uint32_t colorBound = z.dynamicColoring ? colorLaunchBound : H.staticUsedColors;
        // One primal sweep over every color of pose buffers `g` (trial sweeps of
        // the learned warm start; the iteration loop inlines the same sequence).
        auto sweep = [&](const DevPtrs& g, cudaStream_t sst) {
            for (uint32_t c = 0; c < colorBound; c++) {
                const uint32_t count = z.dynamicColoring ? 0xFFFFFFFFu : H.colorCounts[c];
                if (count == 0) continue;
                launch_primal_color(P, g, z, c, count, H.colorLanes[c], sst);
                if (P.ogc)
                    launch_publish_color(P, g, c, count, z.dynamicColoring ? NO_HOST_START : H.colorStart[c], sst);
            }
            if (z.dynamicColoring) launch_primal_tail(P, g, z, colorLaunchBound, sst);
        };
        const bool tuningFrame = primalEvents != nullptr;
        const bool learned = !tuningFrame && learnMode == AVBD_WARM_START_LEARNED && modelSet && z.numLearn;
        const bool capture = !tuningFrame && learnCapture && z.numLearn;
        const bool trace = residualTrace;     // tuning frames too: they solve like any other
        // With one trial sweep the winner's swept pose is kept as the primal
        // half of the first iteration (the dual follows as usual); with more
        // trial sweeps both branches are undone and the solve restarts from
        // the chosen warm start.
        const bool reuseTrial = learned && learnTrials == 1 && P.iterations > 0;
        const size_t poseBytes = sizeof(float4) * z.numBodies;
        if (learned || capture || trace) {
            mark(AVBD_STAGE_LEARNED);
            if (learned || capture) launch_learn_features(P, f, z, st);
            if (capture || (learned && !reuseTrial)) {
                cudaMemcpyAsync(f.learnSaveLin, f.posLin, poseBytes, cudaMemcpyDeviceToDevice, st);
                cudaMemcpyAsync(f.learnSaveAng, f.posAng, poseBytes, cudaMemcpyDeviceToDevice, st);
            }
            if (trace) launch_residual(P, f, z, f.learnResidBodies, f.learnTrace + 0, st);
        }
        if (learned) {
            // The predicted branch runs in its own pose buffers (fb); the
            // plain branch sweeps the solver's pose in place.
            DevPtrs fb = f, fp = f;
            fb.posLin = f.learnSweptLin;
            fb.posAng = f.learnSweptAng;
            // the trial sweeps count OGC bound exceeders in slots 2 (plain) and 3 (predicted)
            if (ogcSlots) { fp.ogcExceed = ogcSlots + 2; fb.ogcExceed = ogcSlots + 3; }
            launch_mlp_infer(f.learnHalf, f.learnPrm, f.learnNorm, f.learnFeat, z.numLearn, f.learnPred,
                             f.failureLatch, st);
            launch_learn_branch(P, f, z, st);
            if (trace) launch_residual(P, fb, z, f.learnResidBodies, f.learnTrace + 1, st);
            // The two trial branches touch disjoint pose buffers (in
            // color-Jacobi scenes the predicted branch also has its own
            // pending-solve buffers), so the predicted one runs on a second
            // stream beside the plain one.
            if (P.colorJacobi) { fb.posNext = f.learnNextLin; fb.angNext = f.learnNextAng; }
            const bool fork = !P.colorJacobi || f.learnNextLin != nullptr;
            cudaStream_t bst = fork ? branchStream : st;
            if (fork) {
                cudaEventRecord(forkEvent, st);
                cudaStreamWaitEvent(bst, forkEvent, 0);
            }
            for (uint32_t t = 0; t < learnTrials; t++) sweep(fb, bst);
            launch_residual(P, fb, z, f.learnResidBodies2, f.learnResid + 1, bst);
            for (uint32_t t = 0; t < learnTrials; t++) sweep(fp, st);
            launch_residual(P, f, z, f.learnResidBodies, f.learnResid + 0, st);
            if (fork) {
                cudaEventRecord(joinEvent, bst);
                cudaStreamWaitEvent(st, joinEvent, 0);
            }
            if (reuseTrial) {
                launch_learn_adopt(P, f, z, st);
            } else {
                if (learnTrials > 0) {  // undo the plain branch's trial sweeps
                    cudaMemcpyAsync(f.posLin, f.learnSaveLin, poseBytes, cudaMemcpyDeviceToDevice, st);
                    cudaMemcpyAsync(f.posAng, f.learnSaveAng, poseBytes, cudaMemcpyDeviceToDevice, st);
                }
                launch_learn_select(P, f, z, st);
            }
        } else if (trace) {
            launch_copy_double(f.learnTrace + 0, f.learnTrace + 1, st);
        }
        if (smallSolve) {
            mark(AVBD_STAGE_PRIMAL);
            launch_solve_small(P, f, z, z.dynamicColoring ? (uint32_t)MAX_COLORS : H.staticUsedColors, st);
        } else {
            for (uint32_t it = 0; it < P.iterations; it++) {
                // OGC bound exceeders of this pass alternate between slots 0 and 1
                DevPtrs g = f;
                if (ogcSlots) g.ogcExceed = ogcSlots + (it & 1u);
                for (uint32_t c = 0; c < colorBound && !(reuseTrial && it == 0); c++) {
                    const uint32_t count = z.dynamicColoring ? 0xFFFFFFFFu : H.colorCounts[c];
                    if (count == 0) continue;
                    mark(AVBD_STAGE_PRIMAL);
                    if (primalEvents) cudaEventRecord(primalEvents[2 * primalLaunch], st);
                    launch_primal_color(P, g, z, c, count, lanes ? lanes[c] : H.colorLanes[c], st, branchStream,
                                        wideFork, wideJoin);
                    if (primalEvents) cudaEventRecord(primalEvents[2 * primalLaunch + 1], st);
                    primalLaunch++;
                    if (P.cloth) {
                        mark(AVBD_STAGE_TRUNCATION);
                        launch_dat_color(P, f, z, c, count, st);
                    } else if (P.ogc) {
                        launch_publish_color(P, f, c, count, z.dynamicColoring ? NO_HOST_START : H.colorStart[c],
                                             st);
                    }
                }
                if (z.dynamicColoring && !(reuseTrial && it == 0)) launch_primal_tail(P, g, z, colorLaunchBound, st);
                mark(AVBD_STAGE_DUAL);
                launch_dual(P, f, z, st);
                if (P.ogc && it + 1 < P.iterations) {
                    mark(AVBD_STAGE_TRUNCATION);
                    launch_ogc_refresh(P, f, z, ogcSlots + (it & 1u), ogcSlots + ((it + 1u) & 1u), st);
                }
                if (trace && it + 2 < kTraceLength)
                    launch_residual(P, f, z, f.learnResidBodies, f.learnTrace + 2 + it, st);
            }
        }
        if (capture) launch_learn_target(P, f, z, st);
        mark(AVBD_STAGE_FINALIZE);
        if (P.cloth) launch_cloth_restore(P, f, z, st);
        launch_finalize(P, f, z, st);
        if (z.numTris) launch_cloth_smoothing(P, f, z, st);
        launch_frame_end(P, f, z, st);
        mark(-1);
    }

    int events_needed() const {
        const uint32_t colorBound = z.dynamicColoring ? colorLaunchBound : H.staticUsedColors;
        return 20 + (int)(P.iterations * (2 * colorBound + 1));
    }

    bool build_graphs() {
        if (profiling) {
            const int need = events_needed();
            while ((int)events.size() < need) {
                cudaEvent_t e;
                if (!check(cudaEventCreate(&e), "event create")) return false;
                events.push_back(e);
            }
            intervalStage.assign(events.size(), -1);
        }
        for (int parity = 0; parity < 2; parity++) {
            if (graph[parity]) { cudaGraphExecDestroy(graph[parity]); graph[parity] = nullptr; }
            cudaGraph_t g = nullptr;
            if (!check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture")) return false;
            encode_frame(parity);
            cudaError_t e = cudaStreamEndCapture(stream, &g);
            if (!check(e, "end capture")) return false;
            size_t nodes = 0;
            cudaGraphGetNodes(g, nullptr, &nodes);
            std::vector<cudaGraphNode_t> list(nodes);
            if (nodes) cudaGraphGetNodes(g, list.data(), &nodes);
            uint64_t kernels = 0;
            for (cudaGraphNode_t n : list) {
                cudaGraphNodeType t;
                if (cudaGraphNodeGetType(n, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) kernels++;
            }
            kernelsPerFrame = kernels;
            e = cudaGraphInstantiate(&graph[parity], g, 0);
            cudaGraphDestroy(g);
            if (!check(e, "graph instantiate")) return false;
        }
        graphsValid = true;
        return true;
    }

    int create(const avbd_scene_desc* s) {
        int rc = upload_scene(s, H, error);
        if (rc != AVBD_OK) return rc;
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) { error = "no CUDA device"; return AVBD_ERR_NO_DEVICE; }
        device = s->device >= 0 ? s->device : 0;
        if (s->device < 0) cudaGetDevice(&device);
        if (device >= count || cudaSetDevice(device) != cudaSuccess) { error = "cannot select CUDA device"; return AVBD_ERR_NO_DEVICE; }
        if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamCreateWithFlags(&branchStream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&forkEvent, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&joinEvent, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&wideFork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&wideJoin, cudaEventDisableTiming) != cudaSuccess) {
            error = "stream creation failed";
            return AVBD_ERR_NO_DEVICE;
        }
        launch = stream;
        settings = s->settings;
        P = H.P;
        sync_params();
        const uint32_t nb = H.numBodies, nc = H.numColliders;
        z.numBodies = nb;
        z.numColliders = nc;
        z.numActiveJoints = (uint32_t)H.activeJoints.size();
        z.numHardSprings = (uint32_t)H.hardSprings.size();
        z.numTets = (uint32_t)H.tets.size();
        z.maxPairs = H.maxPairs;
        z.producers = P.numHashed + P.numGlobals;
        z.numDynamicBodies = H.numDynamicBodies;
        z.dynamicColoring = H.dynamicColoring;
        z.particleFastPath = H.particleFastPath;
        z.numTris = H.numTris;
        z.numParticles = P.numParticles;
        z.numEdges = P.numEdges;
        z.numMembranes = (uint32_t)H.membranes.size();
        z.numBends = (uint32_t)H.bends.size();
        z.maxDatPairs = H.maxDatPairs;
        z.maxSoft = P.maxSoft;
        z.elemHashSize = H.elemHashSize;
        z.numLearnAll = P.cloth ? 0u : (uint32_t)H.learnIdx.size();
        z.numLearn = P.cloth ? 0u : P.learnParticles;
        z.colorCounts = H.dynamicColoring ? nullptr : H.colorCounts.data();
        z.colorLanes = H.colorLanes.data();
        z.colorLean = H.colorLean.data();
        z.colorStartHost = H.dynamicColoring ? nullptr : H.colorStart.data();
        z.numDynamicRigid = 0;
        for (uint32_t b = 0; b < nb; b++) z.numDynamicRigid += (H.posLin[b].w > 0.0f && H.shape[b].w >= 0.0f) ? 1u : 0u;
        const uint32_t scanLimit = 1024u * 1024u;
        if (P.gridHashSize > scanLimit || z.producers > scanLimit || nb > scanLimit) {
            error = "scene exceeds the 1M-element scan limit of this library";
            return AVBD_ERR_UNSUPPORTED;
        }
        bool ok = true;
        // bodies
        ok = ok && upload(reinterpret_cast<f4*&>(d.posLin), H.posLin, "posLin", true);
        ok = ok && upload(reinterpret_cast<f4*&>(d.posAng), H.posAng, "posAng", true);
        ok = ok && alloc(d.initLin, nb, "initLin", true) && alloc(d.initAng, nb, "initAng", true);
        ok = ok && alloc(d.inertLin, nb, "inertLin", true) && alloc(d.inertAng, nb, "inertAng", true);
        ok = ok && upload(reinterpret_cast<f4*&>(d.velLin), H.velLin, "velLin", true);
        ok = ok && upload(reinterpret_cast<f4*&>(d.velAng), H.velAng, "velAng", true);
        ok = ok && upload(reinterpret_cast<f4*&>(d.prevVelLin), H.prevVelLin, "prevVelLin", true);
        ok = ok && upload(reinterpret_cast<f4*&>(d.props), H.props, "props");
        ok = ok && upload(reinterpret_cast<f4*&>(d.shape), H.shape, "shape");
        ok = ok && upload(reinterpret_cast<f4*&>(d.spinVel), H.spinVel, "spinVel");
        ok = ok && upload(d.gravityScale, H.gravityScale, "gravityScale");
        ok = ok && upload(d.clothGroup, H.clothGroup, "clothGroup");
        ok = ok && upload(d.bodyShape, H.shapeType, "bodyShape");
        // colliders
        ok = ok && upload(d.colOwner, H.colOwner, "colliderOwner") && upload(d.colShapeType, H.colShapeType, "colliderShapeType");
        ok = ok && upload(d.colGroup, H.colGroup, "colliderGroup") && upload(d.colShared, H.colShared, "colliderShared");
        ok = ok && upload(reinterpret_cast<f4*&>(d.colShape), H.colShape, "colliderShape");
        ok = ok && upload(reinterpret_cast<f4*&>(d.colLocalPos), H.colLocalPos, "colliderLocalPosition");
        ok = ok && upload(reinterpret_cast<f4*&>(d.colLocalRot), H.colLocalRot, "colliderLocalRotation");
        ok = ok && upload(reinterpret_cast<float*&>(d.colFriction), H.colFriction, "colliderFriction");
        ok = ok && upload(reinterpret_cast<uint32_t*&>(d.colHullRange), H.colHullRange, "colliderHullRange");
        ok = ok && upload(reinterpret_cast<f4*&>(d.hullVerts), H.hullVerts, "convexHullVertices");
        ok = ok && upload(d.hashedIdx, H.hashedIdx, "hashedIdx") && upload(d.globalIdx, H.globalIdx, "globalIdx");
        ok = ok && upload(d.exclusions, H.exclusions, "exclusions");
        // broadphase
        ok = ok && alloc(d.cellCount, P.gridHashSize, "cellCount") && alloc(d.cellStart, P.gridHashSize, "cellStart");
        ok = ok && alloc(d.cellRigid, P.gridHashSize, "cellRigid") && alloc(d.cellBodies, P.numHashed, "cellBodies");
        ok = ok && alloc(d.bodyCellSlot, P.numHashed, "bodyCellSlot") && alloc(d.cellTmp, P.numHashed, "cellBodiesUnsorted");
        ok = ok && alloc(d.colBucket, nc, "colliderBucket") && alloc(d.rigidStart, P.gridHashSize, "rigidStart");
        ok = ok && alloc(d.rigidCells, P.numHashed, "rigidCells");
        z.numHeavyProducers = 0;
        if (P.fineBP) {
            std::vector<uint32_t> heavy;
            for (uint32_t i = 0; i < P.numHashed; i++)
                if (H.colShape[H.hashedIdx[i]].w >= 0.0f) heavy.push_back(i);
            z.numHeavyProducers = (uint32_t)heavy.size();
            ok = ok && upload(d.heavyProducers, heavy, "heavyProducers");
            ok = ok && alloc(d.fineCount, P.fineHashSize, "fineCount") && alloc(d.fineStart, P.fineHashSize, "fineStart");
            ok = ok && alloc(d.fineTmp, P.numHashed, "fineCellsUnsorted") && alloc(d.fineCells, P.numHashed, "fineCells");
            ok = ok && alloc(d.fineSlot, P.numHashed, "fineSlot");
        }
        ok = ok && alloc(d.pairCount, z.producers, "pairCount") && alloc(d.pairStart, z.producers, "pairStart");
        ok = ok && alloc(d.pairLaneCount, (size_t)z.producers * 32, "pairLaneCount");
        ok = ok && alloc(d.pairs, H.maxPairs, "pairs");
        ok = ok && alloc(d.colCenter, nc, "colliderCenter") && alloc(d.colMeta, nc, "colliderMeta");
        ok = ok && alloc(d.globalChunk, 4 * (size_t)std::max<uint32_t>(1, (P.numGlobals + 31) / 32), "globalChunkBoxes");
        {
            std::vector<uint32_t> owners(std::max<size_t>(1, H.globalIdx.size()), 0u);
            for (size_t g = 0; g < H.globalIdx.size(); g++) owners[g] = H.colOwner[H.globalIdx[g]];
            ok = ok && upload(d.globalOwner, owners, "globalOwner");
            ok = ok && alloc(d.globalRec, 3 * (size_t)std::max<uint32_t>(1, P.numGlobals), "globalRecords");
        }
        ok = ok && alloc(d.manifolds, H.maxPairs, "manifolds", true) && alloc(d.prevManifolds, H.maxPairs, "prevManifolds", true);
        ok = ok && alloc(d.mapKeyA, H.mapCapacity, "mapKeyA", true) && alloc(d.mapKeyB, H.mapCapacity, "mapKeyB", true);
        ok = ok && alloc(d.mapVal, H.mapCapacity, "mapVal", true);
        // constraints
        ok = ok && upload(d.joints, H.joints, "joints", true) && upload(d.activeJoints, H.activeJoints, "activeJoints");
        ok = ok && upload(reinterpret_cast<f4*&>(d.initPenLin), H.initPenLin, "initialJointPenaltyLin");
        ok = ok && upload(reinterpret_cast<f4*&>(d.initPenAng), H.initPenAng, "initialJointPenaltyAng");
        ok = ok && upload(d.springs, H.springs, "springs", true) && upload(d.hardSprings, H.hardSprings, "hardSprings");
        ok = ok && upload(d.tets, H.tets, "tets");
        // adjacency
        ok = ok && upload(reinterpret_cast<u4*&>(d.staticSeg), H.staticSeg, "staticSeg");
        ok = ok && upload(d.preList, H.preList, "preList") && upload(d.postList, H.postList, "postList");
        ok = ok && alloc(d.dynCount, nb, "dynCount") && alloc(d.dynStart, nb, "dynStart") && alloc(d.dynCursor, nb, "dynCursor");
        ok = ok && alloc(d.dynSplit, nb, "dynSplit") && upload(d.postTets, H.postTets, "postTets");
        d.tetInc = nullptr;
#ifndef AVBD_NO_TET_INCIDENCE
        if (ok && !H.tetInc.empty()) {
            TetGPU* ti = nullptr;
            ok = upload(ti, H.tetInc, "tetIncidence");
            d.tetInc = ti;
        }
#endif
        ok = ok && alloc(d.adjLongQueue, nb, "adjLongQueue");
        ok = ok && alloc(d.dynList, 2 * (size_t)H.maxPairs + ((P.cloth || P.ogc) ? 4 * (size_t)P.maxSoft : 0), "dynList");
        // coloring
        ok = ok && upload(d.colorsA, H.colors, "colorsA", true) && upload(d.colorsB, H.colors, "colorsB");
        ok = ok && alloc(d.bodySlot, nb, "bodySlot");
        if (H.dynamicColoring) {
            ok = ok && alloc(d.colorList, nb, "colorList");
        } else {
            ok = ok && upload(d.colorList, H.colorList, "colorList");
            ok = ok && upload(d.colorLaunch, H.colorLaunch, "colorLaunch");
            ok = ok && upload(d.colorStart, H.colorStart, "colorStart");
        }
        // control
        ok = ok && alloc(d.counters, 1, "counters") && alloc(d.scanScratch, 1024 + 32, "scanScratch");
        ok = ok && alloc(d.diag, 1, "diag") && alloc(d.resetFlags, nb, "resetFlags");
        ok = ok && alloc(d.failureLatch, 4, "failureLatch") && alloc(d.frameCounter, 1, "frameCounter", true);
        if (H.dynamicColoring)
            d.colorStart = reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(d.counters) + offsetof(Counters, colorStart));
        if (ok) d.ogcExceed = reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(d.counters) + offsetof(Counters, ogcSlots));
        if (z.numLearnAll) {
            const uint32_t nl = z.numLearnAll;
            ok = ok && upload(d.learnIdx, H.learnIdx, "learnIdx");
            std::vector<uint32_t> slot(nb, 0xFFFFFFFFu);
            for (uint32_t i = 0; i < nl; i++) slot[H.learnIdx[i]] = i;
            ok = ok && upload(d.learnSlot, slot, "learnSlot");
            // static feature parts: incident stiffness (springs, then tets /
            // membranes / bends, in adjacency order) and the 1-ring of
            // vertices sharing a spring or tet, with multiplicities
            std::vector<float> stiff(nl, 0.0f), ringN(nl, 0.0f);
            std::vector<uint32_t> ringStart(nl + 1, 0);
            std::vector<uint2> ring;
            for (uint32_t i = 0; i < nl; i++) {
                const uint32_t v = H.learnIdx[i];
                const u4 sg = H.staticSeg[v];
                float k = 0.0f;
                std::vector<std::pair<uint32_t, uint32_t>> nbr;   // (slot, multiplicity) in first-visit order
                auto visit = [&](uint32_t u) {
                    if (u == v || u == WORLD_BODY) return;
                    ringN[i] += 1.0f;
                    if (!(H.posLin[u].w > 0.0f) || slot[u] == 0xFFFFFFFFu) return;
                    for (auto& e : nbr) if (e.first == slot[u]) { e.second++; return; }
                    nbr.push_back({slot[u], 1u});
                };
                for (uint32_t q = 0; q < sg.y; q++) {
                    const uint32_t e = H.preList[sg.x + q];
                    if ((e >> ADJ_KIND_SHIFT) != FK_SPRING) continue;
                    const SpringGPU& sp = H.springs[e & ADJ_INDEX_MASK];
                    k += sp.rA.w;
                    visit(sp.header.x == v ? sp.header.y : sp.header.x);
                }
                for (uint32_t q = 0; q < sg.w; q++) {
                    const uint32_t e = H.postList[sg.z + q], kind = e >> ADJ_KIND_SHIFT, idx = e & ADJ_INDEX_MASK;
                    if (kind == FK_TET) {
                        k += H.tets[idx].r1.w + H.tets[idx].r2.w;
                        visit(H.tets[idx].ids.x); visit(H.tets[idx].ids.y);
                        visit(H.tets[idx].ids.z); visit(H.tets[idx].ids.w);
                    } else if (kind == FK_MEMBRANE) {
                        k += H.membranes[idx].mat.x + H.membranes[idx].mat.y;
                    } else if (kind == FK_BEND) {
                        k += H.bends[idx].mat.x;
                    }
                }
                stiff[i] = k;
                for (auto& e : nbr) ring.push_back(make_uint2(e.first, e.second));
                ringStart[i + 1] = (uint32_t)ring.size();
            }
            ok = ok && upload(d.learnStiff, stiff, "learnStiffness") && upload(d.learnRingN, ringN, "learnRingSize");
            ok = ok && upload(d.learnRingStart, ringStart, "learnRingStart") && upload(d.learnRing, ring, "learnRing");
            ok = ok && alloc(d.learnStat, nl, "learnContactState") && alloc(d.learnGap, nl, "learnContactGap");
            ok = ok && alloc(d.learnFeat, 32 * (size_t)nl, "learnFeatures") && alloc(d.learnPred, 6 * (size_t)nl, "learnPrediction");
            ok = ok && alloc(d.learnTarget, 6 * (size_t)nl, "learnTarget");
            ok = ok && alloc(d.learnPrm, mlp_param_count(), "mlpParams") && alloc(d.learnNorm, mlp_norm_count(), "mlpNorm");
            uint16_t* half = nullptr;
            ok = ok && alloc(half, mlp_half_count(), "mlpWeightsBF16");
            d.learnHalf = half;
        }
        ok = ok && alloc(d.learnSaveLin, nb, "plainWarmStartLin") && alloc(d.learnSaveAng, nb, "plainWarmStartAng");
        ok = ok && alloc(d.learnSweptLin, nb, "plainTrialLin") && alloc(d.learnSweptAng, nb, "plainTrialAng");
        ok = ok && alloc(d.learnResidBodies, std::max<uint32_t>(1, H.numDynamicBodies), "residualBodies");
        ok = ok && alloc(d.learnResidBodies2, std::max<uint32_t>(1, H.numDynamicBodies), "residualBodiesBranch");
        if (z.numLearnAll && P.colorJacobi)
            ok = ok && alloc(d.learnNextLin, nb, "branchNextLin") && alloc(d.learnNextAng, nb, "branchNextAng");
        ok = ok && alloc(d.learnResid, 4, "residual") && alloc(d.learnTrace, kTraceLength, "residualTrace");
        ok = ok && alloc(d.learnAccepted, 1, "learnAccepted", true);
        if (H.numTris > 0) {
            // element topology
            ok = ok && upload(reinterpret_cast<u4*&>(d.tris), H.tris, "tris");
            ok = ok && upload(reinterpret_cast<uint32_t*&>(d.edges), H.edges, "edges");
            ok = ok && upload(d.nbrStart, H.nbrStart, "nbrStart") && upload(d.nbrCount, H.nbrCount, "nbrCount");
            ok = ok && upload(d.nbrList, H.nbrList, "nbrList") && upload(d.particleIdx, H.particleIdx, "particleIdx");
            ok = ok && upload(d.selfCollision, H.selfCollision, "softSelfCollision");
            ok = ok && upload(d.membranes, H.membranes, "membranes") && upload(d.bends, H.bends, "bends");
        }
        if (P.cloth || P.ogc) {
            // element grid, pair streams, element contacts
            const size_t elems = (size_t)H.numTris + H.numEdges;
            const uint32_t owners = P.numParticles + H.numEdges;
            ok = ok && alloc(d.elemCellCount, 2 * (size_t)H.elemHashSize, "elemCellCount");
            ok = ok && alloc(d.elemCellStart, 2 * (size_t)H.elemHashSize, "elemCellStart");
            ok = ok && alloc(d.elemCursor, 2 * (size_t)H.elemHashSize, "elemCursor");
            ok = ok && alloc(d.elemCells, (P.ogc ? 27 : 64) * elems, "elemCells");
            ok = ok && alloc(d.datOwnerCount, owners, "datOwnerCount") && alloc(d.datOwnerStart, owners, "datOwnerStart");
            ok = ok && alloc(d.datEmit, owners, "datEmit") && alloc(d.datEmitStart, owners, "datEmitStart");
            ok = ok && alloc(d.rtCount, H.numTris, "rtCount") && alloc(d.rtStart, H.numTris, "rtStart");
            ok = ok && alloc(d.rtCand, RT_MAX_PER_TRI * (size_t)H.numTris, "rtCandidates");
            ok = ok && alloc(d.soft, P.maxSoft, "softContacts", true) && alloc(d.prevSoft, P.maxSoft, "prevSoftContacts", true);
            ok = ok && alloc(d.softKeyA, P.softMapCapacity, "softMapKeyA", true);
            ok = ok && alloc(d.softKeyB, P.softMapCapacity, "softMapKeyB", true) &&
                 alloc(d.softVal, P.softMapCapacity, "softMapVal", true);
            ok = ok && alloc(d.ogcPrev, nb, "ogcPrev", true) && alloc(d.posNext, nb, "posNext", true) && alloc(d.angNext, nb, "angNext", true);
            const uint32_t scanMax = std::max(std::max(2 * H.elemHashSize, owners), H.numTris);
            ok = ok && alloc(d.bigScanScratch, scan_large_scratch_words(scanMax), "scanScratchLarge");
        }
        if (P.cloth) {
            const size_t elems = (size_t)H.numTris + H.numEdges;
            ok = ok && alloc(d.elemBox, 2 * elems, "elemBox");
            ok = ok && alloc(d.elemRange, elems, "elemRange");
            ok = ok && alloc(d.datPairs, H.maxDatPairs, "planarDATPairs");
            ok = ok && alloc(d.datCache, 16 * ((size_t)P.numParticles + H.numEdges), "planarDATPairCache");
            std::vector<uint32_t> ones(nb, 0x3F800000u);
            ok = ok && upload(d.truncBits, ones, "planarDATT");
        }
        if (P.ogc) {
            const size_t elems = (size_t)H.numTris + P.numEdges;
            ok = ok && upload(reinterpret_cast<u4*&>(d.triAdj), H.triAdj, "triAdj");
            ok = ok && upload(d.nbr2Start, H.nbr2Start, "nbr2Start") && upload(d.nbr2Count, H.nbr2Count, "nbr2Count");
            ok = ok && upload(d.nbr2List, H.nbr2List, "nbr2List");
            ok = ok && upload(d.vertEdgeStart, H.vertEdgeStart, "vertEdgeStart") &&
                 upload(d.vertEdgeCount, H.vertEdgeCount, "vertEdgeCount");
            ok = ok && upload(d.vertEdgeList, H.vertEdgeList, "vertEdgeList") && upload(d.clothVert, H.clothVert, "clothVertFlag");
            std::vector<u4> none(nb, u4{0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu});
            ok = ok && upload(reinterpret_cast<u4*&>(d.vtTrack), none, "vtTrack", true) &&
                 upload(reinterpret_cast<u4*&>(d.vtTrackPrev), none, "vtTrackPrev", true);
            none.assign(std::max<uint32_t>(1, H.numEdges), u4{0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu});
            ok = ok && upload(reinterpret_cast<u4*&>(d.eeTrack), none, "eeTrack", true) &&
                 upload(reinterpret_cast<u4*&>(d.eeTrackPrev), none, "eeTrackPrev", true);
            ok = ok && alloc(d.ogcBounds, nb, "ogcBounds") && alloc(d.elemCellsTmp, 27 * elems, "elemCellsUnsorted");
            ok = ok && alloc(d.ogcPartial, 3 * ((size_t)P.numParticles + P.numEdges), "ogcPartialTrack");
        }
        std::vector<uint32_t> spB, rJ;
        std::vector<f4> spA;
        std::vector<float> rV;
        for (const auto& sp : H.spinners) { spB.push_back((uint32_t)sp.body); spA.push_back(f4{sp.axis[0], sp.axis[1], sp.axis[2], sp.omega}); }
        for (const auto& rm : H.rateMotors) { rJ.push_back(rm.first); rV.push_back(rm.second); }
        ok = ok && upload(d.spinnerBody, spB, "spinnerBody") && upload(reinterpret_cast<f4*&>(d.spinnerAxisOmega), spA, "spinnerAxis");
        ok = ok && upload(d.rateJoint, rJ, "rateJoint") && upload(d.rateValue, rV, "rateValue");
        d.numSpinners = (uint32_t)spB.size();
        d.numRateMotors = (uint32_t)rJ.size();
        if (!ok) return AVBD_ERR_ALLOC_FAILED;
        if (cudaMallocHost(&hostLatch, 4 * sizeof(uint32_t)) != cudaSuccess) {
            error = "pinned allocation failed";
            return AVBD_ERR_ALLOC_FAILED;
        }
        std::memset(hostLatch, 0, 4 * sizeof(uint32_t));
        // Small scenes run their whole iteration loop in one thread block.
        update_small_solve();
        tuneStage = tuning_applies() ? 0 : -1;
        dyn_tune_setup();
        if (cudaDeviceSynchronize() != cudaSuccess) { error = "device error during upload"; return AVBD_ERR_NO_DEVICE; }
        return AVBD_OK;
    }

    // Wait for the stream, then surface an execution error or a latched
    // capacity/coloring failure.
    int retire() {
        if (!check(cudaStreamSynchronize(launch), "frame execution")) return AVBD_ERR_RUNTIME_FAILURE;
        if (!check(cudaMemcpy(hostLatch, d.failureLatch, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost), "latch readback"))
            return AVBD_ERR_RUNTIME_FAILURE;
        if (z.dynamicColoring && hostLatch[3] > 0) {
            // first retirement: fit the bound to the palette seen so far
            // (two colors of headroom); later frames only grow it
            const uint32_t want = std::min<uint32_t>(MAX_COLORS, hostLatch[3] + 2);
            if (want > colorLaunchBound || (!colorBoundFitted && want < colorLaunchBound)) {
                colorLaunchBound = want;
                graphsValid = false;
            }
            colorBoundFitted = true;
        }
        if (hostLatch[0] != 0 && failure == AVBD_FAIL_NONE) {
            failure = (int)hostLatch[0];
            char buf[160];
            if (failure == AVBD_FAIL_RIGID_PAIR_CAPACITY)
                std::snprintf(buf, sizeof buf, "rigid pair capacity exceeded at frame %u: %u candidates > %u",
                              hostLatch[1], hostLatch[2], H.maxPairs);
            else if (failure == AVBD_FAIL_SOFT_CONTACT_CAPACITY)
                std::snprintf(buf, sizeof buf, "soft contact capacity exceeded at frame %u: %u records > %u",
                              hostLatch[1], hostLatch[2], P.maxSoft);
            else if (failure == AVBD_FAIL_PLANAR_DAT_PAIR_CAPACITY)
                std::snprintf(buf, sizeof buf, "Planar-DAT pair capacity exceeded at frame %u: %u pairs > %u",
                              hostLatch[1], hostLatch[2], P.maxDatPairs);
            else if (failure == AVBD_FAIL_PLANAR_DAT_GRID_SPAN)
                std::snprintf(buf, sizeof buf, "Planar-DAT element grid span exceeded at frame %u: %u elements",
                              hostLatch[1], hostLatch[2]);
            else if (failure == AVBD_FAIL_WAIT_TIMEOUT)
                std::snprintf(buf, sizeof buf, "a bounded device wait (warm-start MLP inference) gave up during "
                              "frame %u", hostLatch[1]);
            else if (failure == AVBD_FAIL_PLANAR_DAT_INVALID_ANCHOR)
                std::snprintf(buf, sizeof buf, "Planar-DAT invalid anchor at frame %u: %u pairs", hostLatch[1],
                              hostLatch[2]);
            else
                std::snprintf(buf, sizeof buf, "unresolved dynamic coloring at frame %u: %u conflicting bodies",
                              hostLatch[1], hostLatch[2]);
            error = buf;
        }
        return failure == AVBD_FAIL_NONE ? AVBD_OK : AVBD_ERR_RUNTIME_FAILURE;
    }

    // Primal variant autotuner.  Each static color's primal can run the
    // grouped kernel with 8, 16 or 32 lanes per body or the staged kernel;
    // the fold order is fixed, so every variant computes the same floats and
    // only speed differs (it depends on the color's body count and adjacency
    // sizes).  The first four frames run eagerly, one variant each, with
    // events around every primal launch; each color then keeps its fastest
    // variant and the frame graphs are captured with it.
    static constexpr int kTuneVariants = 4;
    static constexpr uint32_t kTuneWidths[kTuneVariants] = {8, 16, 32, AVBD_PRIMAL_STAGED};
    int tuneStage = -1;                       // -1 off / done, else the next variant
    double tuneMs[kTuneVariants][MAX_COLORS] = {};
    std::vector<cudaEvent_t> tuneEvents;

    bool tuning_applies() const { return !z.dynamicColoring && !smallSolve && H.staticUsedColors > 0; }

    int tune_frame() {
        const uint32_t colorBound = H.staticUsedColors;
        const size_t need = 2 * (size_t)P.iterations * colorBound;
        while (tuneEvents.size() < need) {
            cudaEvent_t e;
            if (!check(cudaEventCreate(&e), "event create")) return AVBD_ERR_RUNTIME_FAILURE;
            tuneEvents.push_back(e);
        }
        uint32_t lanes[MAX_COLORS];
        for (int c = 0; c < MAX_COLORS; c++) lanes[c] = kTuneWidths[tuneStage];
        encode_frame_on((int)(frame & 1), launch, lanes, tuneEvents.data());
        if (!check(cudaGetLastError(), "tuning frame")) return AVBD_ERR_RUNTIME_FAILURE;
        frame++;
        if (!check(cudaStreamSynchronize(launch), "tuning frame")) return AVBD_ERR_RUNTIME_FAILURE;
        uint32_t k = 0;
        for (uint32_t it = 0; it < P.iterations; it++)
            for (uint32_t c = 0; c < colorBound; c++) {
                if (H.colorCounts[c] == 0) continue;
                float ms = 0.0f;
                if (!check(cudaEventElapsedTime(&ms, tuneEvents[2 * k], tuneEvents[2 * k + 1]), "tuning timing"))
                    return AVBD_ERR_RUNTIME_FAILURE;
                tuneMs[tuneStage][c] += ms;
                k++;
            }
        if (++tuneStage == kTuneVariants) {
            for (uint32_t c = 0; c < colorBound; c++) {
                int best = 0;
                for (int w = 1; w < kTuneVariants; w++) if (tuneMs[w][c] < tuneMs[best][c]) best = w;
                H.colorLanes[c] = kTuneWidths[best];
            }
            tuneStage = -1;
            graphsValid = false;
        }
        return AVBD_OK;
    }

    // Block-shape autotuner of the dynamic-coloring primal (rigid scenes,
    // batched worlds).  Its grid-stride launch gives every body to one 8-lane
    // group whatever the grid, so each candidate computes the same floats;
    // only speed differs, and that depends on how many bodies a color holds.
    // The first solver of a body-count bucket (floor(log2(dynamic bodies)))
    // on a device times one eager frame per candidate, with events around
    // every primal launch, and keeps the fastest; later solvers of the
    // bucket reuse it.
    struct DynShape { uint32_t blocksPerSM, threads; };
    static constexpr DynShape kDynShapes[7] = {{1, 128}, {2, 128}, {3, 128}, {4, 128}, {4, 64}, {6, 64}, {8, 64}};
    int dynTuneStage = -1;
    double dynTuneMs[7] = {};
    uint32_t dynBucket = 0, dynCandidates = 0;
    static std::mutex& dyn_cache_mutex() { static std::mutex m; return m; }
    static std::map<std::pair<int, uint32_t>, std::pair<uint32_t, uint32_t>>& dyn_cache() {
        static std::map<std::pair<int, uint32_t>, std::pair<uint32_t, uint32_t>> c;
        return c;
    }
    void dyn_tune_setup() {
        z.dynBlocks = 148u * 4u;
        z.dynThreads = 128u;
        if (!z.dynamicColoring || smallSolve || z.numDynamicBodies == 0) return;
        uint32_t b = 0;
        while ((2u << b) <= z.numDynamicBodies) b++;
        dynBucket = b;
        std::lock_guard<std::mutex> lock(dyn_cache_mutex());
        auto it = dyn_cache().find({device, b});
        if (it != dyn_cache().end()) {
            z.dynBlocks = it->second.first;
            z.dynThreads = it->second.second;
            return;
        }
        dynTuneStage = 0;
    }
    int dyn_tune_frame() {
        const DynShape sh = kDynShapes[dynTuneStage];
        z.dynBlocks = 148u * sh.blocksPerSM;
        z.dynThreads = sh.threads;
        const size_t need = 2 * (size_t)P.iterations * (colorLaunchBound + 1);
        while (tuneEvents.size() < need) {
            cudaEvent_t e;
            if (!check(cudaEventCreate(&e), "event create")) return AVBD_ERR_RUNTIME_FAILURE;
            tuneEvents.push_back(e);
        }
        const uint32_t launches = P.iterations * colorLaunchBound;
        encode_frame_on((int)(frame & 1), launch, nullptr, tuneEvents.data());
        if (!check(cudaGetLastError(), "tuning frame")) return AVBD_ERR_RUNTIME_FAILURE;
        frame++;
        if (!check(cudaStreamSynchronize(launch), "tuning frame")) return AVBD_ERR_RUNTIME_FAILURE;
        double total = 0.0;
        for (uint32_t k = 0; k < launches; k++) {
            float ms = 0.0f;
            if (!check(cudaEventElapsedTime(&ms, tuneEvents[2 * k], tuneEvents[2 * k + 1]), "tuning timing"))
                return AVBD_ERR_RUNTIME_FAILURE;
            total += ms;
        }
        dynTuneMs[dynTuneStage] = total;
        if (++dynTuneStage == 7) {
            int best = 3;   // the untuned default wins ties
            for (int k = 0; k < 7; k++) if (dynTuneMs[k] < dynTuneMs[best]) best = k;
            z.dynBlocks = 148u * kDynShapes[best].blocksPerSM;
            z.dynThreads = kDynShapes[best].threads;
            dynCandidates = 7;
            {
                std::lock_guard<std::mutex> lock(dyn_cache_mutex());
                dyn_cache()[{device, dynBucket}] = {z.dynBlocks, z.dynThreads};
            }
            dynTuneStage = -1;
            graphsValid = false;
        }
        return AVBD_OK;
    }

    int step(uint32_t frames) {
        if (failure != AVBD_FAIL_NONE) return AVBD_ERR_RUNTIME_FAILURE;
        uint32_t f = 0;
        while (tuneStage >= 0 && f < frames) {
            int rc = tune_frame();
            if (rc != AVBD_OK) return rc;
            f++;
        }
        while (dynTuneStage >= 0 && f < frames) {
            int rc = dyn_tune_frame();
            if (rc != AVBD_OK) return rc;
            f++;
        }
        if (f == frames) return AVBD_OK;
        if (!graphsValid && !build_graphs()) return AVBD_ERR_RUNTIME_FAILURE;
        for (; f < frames; f++) {
            if (!check(cudaGraphLaunch(graph[frame & 1], launch), "graph launch")) return AVBD_ERR_RUNTIME_FAILURE;
            frame++;
            if (profiling) {
                // profiled frames retire synchronously, as in the reference
                int rc = retire();
                if (rc != AVBD_OK) return rc;
                for (int k = 0; k + 1 < usedEvents; k++) {
                    float ms = 0.0f;
                    if (!check(cudaEventElapsedTime(&ms, events[k], events[k + 1]), "event timing")) return AVBD_ERR_RUNTIME_FAILURE;
                    const int stg = intervalStage[k];
                    if (stg >= 0) { prof.stage_ms[stg] += ms; prof.stage_launches[stg] += 1; }
                }
                prof.frames++;
            }
        }
        return AVBD_OK;
    }

    void* staging(size_t bytes) {
        if (bytes > stageBytes) {
            if (stage) cudaFree(stage);
            stage = nullptr;
            stageBytes = 0;
            if (cudaMalloc(&stage, bytes) != cudaSuccess) return nullptr;
            stageBytes = bytes;
        }
        return stage;
    }
};

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int avbd_create(const avbd_scene_desc* scene, avbd_solver** out) {
    if (!out) return AVBD_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    avbd_solver* s = nullptr;
    try {
        s = new avbd_solver();
        int rc = s->create(scene);
        if (rc != AVBD_OK) {
            g_last_error = s->error;
            delete s;
            return rc;
        }
    } catch (const std::exception& e) {
        g_last_error = e.what();
        delete s;
        return AVBD_ERR_ALLOC_FAILED;
    }
    g_last_error.clear();
    *out = s;
    return AVBD_OK;
}

// Batched worlds (vector environments): ragged body ranges packed in one
// scene, one collision group per world (RL/PushTEnv.swift:137-180).
int avbd_create_batched(const avbd_scene_desc* scene, const uint32_t* world_offsets, uint32_t num_worlds,
                        avbd_solver** out) {
    if (!out) return AVBD_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    auto fail = [](const char* msg) { g_last_error = msg; return AVBD_ERR_INVALID_ARGUMENT; };
    if (!scene || (num_worlds && !world_offsets)) return fail("avbd_create_batched: null scene or offsets");
    const uint32_t nb = scene->num_bodies;
    for (uint32_t w = 0; w < num_worlds; w++)
        if (world_offsets[w] > world_offsets[w + 1]) return fail("avbd_create_batched: world offsets must not decrease");
    if (num_worlds && world_offsets[num_worlds] > nb) return fail("avbd_create_batched: world offsets beyond the bodies");
    // world of every body (0xFFFFFFFF = shared)
    std::vector<uint32_t> worldOf(nb, 0xFFFFFFFFu);
    for (uint32_t w = 0; w < num_worlds; w++)
        for (uint32_t b = world_offsets[w]; b < world_offsets[w + 1]; b++) worldOf[b] = w;
    auto world_of = [&](int32_t b) { return (b < 0 || (uint32_t)b >= nb) ? 0xFFFFFFFFu : worldOf[b]; };
    auto joins_two = [&](const int32_t* ids, int n) {
        uint32_t seen = 0xFFFFFFFFu;
        for (int k = 0; k < n; k++) {
            const uint32_t w = world_of(ids[k]);
            if (w == 0xFFFFFFFFu) continue;
            if (seen != 0xFFFFFFFFu && seen != w) return true;
            seen = w;
        }
        return false;
    };
    for (uint32_t i = 0; i < scene->num_joints; i++) {
        const int32_t ids[2] = {scene->joints[i].body_a, scene->joints[i].body_b};
        if (joins_two(ids, 2)) return fail("avbd_create_batched: a joint joins two worlds");
    }
    for (uint32_t i = 0; i < scene->num_springs; i++) {
        const int32_t ids[2] = {scene->springs[i].body_a, scene->springs[i].body_b};
        if (joins_two(ids, 2)) return fail("avbd_create_batched: a spring joins two worlds");
    }
    for (uint32_t i = 0; i < scene->num_tets; i++)
        if (joins_two(scene->tets[i].ids, 4)) return fail("avbd_create_batched: a tet joins two worlds");
    for (uint32_t i = 0; i < scene->num_tris; i++)
        if (joins_two(scene->tris[i].ids, 3)) return fail("avbd_create_batched: a triangle joins two worlds");
    for (uint32_t i = 0; i < scene->num_exclusions; i++) {
        const int32_t ids[2] = {scene->exclusions[i].body_a, scene->exclusions[i].body_b};
        if (joins_two(ids, 2)) return fail("avbd_create_batched: an exclusion joins two worlds");
    }
    std::vector<avbd_collider_desc> cols(scene->colliders, scene->colliders + scene->num_colliders);
    for (avbd_collider_desc& c : cols) {
        const uint32_t w = world_of(c.body);
        c.collision_group = w == 0xFFFFFFFFu ? 0u : w + 1u;
    }
    avbd_scene_desc desc = *scene;
    desc.colliders = cols.data();
    avbd_solver* s = nullptr;
    int rc = avbd_create(&desc, &s);
    if (rc != AVBD_OK) return rc;
    s->worldOffsets.assign(world_offsets, world_offsets + num_worlds + (num_worlds ? 1 : 0));
    s->initialStates.resize(nb);
    for (uint32_t b = 0; b < nb; b++) {
        const avbd_body_desc& bd = scene->bodies[b];
        avbd_body_state& st = s->initialStates[b];
        std::memcpy(st.position, bd.position, sizeof st.position);
        std::memcpy(st.rotation, bd.rotation, sizeof st.rotation);
        std::memcpy(st.velocity, bd.velocity, sizeof st.velocity);
        st.angular_velocity[0] = st.angular_velocity[1] = st.angular_velocity[2] = 0.0f;
    }
    s->worldMotors.assign(num_worlds, {});
    s->initialMotorTargets.resize(s->H.joints.size());
    for (uint32_t j = 0; j < s->H.joints.size(); j++) {
        s->initialMotorTargets[j] = s->H.joints[j].motor.x;
        if ((s->H.joints[j].header.w & MOTOR_MODE_MASK) == 0u) continue;
        const uint32_t w = world_of((int32_t)s->H.joints[j].header.y);
        if (w != 0xFFFFFFFFu) s->worldMotors[w].push_back(j);
    }
    *out = s;
    return AVBD_OK;
}

int avbd_get_world_offsets(avbd_solver* s, uint32_t* num_worlds, uint32_t* offsets) {
    if (!s || !num_worlds) return AVBD_ERR_INVALID_ARGUMENT;
    *num_worlds = s->worldOffsets.empty() ? 0u : (uint32_t)s->worldOffsets.size() - 1u;
    if (offsets) std::copy(s->worldOffsets.begin(), s->worldOffsets.end(), offsets);
    return AVBD_OK;
}

int avbd_set_world_body_states(avbd_solver* s, uint32_t world, const uint32_t* local_ids, uint32_t n,
                               const avbd_body_state* states) {
    const uint32_t nw = !s || s->worldOffsets.empty() ? 0u : (uint32_t)s->worldOffsets.size() - 1u;
    if (!s || world >= nw || (n && (!local_ids || !states))) return AVBD_ERR_INVALID_ARGUMENT;
    const uint32_t first = s->worldOffsets[world], size = s->worldOffsets[world + 1] - first;
    std::vector<uint32_t> ids(n);
    for (uint32_t i = 0; i < n; i++) {
        if (local_ids[i] >= size) return AVBD_ERR_INVALID_ARGUMENT;
        ids[i] = first + local_ids[i];
    }
    return avbd_set_body_states(s, ids.data(), n, states);
}

int avbd_reset_worlds(avbd_solver* s, const uint32_t* worlds, uint32_t n) {
    if (!s || (n && !worlds)) return AVBD_ERR_INVALID_ARGUMENT;
    const uint32_t nw = s->worldOffsets.empty() ? 0u : (uint32_t)s->worldOffsets.size() - 1u;
    std::vector<uint32_t> ids, motors, velMotors;
    std::vector<avbd_body_state> states;
    std::vector<float> targets, velTargets;
    for (uint32_t i = 0; i < n; i++) {
        const uint32_t w = worlds[i];
        if (w >= nw) return AVBD_ERR_INVALID_ARGUMENT;
        for (uint32_t b = s->worldOffsets[w]; b < s->worldOffsets[w + 1]; b++) {
            ids.push_back(b);
            states.push_back(s->initialStates[b]);
        }
        for (uint32_t j : s->worldMotors[w]) {
            const bool velocity = (s->H.joints[j].header.w & MOTOR_MODE_MASK) == MOTOR_VELOCITY;
            (velocity ? velMotors : motors).push_back(j);
            (velocity ? velTargets : targets).push_back(s->initialMotorTargets[j]);
        }
    }
    if (ids.empty()) return AVBD_OK;
    int rc = avbd_set_body_states(s, ids.data(), (uint32_t)ids.size(), states.data());
    if (rc != AVBD_OK) return rc;
    if (!motors.empty()) rc = avbd_set_motor_targets(s, motors.data(), (uint32_t)motors.size(), targets.data());
    if (rc == AVBD_OK && !velMotors.empty())
        rc = avbd_set_motor_velocities(s, velMotors.data(), (uint32_t)velMotors.size(), velTargets.data());
    return rc;
}

int avbd_get_world_motor_joints(avbd_solver* s, uint32_t world, uint32_t* ids, uint32_t cap, uint32_t* count) {
    if (!s || !count || world >= s->worldMotors.size() || (cap && !ids)) return AVBD_ERR_INVALID_ARGUMENT;
    const std::vector<uint32_t>& m = s->worldMotors[world];
    *count = (uint32_t)m.size();
    for (uint32_t i = 0; i < cap && i < m.size(); i++) ids[i] = m[i];
    return AVBD_OK;
}

void avbd_destroy(avbd_solver* s) { delete s; }

int avbd_set_settings(avbd_solver* s, const avbd_settings* st) {
    if (!s || !st) return AVBD_ERR_INVALID_ARGUMENT;
    if (s->failure != AVBD_FAIL_NONE) return AVBD_ERR_RUNTIME_FAILURE;
    if (!(st->dt > 0.0f) || st->iterations < 0) return AVBD_ERR_INVALID_ARGUMENT;
    s->settings = *st;
    s->sync_params();
    s->graphsValid = false;   // parameters are baked into the frame graphs
    return AVBD_OK;
}

int avbd_get_settings(const avbd_solver* s, avbd_settings* out) {
    if (!s || !out) return AVBD_ERR_INVALID_ARGUMENT;
    *out = s->settings;
    return AVBD_OK;
}

int avbd_step(avbd_solver* s, uint32_t frames) {
    if (!s) return AVBD_ERR_INVALID_ARGUMENT;
    return s->step(frames);
}

int avbd_sync(avbd_solver* s) {
    if (!s) return AVBD_ERR_INVALID_ARGUMENT;
    return s->retire();
}

int avbd_get_positions(avbd_solver* s, uint32_t n, float* pos, float* rot) {
    if (!s || n > s->z.numBodies) return AVBD_ERR_INVALID_ARGUMENT;
    int rc = s->retire();
    if (rc != AVBD_OK) return rc;
    if (pos && !s->check(cudaMemcpy(pos, s->d.posLin, (size_t)n * 16, cudaMemcpyDeviceToHost), "position readback")) return AVBD_ERR_RUNTIME_FAILURE;
    if (rot && !s->check(cudaMemcpy(rot, s->d.posAng, (size_t)n * 16, cudaMemcpyDeviceToHost), "rotation readback")) return AVBD_ERR_RUNTIME_FAILURE;
    return AVBD_OK;
}

int avbd_get_body_states(avbd_solver* s, const uint32_t* ids, uint32_t n, avbd_body_state* out) {
    if (!s || !out) return AVBD_ERR_INVALID_ARGUMENT;
    const uint32_t nb = s->z.numBodies;
    if (!ids && n > nb) return AVBD_ERR_INVALID_ARGUMENT;
    for (uint32_t i = 0; ids && i < n; i++) if (ids[i] >= nb) return AVBD_ERR_INVALID_ARGUMENT;
    int rc = s->retire();
    if (rc != AVBD_OK) return rc;
    std::vector<float4> pl(nb), pa(nb), vl(nb), va(nb);
    if (!s->check(cudaMemcpy(pl.data(), s->d.posLin, nb * 16, cudaMemcpyDeviceToHost), "state readback") ||
        !s->check(cudaMemcpy(pa.data(), s->d.posAng, nb * 16, cudaMemcpyDeviceToHost), "state readback") ||
        !s->check(cudaMemcpy(vl.data(), s->d.velLin, nb * 16, cudaMemcpyDeviceToHost), "state readback") ||
        !s->check(cudaMemcpy(va.data(), s->d.velAng, nb * 16, cudaMemcpyDeviceToHost), "state readback"))
        return AVBD_ERR_RUNTIME_FAILURE;
    for (uint32_t i = 0; i < n; i++) {
        const uint32_t b = ids ? ids[i] : i;
        avbd_body_state& o = out[i];
        o.position[0] = pl[b].x; o.position[1] = pl[b].y; o.position[2] = pl[b].z;
        o.rotation[0] = pa[b].x; o.rotation[1] = pa[b].y; o.rotation[2] = pa[b].z; o.rotation[3] = pa[b].w;
        o.velocity[0] = vl[b].x; o.velocity[1] = vl[b].y; o.velocity[2] = vl[b].z;
        o.angular_velocity[0] = va[b].x; o.angular_velocity[1] = va[b].y; o.angular_velocity[2] = va[b].z;
    }
    return AVBD_OK;
}

int avbd_set_body_states(avbd_solver* s, const uint32_t* ids, uint32_t n, const avbd_body_state* states) {
    if (!s || (!states && n)) return AVBD_ERR_INVALID_ARGUMENT;
    if (n == 0) return AVBD_OK;
    const uint32_t nb = s->z.numBodies;
    if (!ids && n > nb) return AVBD_ERR_INVALID_ARGUMENT;
    for (uint32_t i = 0; ids && i < n; i++) if (ids[i] >= nb) return AVBD_ERR_INVALID_ARGUMENT;
    int rc = s->retire();
    if (rc != AVBD_OK) return rc;
    const size_t bytesStates = sizeof(avbd_body_state) * n, bytesIds = ids ? 4 * (size_t)n : 0;
    uint8_t* st = static_cast<uint8_t*>(s->staging(bytesStates + bytesIds + 16));
    if (!st) return AVBD_ERR_ALLOC_FAILED;
    uint32_t* dIds = ids ? reinterpret_cast<uint32_t*>(st + bytesStates) : nullptr;
    if (!s->check(cudaMemcpyAsync(st, states, bytesStates, cudaMemcpyHostToDevice, s->launch), "state upload")) return AVBD_ERR_RUNTIME_FAILURE;
    if (ids && !s->check(cudaMemcpyAsync(dIds, ids, bytesIds, cudaMemcpyHostToDevice, s->launch), "state upload")) return AVBD_ERR_RUNTIME_FAILURE;
    cudaMemsetAsync(s->d.resetFlags, 0, 4 * (size_t)nb, s->launch);
    k_set_states<<<(n + 127) / 128, 128, 0, s->launch>>>(s->d, dIds, reinterpret_cast<const avbd_body_state*>(st), n);
    launch_reset_bodies(s->P, s->d, s->z, s->launch);
    return s->retire();
}

int avbd_set_positions(avbd_solver* s, uint32_t n, const float* xyz) {
    if (!s || !xyz || n > s->z.numBodies) return AVBD_ERR_INVALID_ARGUMENT;
    if (s->failure != AVBD_FAIL_NONE) return AVBD_ERR_RUNTIME_FAILURE;
    float* st = static_cast<float*>(s->staging((size_t)n * 12 + 16));
    if (!st) return AVBD_ERR_ALLOC_FAILED;
    if (!s->check(cudaMemcpyAsync(st, xyz, (size_t)n * 12, cudaMemcpyHostToDevice, s->launch), "position upload")) return AVBD_ERR_RUNTIME_FAILURE;
    k_set_positions<<<(n + 255) / 256, 256, 0, s->launch>>>(s->d.posLin, st, n);
    return s->check(cudaGetLastError(), "position upload") ? AVBD_OK : AVBD_ERR_RUNTIME_FAILURE;
}

int avbd_set_motor_targets(avbd_solver* s, const uint32_t* joints, uint32_t n, const float* targets) {
    if (!s || (n && (!joints || !targets))) return AVBD_ERR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < n; i++) {
        if (joints[i] >= s->H.joints.size() || !std::isfinite(targets[i])) return AVBD_ERR_INVALID_ARGUMENT;
        uint32_t mode = s->H.joints[joints[i]].header.w & MOTOR_MODE_MASK;
        if (mode == MOTOR_VELOCITY) return AVBD_ERR_INVALID_ARGUMENT;  // requires a position-PD motor
    }
    if (n == 0) return AVBD_OK;
    if (s->failure != AVBD_FAIL_NONE) return AVBD_ERR_RUNTIME_FAILURE;
    uint8_t* st = static_cast<uint8_t*>(s->staging(8 * (size_t)n + 16));
    if (!st) return AVBD_ERR_ALLOC_FAILED;
    cudaMemcpyAsync(st, joints, 4 * (size_t)n, cudaMemcpyHostToDevice, s->launch);
    cudaMemcpyAsync(st + 4 * (size_t)n, targets, 4 * (size_t)n, cudaMemcpyHostToDevice, s->launch);
    k_set_motor_targets<<<(n + 127) / 128, 128, 0, s->launch>>>(s->d.joints, reinterpret_cast<uint32_t*>(st),
                                                                 reinterpret_cast<float*>(st + 4 * (size_t)n), n);
    return s->check(cudaGetLastError(), "motor targets") ? AVBD_OK : AVBD_ERR_RUNTIME_FAILURE;
}

namespace {
// Copies ids and n * width floats into staging and launches one setter.
int joint_update(avbd_solver* s, const uint32_t* joints, uint32_t n, const float* vals, int width, int which,
                 const char* label) {
    if (n == 0) return AVBD_OK;
    if (s->failure != AVBD_FAIL_NONE) return AVBD_ERR_RUNTIME_FAILURE;
    const size_t idBytes = 4 * (size_t)n, valBytes = 4 * (size_t)n * width;
    const size_t valOff = (idBytes + 15) & ~(size_t)15;
    uint8_t* st = static_cast<uint8_t*>(s->staging(valOff + valBytes + 16));
    if (!st) return AVBD_ERR_ALLOC_FAILED;
    cudaMemcpyAsync(st, joints, idBytes, cudaMemcpyHostToDevice, s->launch);
    cudaMemcpyAsync(st + valOff, vals, valBytes, cudaMemcpyHostToDevice, s->launch);
    const uint32_t* ids = reinterpret_cast<uint32_t*>(st);
    const float* v = reinterpret_cast<float*>(st + valOff);
    if (which == 0) k_set_joint_anchors<<<(n + 127) / 128, 128, 0, s->launch>>>(s->d.joints, ids, v, n);
    else k_set_motor_field<<<(n + 127) / 128, 128, 0, s->launch>>>(s->d.joints, ids, v, n, which == 2 ? 1 : 0);
    return s->check(cudaGetLastError(), label) ? AVBD_OK : AVBD_ERR_RUNTIME_FAILURE;
}
}  // namespace

int avbd_set_joint_world_anchors(avbd_solver* s, const uint32_t* joints, uint32_t n, const float* points_xyz) {
    if (!s || (n && (!joints || !points_xyz))) return AVBD_ERR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < n; i++) {
        if (joints[i] >= s->H.joints.size()) return AVBD_ERR_INVALID_ARGUMENT;
        for (int k = 0; k < 3; k++)
            if (!std::isfinite(points_xyz[3 * i + k])) return AVBD_ERR_INVALID_ARGUMENT;
    }
    return joint_update(s, joints, n, points_xyz, 3, 0, "joint anchors");
}

int avbd_set_motor_velocities(avbd_solver* s, const uint32_t* joints, uint32_t n, const float* rad_per_s) {
    if (!s || (n && (!joints || !rad_per_s))) return AVBD_ERR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < n; i++) {
        if (joints[i] >= s->H.joints.size() || !std::isfinite(rad_per_s[i])) return AVBD_ERR_INVALID_ARGUMENT;
        if ((s->H.joints[joints[i]].header.w & MOTOR_MODE_MASK) != MOTOR_VELOCITY) return AVBD_ERR_INVALID_ARGUMENT;
    }
    return joint_update(s, joints, n, rad_per_s, 1, 1, "motor velocities");
}

int avbd_set_motor_torques(avbd_solver* s, const uint32_t* joints, uint32_t n, const float* torques) {
    if (!s || (n && (!joints || !torques))) return AVBD_ERR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < n; i++) {
        if (joints[i] >= s->H.joints.size() || !std::isfinite(torques[i]) || torques[i] < 0.0f) return AVBD_ERR_INVALID_ARGUMENT;
        const JointGPU& j = s->H.joints[joints[i]];
        if ((j.header.w & MOTOR_MODE_MASK) == 0) return AVBD_ERR_INVALID_ARGUMENT;  // no authored motor
        // a joint authored with zero stiffness and zero effort is never
        // solved (no stage reads it); raising its effort is not supported
        if (j.rA.w == 0.0f && j.rB.w == 0.0f && j.motor.y == 0.0f && torques[i] > 0.0f) return AVBD_ERR_UNSUPPORTED;
    }
    return joint_update(s, joints, n, torques, 1, 2, "motor torques");
}

int avbd_get_motor_states(avbd_solver* s, const uint32_t* joints, uint32_t n, float* angles, float* velocities) {
    if (!s || (n && (!joints || !angles || !velocities))) return AVBD_ERR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < n; i++)
        if (joints[i] >= s->H.joints.size()) return AVBD_ERR_INVALID_ARGUMENT;
    if (n == 0) return AVBD_OK;
    int rc = s->retire();
    if (rc != AVBD_OK) return rc;
    const size_t idBytes = ((4 * (size_t)n) + 15) & ~(size_t)15;
    uint8_t* st = static_cast<uint8_t*>(s->staging(idBytes + 8 * (size_t)n + 16));
    if (!st) return AVBD_ERR_ALLOC_FAILED;
    float* dOut = reinterpret_cast<float*>(st + idBytes);
    cudaMemcpyAsync(st, joints, 4 * (size_t)n, cudaMemcpyHostToDevice, s->launch);
    k_motor_states<<<(n + 127) / 128, 128, 0, s->launch>>>(s->d.joints, s->d.posAng, s->d.velAng,
                                                           reinterpret_cast<uint32_t*>(st), n, dOut);
    std::vector<float> out(2 * (size_t)n);
    if (!s->check(cudaGetLastError(), "motor states") ||
        !s->check(cudaMemcpyAsync(out.data(), dOut, 8 * (size_t)n, cudaMemcpyDeviceToHost, s->launch), "motor states readback") ||
        !s->check(cudaStreamSynchronize(s->launch), "motor states"))
        return AVBD_ERR_RUNTIME_FAILURE;
    for (uint32_t i = 0; i < n; i++) { angles[i] = out[2 * i]; velocities[i] = out[2 * i + 1]; }
    return AVBD_OK;
}

// ---------------------------------------------------------------------------
// Headless render and observation compute (render.cu)
// ---------------------------------------------------------------------------
namespace {
// Staging layout: `in` bytes of inputs, then (host output only) `out` bytes.
uint8_t* render_staging(avbd_solver* s, size_t in, size_t out, size_t& outOff) {
    outOff = (in + 255) & ~(size_t)255;
    return static_cast<uint8_t*>(s->staging(outOff + out + 16));
}
// Goal heading of a Push-T environment: cos and sin of the yaw, evaluated in
// double and rounded once.
void goal_heading(float yaw, float& c, float& s) {
    c = (float)std::cos((double)yaw);
    s = (float)std::sin((double)yaw);
}

// Rest normal (unit, +z when zero) and rest inverse of a skin binding; a
// zero inverse becomes the inverse of the four bodies' scene-pose edge
// matrix [d0 d1 d2] (rows cross(d1,d2), cross(d2,d0), cross(d0,d1) over the
// determinant; the identity when it is singular), GPUSolver.swift:1866-1896.
void skin_rest_frame(const avbd_skin_binding& g, const std::vector<f4>& pos, SkinBinding& o) {
    const float* rn = g.rest_normal;
    const float l2 = rn[0] * rn[0] + rn[1] * rn[1] + rn[2] * rn[2];
    if (l2 > 1e-12f) {
        const float l = std::sqrt(l2);
        o.restNormal = make_float4(rn[0] / l, rn[1] / l, rn[2] / l, 0.0f);
    } else {
        o.restNormal = make_float4(0.0f, 0.0f, 1.0f, 0.0f);
    }
    auto sq = [](const float* v) { return v[0] * v[0] + v[1] * v[1] + v[2] * v[2]; };
    if (sq(g.inv0) + sq(g.inv1) + sq(g.inv2) > 1e-16f) {
        o.inv0 = make_float4(g.inv0[0], g.inv0[1], g.inv0[2], 0.0f);
        o.inv1 = make_float4(g.inv1[0], g.inv1[1], g.inv1[2], 0.0f);
        o.inv2 = make_float4(g.inv2[0], g.inv2[1], g.inv2[2], 0.0f);
        return;
    }
    auto P = [&](uint32_t i) { return std::array<float, 3>{pos[i].x, pos[i].y, pos[i].z}; };
    auto sub3 = [](std::array<float, 3> a, std::array<float, 3> b) {
        return std::array<float, 3>{a[0] - b[0], a[1] - b[1], a[2] - b[2]};
    };
    auto crs = [](std::array<float, 3> a, std::array<float, 3> b) {
        return std::array<float, 3>{a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
    };
    const auto x0 = P(g.ids[0]);
    const auto d0 = sub3(P(g.ids[1]), x0), d1 = sub3(P(g.ids[2]), x0), d2 = sub3(P(g.ids[3]), x0);
    const auto r0 = crs(d1, d2), r1 = crs(d2, d0), r2 = crs(d0, d1);
    const float det = d0[0] * r0[0] + d0[1] * r0[1] + d0[2] * r0[2];
    if (std::fabs(det) > 1e-12f) {
        o.inv0 = make_float4(r0[0] / det, r0[1] / det, r0[2] / det, 0.0f);
        o.inv1 = make_float4(r1[0] / det, r1[1] / det, r1[2] / det, 0.0f);
        o.inv2 = make_float4(r2[0] / det, r2[1] / det, r2[2] / det, 0.0f);
    } else {
        o.inv0 = make_float4(1.0f, 0.0f, 0.0f, 0.0f);
        o.inv1 = make_float4(0.0f, 1.0f, 0.0f, 0.0f);
        o.inv2 = make_float4(0.0f, 0.0f, 1.0f, 0.0f);
    }
}

// Host output: copy back and wait; device output: return at once.
int render_finish(avbd_solver* s, void* hostOut, const void* devOut, size_t bytes, const char* label) {
    if (!s->check(cudaGetLastError(), label)) return AVBD_ERR_RUNTIME_FAILURE;
    if (hostOut) {
        if (!s->check(cudaMemcpyAsync(hostOut, devOut, bytes, cudaMemcpyDeviceToHost, s->launch), label) ||
            !s->check(cudaStreamSynchronize(s->launch), label))
            return AVBD_ERR_RUNTIME_FAILURE;
    }
    return AVBD_OK;
}
}  // namespace

int avbd_build_instances(avbd_solver* s, const uint32_t* colliders, uint32_t n, const float* colors_rgba,
                         uint32_t color_mode, avbd_render_instance* out, int out_on_device) {
    if (!s || (n && (!colliders || !out)) || color_mode > 1) return AVBD_ERR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < n; i++)
        if (colliders[i] >= s->H.numColliders) return AVBD_ERR_INVALID_ARGUMENT;
    if (s->failure != AVBD_FAIL_NONE) return AVBD_ERR_RUNTIME_FAILURE;
    if (n == 0) return AVBD_OK;
    const size_t idBytes = ((4 * (size_t)n) + 15) & ~(size_t)15, colBytes = colors_rgba ? 16 * (size_t)n : 0;
    const size_t outBytes = sizeof(avbd_render_instance) * (size_t)n;
    size_t outOff;
    uint8_t* st = render_staging(s, idBytes + colBytes, out_on_device ? 0 : outBytes, outOff);
    if (!st) return AVBD_ERR_ALLOC_FAILED;
    cudaMemcpyAsync(st, colliders, 4 * (size_t)n, cudaMemcpyHostToDevice, s->launch);
    if (colors_rgba) cudaMemcpyAsync(st + idBytes, colors_rgba, colBytes, cudaMemcpyHostToDevice, s->launch);
    float* dOut = out_on_device ? reinterpret_cast<float*>(out) : reinterpret_cast<float*>(st + outOff);
    launch_build_instances(s->d, reinterpret_cast<uint32_t*>(st),
                           colors_rgba ? reinterpret_cast<float4*>(st + idBytes) : nullptr, n, color_mode, dOut,
                           s->launch);
    return render_finish(s, out_on_device ? nullptr : out, dOut, outBytes, "build instances");
}

int avbd_soft_normals(avbd_solver* s, float cloth_scale, float* out, int out_on_device) {
    if (!s || !out || !std::isfinite(cloth_scale)) return AVBD_ERR_INVALID_ARGUMENT;
    if (s->failure != AVBD_FAIL_NONE) return AVBD_ERR_RUNTIME_FAILURE;
    const uint32_t nt = s->H.numTris, nb = s->H.numBodies;
    if (nt == 0) return AVBD_OK;
    if (!s->renderSurfaceReady) {
        // vertex -> incident surface triangles, vertices ascending, triangles
        // in surface order (GPUSolver.swift:1812-1842)
        std::vector<uint32_t> cnt(nb, 0);
        for (const u4& t : s->H.tris) { cnt[t.x]++; cnt[t.y]++; cnt[t.z]++; }
        std::vector<uint32_t> verts, start, count, list, pos(nb, 0);
        for (uint32_t v = 0; v < nb; v++)
            if (cnt[v]) { verts.push_back(v); start.push_back((uint32_t)list.size()); count.push_back(cnt[v]); pos[v] = (uint32_t)list.size(); list.resize(list.size() + cnt[v]); }
        for (uint32_t t = 0; t < nt; t++) {
            const u4 tr = s->H.tris[t];
            for (uint32_t v : {tr.x, tr.y, tr.z}) list[pos[v]++] = t;
        }
        std::vector<uint32_t> cloth = s->H.clothVert;
        cloth.resize(nb, 0);
        bool ok = s->upload(s->surfVerts, verts, "surfaceVertices") && s->upload(s->surfVtStart, start, "surfaceVtStart") &&
                  s->upload(s->surfVtCount, count, "surfaceVtCount") && s->upload(s->surfVtList, list, "surfaceVtList") &&
                  s->upload(s->surfClothVert, cloth, "surfaceClothVert") &&
                  s->alloc(s->faceNormals, nt, "faceNormals");
        if (!ok) return AVBD_ERR_ALLOC_FAILED;
        s->numSurfVerts = (uint32_t)verts.size();
        s->renderSurfaceReady = true;
    }
    const size_t outBytes = 16 * (size_t)nb;
    size_t outOff;
    uint8_t* st = render_staging(s, 0, out_on_device ? 0 : outBytes, outOff);
    if (!st) return AVBD_ERR_ALLOC_FAILED;
    float4* dOut = out_on_device ? reinterpret_cast<float4*>(out) : reinterpret_cast<float4*>(st + outOff);
    if (!out_on_device) cudaMemcpyAsync(dOut, out, outBytes, cudaMemcpyHostToDevice, s->launch);  // untouched entries
    DevPtrs d = s->d;
    d.clothVert = s->surfClothVert;
    launch_soft_normals(d, nt, s->surfVerts, s->surfVtStart, s->surfVtCount, s->surfVtList, s->numSurfVerts,
                        s->faceNormals, cloth_scale, dOut, s->launch);
    return render_finish(s, out_on_device ? nullptr : out, dOut, outBytes, "soft normals");
}

int avbd_set_skin_bindings(avbd_solver* s, const avbd_skin_binding* b, uint32_t n) {
    if (!s || (n && !b)) return AVBD_ERR_INVALID_ARGUMENT;
    const uint32_t nb = s->H.numBodies;
    std::vector<SkinBinding> host(n);
    for (uint32_t i = 0; i < n; i++) {
        const avbd_skin_binding& g = b[i];
        for (int k = 0; k < 4; k++)
            if (g.ids[k] >= nb) return AVBD_ERR_INVALID_ARGUMENT;
        SkinBinding& o = host[i];
        o.ids = make_uint4(g.ids[0], g.ids[1], g.ids[2], g.ids[3]);
        o.weights = make_float4(g.weights[0], g.weights[1], g.weights[2], g.weights[3]);
        skin_rest_frame(g, s->H.posLin, o);
    }
    if (s->launch) cudaStreamSynchronize(s->launch);
    if (s->skin) { cudaFree(s->skin); s->skin = nullptr; }
    s->numSkin = 0;
    if (n == 0) return AVBD_OK;
    if (cudaMalloc(&s->skin, sizeof(SkinBinding) * (size_t)n) != cudaSuccess) return AVBD_ERR_ALLOC_FAILED;
    if (cudaMemcpy(s->skin, host.data(), sizeof(SkinBinding) * (size_t)n, cudaMemcpyHostToDevice) != cudaSuccess)
        return AVBD_ERR_ALLOC_FAILED;
    s->numSkin = n;
    return AVBD_OK;
}

int avbd_skin_deform(avbd_solver* s, float* out, int out_on_device) {
    if (!s || !out) return AVBD_ERR_INVALID_ARGUMENT;
    if (s->failure != AVBD_FAIL_NONE) return AVBD_ERR_RUNTIME_FAILURE;
    if (s->numSkin == 0) return AVBD_OK;
    const size_t outBytes = 32 * (size_t)s->numSkin;
    size_t outOff;
    uint8_t* st = render_staging(s, 0, out_on_device ? 0 : outBytes, outOff);
    if (!st) return AVBD_ERR_ALLOC_FAILED;
    float4* dOut = out_on_device ? reinterpret_cast<float4*>(out) : reinterpret_cast<float4*>(st + outOff);
    launch_skin_deform(s->d.posLin, s->skin, s->numSkin, dOut, s->launch);
    return render_finish(s, out_on_device ? nullptr : out, dOut, outBytes, "skin deform");
}

int avbd_render_pusht_obs(avbd_solver* s, const avbd_pusht_env* envs, uint32_t num_envs, uint32_t res,
                          uint8_t* out, int out_on_device) {
    if (!s || (num_envs && (!envs || !out)) || res < 2 || res > 4096) return AVBD_ERR_INVALID_ARGUMENT;
    if (out_on_device && (res % 4u == 0u) && (reinterpret_cast<uintptr_t>(out) & 15u)) return AVBD_ERR_INVALID_ARGUMENT;
    if (s->failure != AVBD_FAIL_NONE) return AVBD_ERR_RUNTIME_FAILURE;
    if (num_envs == 0) return AVBD_OK;
    const bool same = s->pushtHost.size() == num_envs &&
                      std::memcmp(s->pushtHost.data(), envs, sizeof(avbd_pusht_env) * (size_t)num_envs) == 0;
    if (!same) {
        const uint32_t nb = s->H.numBodies;
        std::vector<PushTDev> table(num_envs);
        for (uint32_t e = 0; e < num_envs; e++) {
            const avbd_pusht_env& v = envs[e];
            for (int k = 0; k < 3; k++)
                if (v.ids[k] >= nb) return AVBD_ERR_INVALID_ARGUMENT;
            PushTDev& t = table[e];
            t.ids = make_uint4(v.ids[0], v.ids[1], v.ids[2], v.ids[3]);
            t.frame = make_float4(v.frame[0], v.frame[1], v.frame[2], v.frame[3]);
            t.goalYaw = v.goal[0];
            t.halfWin = v.goal[1];
            goal_heading(v.goal[0], t.goalCos, t.goalSin);
        }
        // earlier observation launches may still read the old table
        if (!s->check(cudaStreamSynchronize(s->launch), "Push-T table")) return AVBD_ERR_RUNTIME_FAILURE;
        if (num_envs > s->pushtCap) {
            if (s->pushtDev) cudaFree(s->pushtDev);
            if (s->pushtShapes) cudaFree(s->pushtShapes);
            s->pushtDev = nullptr;
            s->pushtShapes = nullptr;
            s->pushtCap = 0;
            if (cudaMalloc(&s->pushtDev, sizeof(PushTDev) * (size_t)num_envs) != cudaSuccess ||
                cudaMalloc(&s->pushtShapes, 6 * sizeof(float4) * (size_t)num_envs) != cudaSuccess)
                return AVBD_ERR_ALLOC_FAILED;
            s->pushtCap = num_envs;
        }
        if (!s->check(cudaMemcpy(s->pushtDev, table.data(), sizeof(PushTDev) * (size_t)num_envs,
                                 cudaMemcpyHostToDevice), "Push-T table"))
            return AVBD_ERR_RUNTIME_FAILURE;
        s->pushtHost.assign(envs, envs + num_envs);
    }
    const size_t outBytes = (size_t)num_envs * res * res * 3;
    size_t outOff = 0;
    uint8_t* st = out_on_device ? nullptr : render_staging(s, 0, outBytes, outOff);
    if (!out_on_device && !st) return AVBD_ERR_ALLOC_FAILED;
    uint8_t* dOut = out_on_device ? out : st + outOff;
    launch_pusht_obs(s->d.posLin, s->d.posAng, s->pushtDev, num_envs, res, s->pushtShapes, dOut, s->launch);
    return render_finish(s, out_on_device ? nullptr : out, dOut, outBytes, "Push-T observation");
}

int avbd_max_constraint_error(avbd_solver* s, float* out) {
    if (!s || !out) return AVBD_ERR_INVALID_ARGUMENT;
    int rc = s->retire();
    if (rc != AVBD_OK) return rc;
    DevPtrs f = s->d;
    if (s->frame & 1) std::swap(f.manifolds, f.prevManifolds);
    launch_max_constraint_error(s->P, f, s->z, s->launch);
    if (!s->check(cudaMemcpyAsync(out, s->d.diag, 4, cudaMemcpyDeviceToHost, s->launch), "diag readback")) return AVBD_ERR_RUNTIME_FAILURE;
    return s->retire();
}

int avbd_get_counters(avbd_solver* s, avbd_counters* out) {
    if (!s || !out) return AVBD_ERR_INVALID_ARGUMENT;
    int rc = s->retire();
    if (rc != AVBD_OK && rc != AVBD_ERR_RUNTIME_FAILURE) return rc;
    Counters c{};
    cudaMemcpy(&c, s->d.counters, sizeof(Counters), cudaMemcpyDeviceToHost);
    std::memset(out, 0, sizeof(*out));
    out->frame = s->frame;
    out->num_pairs = c.numPairs;
    out->pair_candidates = c.pairCandidates;
    out->color_conflicts = c.colorConflicts;
    out->ogc_exceeded = c.ogcExceeded;
    if (s->z.dynamicColoring) {
        out->used_colors = c.usedColors;
        for (int i = 0; i < 64; i++) out->color_counts[i] = c.colorCount[i];
    } else {
        out->used_colors = s->H.staticUsedColors;
        for (int i = 0; i < 64; i++) out->color_counts[i] = s->H.colorCounts[i];
    }
    out->num_soft = c.numSoft;
    out->soft_candidates = c.softRaw;
    out->dat_pairs = c.datPairsPeak;
    out->dat_vt_pairs = c.datVTPeak;
    out->dat_ee_pairs = c.datEEPeak;
    out->dat_grid_overflows = c.datGridOverflow;
    out->dat_invalid_anchors = c.datInvalidAnchor;
    out->dat_truncations = c.datTruncations;
    out->dat_vt_degenerate = c.datVTDegenerate;
    out->dat_ee_degenerate = c.datEEDegenerate;
    out->dat_nonfinite = c.datNonfinite;
    out->dat_tet_degenerate = c.datTetDegenerate;
    uint32_t accepted = 0;
    if (s->d.learnAccepted) cudaMemcpy(&accepted, s->d.learnAccepted, 4, cudaMemcpyDeviceToHost);
    out->learn_accepted = accepted;
    if (s->P.ogc) {
        out->soft_rt = c.numSoftRT;
        out->soft_vt = c.numSoftVT;
        out->soft_ee = c.numSoftEE;
    }
    return AVBD_OK;
}

int avbd_set_warm_start_model(avbd_solver* s, const float* params, const float* norm, uint32_t trial_sweeps) {
    if (!s || !params || !norm || trial_sweeps > 16) return AVBD_ERR_INVALID_ARGUMENT;
    if (s->z.numLearnAll == 0) {
        s->error = "the scene has no dynamic bodies for the learned warm start (cloth is not supported)";
        return AVBD_ERR_UNSUPPORTED;
    }
    int rc = s->retire();
    if (rc != AVBD_OK) return rc;
    const DevPtrs& d = s->d;
    if (!s->check(cudaMemcpy(d.learnPrm, params, sizeof(float) * mlp_param_count(), cudaMemcpyHostToDevice), "model upload") ||
        !s->check(cudaMemcpy(d.learnNorm, norm, sizeof(float) * mlp_norm_count(), cudaMemcpyHostToDevice), "model upload"))
        return AVBD_ERR_RUNTIME_FAILURE;
    launch_mlp_mirror(d.learnPrm, d.learnHalf, s->launch);
    if (!s->check(cudaStreamSynchronize(s->launch), "model upload")) return AVBD_ERR_RUNTIME_FAILURE;
    s->modelSet = true;
    s->learnTrials = trial_sweeps;
    s->graphsValid = false;
    return AVBD_OK;
}

int avbd_set_warm_start_mode(avbd_solver* s, int mode) {
    if (!s || (mode != AVBD_WARM_START_PLAIN && mode != AVBD_WARM_START_LEARNED)) return AVBD_ERR_INVALID_ARGUMENT;
    if (mode == AVBD_WARM_START_LEARNED && !s->modelSet) {
        s->error = "no warm-start model: call avbd_set_warm_start_model first";
        return AVBD_ERR_INVALID_ARGUMENT;
    }
    if (mode == AVBD_WARM_START_LEARNED && s->z.numLearn == 0) {
        s->error = "the learned rows cover no body of this scene (rigid bodies need avbd_set_warm_start_rigid)";
        return AVBD_ERR_UNSUPPORTED;
    }
    s->learnMode = mode;
    s->update_small_solve();
    s->graphsValid = false;
    return AVBD_OK;
}

int avbd_set_learning_capture(avbd_solver* s, int enabled) {
    if (!s) return AVBD_ERR_INVALID_ARGUMENT;
    if (enabled && s->z.numLearn == 0) {
        s->error = "the learned rows cover no body of this scene (rigid bodies need avbd_set_warm_start_rigid)";
        return AVBD_ERR_UNSUPPORTED;
    }
    s->learnCapture = enabled != 0;
    s->update_small_solve();
    s->graphsValid = false;
    return AVBD_OK;
}

int avbd_set_warm_start_rigid(avbd_solver* s, int enabled) {
    if (!s) return AVBD_ERR_INVALID_ARGUMENT;
    if (s->z.numLearnAll == 0) {
        s->error = "the scene has no dynamic bodies for the learned warm start (cloth is not supported)";
        return AVBD_ERR_UNSUPPORTED;
    }
    int rc = s->retire();
    if (rc != AVBD_OK) return rc;
    s->P.learnRigid = enabled ? 1u : 0u;
    s->z.numLearn = enabled ? s->z.numLearnAll : s->P.learnParticles;
    if (s->z.numLearn == 0) {    // a rigid-only scene without rigid rows: learning and the learned mode stop
        s->learnCapture = false;
        if (s->learnMode == AVBD_WARM_START_LEARNED) s->learnMode = AVBD_WARM_START_PLAIN;
    }
    s->update_small_solve();
    s->graphsValid = false;
    return AVBD_OK;
}

int avbd_set_residual_trace(avbd_solver* s, int enabled) {
    if (!s) return AVBD_ERR_INVALID_ARGUMENT;
    s->residualTrace = enabled != 0;
    s->update_small_solve();
    s->graphsValid = false;
    return AVBD_OK;
}

int avbd_get_residual_trace(avbd_solver* s, double* out, uint32_t n) {
    if (!s || !out) return AVBD_ERR_INVALID_ARGUMENT;
    int rc = s->retire();
    if (rc != AVBD_OK) return rc;
    const uint32_t len = std::min<uint32_t>(n, avbd_solver::kTraceLength);
    std::vector<double> sq(len);
    if (!s->check(cudaMemcpy(sq.data(), s->d.learnTrace, sizeof(double) * len, cudaMemcpyDeviceToHost), "trace readback"))
        return AVBD_ERR_RUNTIME_FAILURE;
    for (uint32_t i = 0; i < len; i++) out[i] = std::sqrt(sq[i]);
    return AVBD_OK;
}

int avbd_runtime_failure(const avbd_solver* s, int* kind) {
    if (!s || !kind) return AVBD_ERR_INVALID_ARGUMENT;
    *kind = s->failure;
    return AVBD_OK;
}

int avbd_last_error(const avbd_solver* s, char* buf, size_t len) {
    if (!buf || len == 0) return AVBD_ERR_INVALID_ARGUMENT;
    const std::string& e = s ? s->error : g_last_error;
    std::snprintf(buf, len, "%s", e.c_str());
    return AVBD_OK;
}

int avbd_snapshot_capture(avbd_solver* s, avbd_snapshot** out) {
    if (!s || !out) return AVBD_ERR_INVALID_ARGUMENT;
    int rc = s->retire();
    if (rc != AVBD_OK) return rc;
    avbd_snapshot* snap = new avbd_snapshot();
    snap->frame = s->frame;
    for (const auto& b : s->state) {
        snap->blobs.emplace_back(b.bytes);
        if (!s->check(cudaMemcpy(snap->blobs.back().data(), b.ptr, b.bytes, cudaMemcpyDeviceToHost), "snapshot")) {
            delete snap;
            return AVBD_ERR_RUNTIME_FAILURE;
        }
    }
    *out = snap;
    return AVBD_OK;
}

int avbd_snapshot_restore(avbd_solver* s, const avbd_snapshot* snap) {
    if (!s || !snap || snap->blobs.size() != s->state.size()) return AVBD_ERR_INVALID_ARGUMENT;
    int rc = s->retire();
    if (rc != AVBD_OK) return rc;
    for (size_t i = 0; i < s->state.size(); i++)
        if (!s->check(cudaMemcpy(s->state[i].ptr, snap->blobs[i].data(), s->state[i].bytes, cudaMemcpyHostToDevice), "restore"))
            return AVBD_ERR_RUNTIME_FAILURE;
    s->frame = snap->frame;
    return AVBD_OK;
}

void avbd_snapshot_free(avbd_snapshot* snap) { delete snap; }

int avbd_set_stream(avbd_solver* s, void* cuda_stream) {
    if (!s) return AVBD_ERR_INVALID_ARGUMENT;
    if (!s->check(cudaStreamSynchronize(s->launch), "stream switch")) return AVBD_ERR_RUNTIME_FAILURE;
    s->launch = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : s->stream;
    return AVBD_OK;
}

int avbd_set_capacity_for_testing(avbd_solver* s, int which, uint32_t value) {
    if (!s) return AVBD_ERR_INVALID_ARGUMENT;
    int rc = s->retire();
    if (rc != AVBD_OK) return rc;
    if (which == AVBD_CAPACITY_SOFT_CONTACTS) s->P.maxSoft = std::min(value, s->z.maxSoft);
    else if (which == AVBD_CAPACITY_PLANAR_DAT_PAIRS) s->P.maxDatPairs = std::min(value, s->H.maxDatPairs);
    else return AVBD_ERR_INVALID_ARGUMENT;
    s->graphsValid = false;   // capacities are baked into the frame graphs
    return AVBD_OK;
}

int avbd_set_profiling(avbd_solver* s, int enabled) {
    if (!s) return AVBD_ERR_INVALID_ARGUMENT;
    int rc = s->retire();
    if (rc != AVBD_OK) return rc;
    if ((enabled != 0) != s->profiling) {
        s->profiling = enabled != 0;
        s->graphsValid = false;
    }
    std::memset(&s->prof, 0, sizeof(s->prof));
    return AVBD_OK;
}

int avbd_set_primal_variant(avbd_solver* s, uint32_t variant) {
    if (!s) return AVBD_ERR_INVALID_ARGUMENT;
    if (variant != 0 && variant != AVBD_PRIMAL_STAGED && variant != 8 && variant != 16 && variant != 32)
        return AVBD_ERR_INVALID_ARGUMENT;
    int rc = s->retire();
    if (rc != AVBD_OK) return rc;
    if (variant == 0) {
        s->tuneStage = s->tuning_applies() ? 0 : -1;
        std::memset(s->tuneMs, 0, sizeof(s->tuneMs));
    } else {
        s->tuneStage = -1;
        for (auto& l : s->H.colorLanes) l = variant;
    }
    s->graphsValid = false;
    return AVBD_OK;
}

int avbd_get_profile(avbd_solver* s, avbd_profile* out) {
    if (!s || !out) return AVBD_ERR_INVALID_ARGUMENT;
    if (!s->graphsValid && !s->build_graphs()) return AVBD_ERR_RUNTIME_FAILURE;
    *out = s->prof;
    out->kernels_per_frame = s->kernelsPerFrame;
    for (int c = 0; c < 64; c++) out->color_lanes[c] = s->H.colorLanes[c];
    out->dyn_blocks = s->z.dynamicColoring ? s->z.dynBlocks : 0u;
    out->dyn_threads = s->z.dynamicColoring ? s->z.dynThreads : 0u;
    out->dyn_bucket = s->dynBucket;
    out->dyn_candidates = s->dynCandidates;
    return AVBD_OK;
}

size_t avbd_debug_buffer_size(avbd_solver* s, int which) {
    if (!s) return 0;
    const HostScene& H = s->H;
    const size_t nb = H.numBodies;
    switch (which) {
    case AVBD_BUF_POS_LIN: case AVBD_BUF_POS_ANG: case AVBD_BUF_VEL_LIN: case AVBD_BUF_VEL_ANG:
    case AVBD_BUF_INIT_LIN: case AVBD_BUF_INERT_LIN: return nb * 16;
    case AVBD_BUF_PAIRS: case AVBD_BUF_MANIFOLDS: case AVBD_BUF_ADJ_LIST: {
        Counters c{};
        cudaStreamSynchronize(s->launch);
        cudaMemcpy(&c, s->d.counters, sizeof(Counters), cudaMemcpyDeviceToHost);
        if (which == AVBD_BUF_PAIRS) return (size_t)c.numPairs * 8;
        if (which == AVBD_BUF_MANIFOLDS) return (size_t)c.numPairs * sizeof(ManifoldGPU);
        std::vector<uint32_t> dc(nb);
        cudaMemcpy(dc.data(), s->d.dynCount, 4 * nb, cudaMemcpyDeviceToHost);
        size_t total = 0;
        for (size_t b = 0; b < nb; b++) total += H.staticSeg[b].y + H.staticSeg[b].w + dc[b];
        return total * 4;
    }
    case AVBD_BUF_ADJ_START: case AVBD_BUF_ADJ_COUNT: case AVBD_BUF_COLORS: return nb * 4;
    case AVBD_BUF_COLOR_START: return (MAX_COLORS + 2) * 4;
    case AVBD_BUF_COLOR_LIST: return (size_t)H.numDynamicBodies * 4;
    case AVBD_BUF_CELL_START: case AVBD_BUF_CELL_COUNT: return (size_t)H.gridHashSize * 4;
    case AVBD_BUF_CELL_BODIES: return H.hashedIdx.size() * 4;
    case AVBD_BUF_MAP_KEY_A: case AVBD_BUF_MAP_KEY_B: case AVBD_BUF_MAP_VAL: return (size_t)H.mapCapacity * 4;
    case AVBD_BUF_JOINTS: return H.joints.size() * sizeof(JointGPU);
    case AVBD_BUF_SPRINGS: return H.springs.size() * sizeof(SpringGPU);
    case AVBD_BUF_TETS: return H.tets.size() * sizeof(TetGPU);
    case AVBD_BUF_EXCLUSIONS: return H.exclusions.size() * 4;
    case AVBD_BUF_HASHED_IDX: return H.hashedIdx.size() * 4;
    case AVBD_BUF_GLOBAL_IDX: return H.globalIdx.size() * 4;
    case AVBD_BUF_TRIS: return H.tris.size() * 16;
    case AVBD_BUF_EDGES: return H.edges.size() * 4;
    case AVBD_BUF_NBR_START: return H.nbrStart.size() * 4;
    case AVBD_BUF_NBR_COUNT: return H.nbrCount.size() * 4;
    case AVBD_BUF_NBR_LIST: return H.nbrList.size() * 4;
    case AVBD_BUF_PARTICLE_IDX: return H.numTris ? (size_t)s->P.numParticles * 4 : 0;
    case AVBD_BUF_MEMBRANES: return H.membranes.size() * sizeof(MembraneGPU);
    case AVBD_BUF_BENDS: return H.bends.size() * sizeof(BendGPU);
    case AVBD_BUF_CLOTH_GROUP: return nb * 4;
    case AVBD_BUF_OGC_PREV: return (s->P.cloth || s->P.ogc) ? nb * 16 : 0;
    case AVBD_BUF_LEARN_IDX: return (size_t)s->z.numLearn * 4;
    case AVBD_BUF_LEARN_FEATURES: return (size_t)s->z.numLearn * 128;
    case AVBD_BUF_LEARN_TARGETS: case AVBD_BUF_LEARN_PREDICTIONS: return (size_t)s->z.numLearn * 24;
    case AVBD_BUF_SOFT: case AVBD_BUF_DAT_PAIRS: {
        if (!s->P.cloth && !(s->P.ogc && which == AVBD_BUF_SOFT)) return 0;
        Counters c{};
        cudaStreamSynchronize(s->launch);
        cudaMemcpy(&c, s->d.counters, sizeof(Counters), cudaMemcpyDeviceToHost);
        return which == AVBD_BUF_SOFT ? (size_t)c.numSoft * sizeof(SoftContactGPU) : (size_t)c.datStored * 16;
    }
    default: return 0;
    }
}

int avbd_debug_read(avbd_solver* s, int which, void* dst, size_t bytes) {
    if (!s || !dst) return AVBD_ERR_INVALID_ARGUMENT;
    if (bytes > avbd_debug_buffer_size(s, which)) return AVBD_ERR_INVALID_ARGUMENT;
    if (!s->check(cudaStreamSynchronize(s->launch), "debug read")) return AVBD_ERR_RUNTIME_FAILURE;
    const DevPtrs& d = s->d;
    const HostScene& H = s->H;
    const size_t nb = H.numBodies;
    // the manifolds written by the last frame live in the buffer that is
    // "previous" for the next frame
    const bool odd = (s->frame & 1) != 0;
    const void* src = nullptr;
    switch (which) {
    case AVBD_BUF_POS_LIN: src = d.posLin; break;
    case AVBD_BUF_POS_ANG: src = d.posAng; break;
    case AVBD_BUF_VEL_LIN: src = d.velLin; break;
    case AVBD_BUF_VEL_ANG: src = d.velAng; break;
    case AVBD_BUF_INIT_LIN: src = d.initLin; break;
    case AVBD_BUF_INERT_LIN: src = d.inertLin; break;
    case AVBD_BUF_PAIRS: src = d.pairs; break;
    case AVBD_BUF_MANIFOLDS: src = odd ? d.manifolds : d.prevManifolds; break;
    case AVBD_BUF_COLORS: src = d.colorsA; break;
    case AVBD_BUF_COLOR_START: src = d.colorStart; break;
    case AVBD_BUF_COLOR_LIST: src = d.colorList; break;
    case AVBD_BUF_CELL_START: src = d.cellStart; break;
    case AVBD_BUF_CELL_COUNT: src = d.cellCount; break;
    case AVBD_BUF_CELL_BODIES: src = d.cellBodies; break;
    case AVBD_BUF_MAP_KEY_A: src = d.mapKeyA; break;
    case AVBD_BUF_MAP_KEY_B: src = d.mapKeyB; break;
    case AVBD_BUF_MAP_VAL: src = d.mapVal; break;
    case AVBD_BUF_JOINTS: src = d.joints; break;
    case AVBD_BUF_SPRINGS: src = d.springs; break;
    case AVBD_BUF_TETS: src = d.tets; break;
    case AVBD_BUF_EXCLUSIONS: src = d.exclusions; break;
    case AVBD_BUF_HASHED_IDX: src = d.hashedIdx; break;
    case AVBD_BUF_GLOBAL_IDX: src = d.globalIdx; break;
    case AVBD_BUF_TRIS: src = d.tris; break;
    case AVBD_BUF_EDGES: src = d.edges; break;
    case AVBD_BUF_NBR_START: src = d.nbrStart; break;
    case AVBD_BUF_NBR_COUNT: src = d.nbrCount; break;
    case AVBD_BUF_NBR_LIST: src = d.nbrList; break;
    case AVBD_BUF_PARTICLE_IDX: src = d.particleIdx; break;
    case AVBD_BUF_MEMBRANES: src = d.membranes; break;
    case AVBD_BUF_BENDS: src = d.bends; break;
    case AVBD_BUF_CLOTH_GROUP: src = d.clothGroup; break;
    case AVBD_BUF_OGC_PREV: src = d.ogcPrev; break;
    // element contacts swap like the manifolds
    case AVBD_BUF_SOFT: src = odd ? d.soft : d.prevSoft; break;
    case AVBD_BUF_DAT_PAIRS: src = d.datPairs; break;
    case AVBD_BUF_LEARN_IDX: src = d.learnIdx; break;
    case AVBD_BUF_LEARN_FEATURES: src = d.learnFeat; break;
    case AVBD_BUF_LEARN_TARGETS: src = d.learnTarget; break;
    case AVBD_BUF_LEARN_PREDICTIONS: src = d.learnPred; break;
    case AVBD_BUF_ADJ_START: case AVBD_BUF_ADJ_COUNT: case AVBD_BUF_ADJ_LIST: {
        // materialise the merged (pre, contacts, post) lists
        std::vector<uint32_t> dc(nb), ds(nb);
        std::vector<uint32_t> dl(2 * (size_t)H.maxPairs + ((s->P.cloth || s->P.ogc) ? 4 * (size_t)s->P.maxSoft : 0));
        cudaMemcpy(dc.data(), d.dynCount, 4 * nb, cudaMemcpyDeviceToHost);
        cudaMemcpy(ds.data(), d.dynStart, 4 * nb, cudaMemcpyDeviceToHost);
        cudaMemcpy(dl.data(), d.dynList, 4 * dl.size(), cudaMemcpyDeviceToHost);
        std::vector<uint32_t> dsp(nb);
        cudaMemcpy(dsp.data(), d.dynSplit, 4 * nb, cudaMemcpyDeviceToHost);
        std::vector<uint32_t> start(nb), count(nb), list;
        for (size_t b = 0; b < nb; b++) {
            // pre, manifolds, tets, element contacts, membranes and bends
            const u4 sg = H.staticSeg[b];
            const uint32_t pt = H.postTets[b];
            start[b] = (uint32_t)list.size();
            count[b] = sg.y + dc[b] + sg.w;
            list.insert(list.end(), H.preList.begin() + sg.x, H.preList.begin() + sg.x + sg.y);
            list.insert(list.end(), dl.begin() + ds[b], dl.begin() + ds[b] + dsp[b]);
            list.insert(list.end(), H.postList.begin() + sg.z, H.postList.begin() + sg.z + pt);
            list.insert(list.end(), dl.begin() + ds[b] + dsp[b], dl.begin() + ds[b] + dc[b]);
            list.insert(list.end(), H.postList.begin() + sg.z + pt, H.postList.begin() + sg.z + sg.w);
        }
        const std::vector<uint32_t>& v = which == AVBD_BUF_ADJ_START ? start : (which == AVBD_BUF_ADJ_COUNT ? count : list);
        std::memcpy(dst, v.data(), bytes);
        return AVBD_OK;
    }
    default: return AVBD_ERR_INVALID_ARGUMENT;
    }
    if (!src) return AVBD_ERR_INVALID_ARGUMENT;
    return s->check(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost), "debug read") ? AVBD_OK : AVBD_ERR_RUNTIME_FAILURE;
}

}  // extern "C"
