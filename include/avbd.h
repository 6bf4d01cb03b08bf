/*
 * avbd.h — C ABI of the B200 AVBD solver step.
 *
 * This is the drop-in boundary for the reference's `GPUSolver` class
 * (Sources/PhysicsAVBD/GPU/GPUSolver.swift:17) and the scene description it
 * is built from (`PhysicsScene`, Sources/SimCore/Scenes/Scene.swift:547).
 * Every entry point returns an `int` status (AVBD_OK on success) and never
 * unwinds across the ABI.  All arguments are plain C types: pointers, sizes
 * and the POD records below.  No CUDA or torch type appears here.
 *
 * Threading: one solver instance is driven by one host thread at a time, as
 * the reference's caller is (GPUSolver.swift:2219-2222).
 */
#ifndef AVBD_H
#define AVBD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AVBD_ABI_VERSION 3u

/* ------------------------------------------------------------------------ */
/* Status codes.  Construction errors mirror `AVBDError`                     */
/* (GPUSolver.swift:640-661); runtime errors mirror `RuntimeFailure`         */
/* (GPUSolver.swift:663-751) and are latched: once a runtime failure is      */
/* recorded every later call on that solver returns AVBD_ERR_RUNTIME_FAILURE */
/* until it is destroyed (GPUSolver.swift:2800-2809).                        */
/* ------------------------------------------------------------------------ */
enum {
    AVBD_OK = 0,
    AVBD_ERR_INVALID_ARGUMENT = 1,   /* bad pointer, index or size           */
    AVBD_ERR_NO_DEVICE = 2,          /* AVBDError.noDevice                   */
    AVBD_ERR_ALLOC_FAILED = 3,       /* AVBDError.allocFailed(label)         */
    AVBD_ERR_KERNEL_MISSING = 4,     /* AVBDError.kernelMissing(name)        */
    AVBD_ERR_RUNTIME_FAILURE = 5,    /* latched RuntimeFailure, see below    */
    AVBD_ERR_UNSUPPORTED = 6         /* scene feature outside this library   */
};

/* Runtime failure kinds reported by avbd_runtime_failure(). */
enum {
    AVBD_FAIL_NONE = 0,
    AVBD_FAIL_COMMAND_EXECUTION = 1,   /* CUDA error on the solver stream    */
    AVBD_FAIL_RIGID_PAIR_CAPACITY = 2, /* broadphase demand > maxPairs       */
    AVBD_FAIL_SOFT_CONTACT_CAPACITY = 3,
    AVBD_FAIL_STATIC_COLOR_CAPACITY = 4,
    AVBD_FAIL_UNRESOLVED_COLORING = 5,
    /* Planar-DAT codes 1-3 (GPUSolver.swift:676-751) */
    AVBD_FAIL_PLANAR_DAT_PAIR_CAPACITY = 6,  /* V-T/E-E pair demand > capacity */
    AVBD_FAIL_PLANAR_DAT_GRID_SPAN = 7,      /* element AABB > 4 cells/axis   */
    AVBD_FAIL_PLANAR_DAT_INVALID_ANCHOR = 8, /* coincident/non-finite anchor  */
    AVBD_FAIL_WAIT_TIMEOUT = 9         /* bounded device wait gave up        */
};

/* Body shape kinds (BodyShape, Scene.swift:6-11). */
enum { AVBD_SHAPE_BOX = 0, AVBD_SHAPE_SPHERE = 1, AVBD_SHAPE_TORUS = 2,
       AVBD_SHAPE_CAPSULE = 3 };

/* Joint motor modes (JointMotorMode, Scene.swift:193-204). */
enum { AVBD_MOTOR_IMPLICIT_POSITION_PD = 0, AVBD_MOTOR_EXPLICIT_TORQUE_PD = 1,
       AVBD_MOTOR_VELOCITY = 2 };

/* Surface truncation selection (GPUSolver.swift:23-35). */
enum { AVBD_TRUNCATION_AUTOMATIC = 0, AVBD_TRUNCATION_ISOTROPIC = 1,
       AVBD_TRUNCATION_PLANAR_DAT = 2 };

/* SimSettings (Scene.swift:485-545); render-only fields are omitted. */
typedef struct avbd_settings {
    float dt;
    float gravity;                 /* along z; negative pulls down            */
    int32_t iterations;
    float collision_margin;
    uint32_t friction_combine_mode; /* 0 geometric .. 4 average               */
    float alpha;
    float beta_lin;
    float beta_ang;
    float gamma;
    float lambda_max;
    float rod_decay_pow;
    float particle_damping;
    float rigid_linear_damping;
    float rigid_angular_damping;
    float cloth_viscosity;
} avbd_settings;

/* SceneBody (Scene.swift:34-105). rotation is (x, y, z, w). */
typedef struct avbd_body_desc {
    float size[3];
    float density;                 /* 0 = static unless explicit mass > 0    */
    float friction;
    float dynamic_friction;
    float position[3];
    float rotation[4];
    float velocity[3];
    uint32_t shape;                /* AVBD_SHAPE_*                            */
    uint32_t is_particle;          /* 3-DOF particle (Scene.swift:57)         */
    uint32_t has_explicit_mass;    /* mass/diagonal_inertia authoritative     */
    float mass;
    float diagonal_inertia[3];
    float gravity_scale;
} avbd_body_desc;

/* SceneCollider (Scene.swift:114-186). */
typedef struct avbd_collider_desc {
    int32_t body;
    float size[3];
    float friction;
    float dynamic_friction;
    float local_position[3];
    float local_rotation[4];
    uint32_t shape;
    uint32_t collision_group;
    uint32_t collides_with_shared;
    uint32_t collision_enabled;
    uint32_t world_round_anchor;   /* usesWorldSpaceRoundAnchor              */
    uint32_t hull_offset;          /* into avbd_scene_desc.hull_vertices     */
    uint32_t hull_count;           /* 0 = analytic shape                     */
} avbd_collider_desc;

/* SceneJoint (Scene.swift:206-315). Infinite stiffness = hard constraint. */
typedef struct avbd_joint_desc {
    int32_t body_a;                /* -1 = world                             */
    int32_t body_b;
    float r_a[3];
    float r_b[3];
    float stiffness_lin;
    float stiffness_ang;
    float fracture;
    uint32_t fracture_linear;
    uint32_t has_hinge;
    float hinge_axis[3];           /* body-B local, unit                     */
    float motor_target;
    float motor_torque;
    float motor_rate;
    float motor_stiffness;
    float motor_damping;
    uint32_t motor_mode;           /* AVBD_MOTOR_*                            */
    float armature;
    float limit_lo;
    float limit_hi;
} avbd_joint_desc;

/* SceneSpring (Scene.swift:433-454). rest < 0: use spawn distance. */
typedef struct avbd_spring_desc {
    int32_t body_a;
    int32_t body_b;
    float r_a[3];
    float r_b[3];
    float stiffness;
    float rest;
    uint32_t hard;
} avbd_spring_desc;

/* SceneTet (Scene.swift:337-360). */
typedef struct avbd_tet_desc {
    int32_t ids[4];
    float mu;
    float lambda;
    uint32_t self_collision;
} avbd_tet_desc;

/* SceneTri (Scene.swift:321-334). */
typedef struct avbd_tri_desc {
    int32_t ids[3];
    float mu;
    float lambda;
    float bend;
} avbd_tri_desc;

/* SceneCollisionExclusion (Scene.swift:474-483). */
typedef struct avbd_exclusion_desc {
    int32_t body_a;
    int32_t body_b;
} avbd_exclusion_desc;

/* SceneSpinner (Scene.swift:459-469). */
typedef struct avbd_spinner_desc {
    int32_t body;
    float axis[3];
    float omega;
} avbd_spinner_desc;

/* PhysicsScene + GPUSolver construction options. */
typedef struct avbd_scene_desc {
    uint32_t abi_version;          /* must be AVBD_ABI_VERSION               */
    uint32_t num_bodies;
    const avbd_body_desc* bodies;
    uint32_t num_colliders;
    const avbd_collider_desc* colliders;
    uint32_t num_hull_vertices;
    const float* hull_vertices;    /* xyz triples                            */
    uint32_t num_joints;
    const avbd_joint_desc* joints;
    uint32_t num_springs;
    const avbd_spring_desc* springs;
    uint32_t num_tets;
    const avbd_tet_desc* tets;
    uint32_t num_tris;
    const avbd_tri_desc* tris;
    uint32_t num_exclusions;
    const avbd_exclusion_desc* exclusions;
    uint32_t num_spinners;
    const avbd_spinner_desc* spinners;
    avbd_settings settings;
    uint32_t max_pairs_per_body;   /* GPUSolver init default 16              */
    uint32_t truncation_selection; /* AVBD_TRUNCATION_*                       */
    uint32_t tet_inversion_prevention;
    int32_t device;                /* CUDA ordinal; -1 = current device      */
} avbd_scene_desc;

/* One body's kinematic state (bodyStates / BodyStateUpdate,
 * GPUSolver.swift:2399-2479, :4431-4486). rotation is (x, y, z, w). */
typedef struct avbd_body_state {
    float position[3];
    float rotation[4];
    float velocity[3];
    float angular_velocity[3];
} avbd_body_state;

/* Frame diagnostics (GPUSolver.swift:313-328). */
typedef struct avbd_counters {
    uint64_t frame;
    uint32_t num_pairs;
    uint32_t pair_candidates;
    uint32_t num_soft;
    uint32_t soft_candidates;
    uint32_t used_colors;
    uint32_t color_conflicts;
    uint32_t ogc_exceeded;
    uint32_t color_counts[64];
    /* Planar-DAT statistics of the last retired frame (lastPlanarDAT*,
     * GPUSolver.swift:318-325)                                             */
    uint32_t dat_pairs;
    uint32_t dat_vt_pairs;
    uint32_t dat_ee_pairs;
    uint32_t dat_grid_overflows;
    uint32_t dat_invalid_anchors;
    uint32_t dat_truncations;
    uint32_t dat_vt_degenerate;
    uint32_t dat_ee_degenerate;
    uint32_t dat_nonfinite;
    uint32_t dat_tet_degenerate;
    uint32_t learn_accepted;      /* frames whose predicted warm start was kept */
    /* isotropic-OGC element contacts of the last retired frame: rigid-
     * triangle, vertex-triangle and edge-edge records (rt_emit, vt_emit,
     * ee_emit, 25_cloth.metal:347-1142)                                    */
    uint32_t soft_rt;
    uint32_t soft_vt;
    uint32_t soft_ee;
} avbd_counters;

typedef struct avbd_solver avbd_solver;
typedef struct avbd_snapshot avbd_snapshot;

/* Build a solver from a scene.  Replaces `GPUSolver.init(scene:device:
 * maxPairsPerBody:)` (GPUSolver.swift:331-336, upload :901-2081).        */
int avbd_create(const avbd_scene_desc* scene, avbd_solver** out);

/* Release every device buffer owned by the solver. */
void avbd_destroy(avbd_solver* solver);

/* Replace the per-frame settings (`GPUSolver.settings`, GPUSolver.swift:45,
 * mirrored into SimParams by syncParams :2097-2142).                        */
int avbd_set_settings(avbd_solver* solver, const avbd_settings* settings);
int avbd_get_settings(const avbd_solver* solver, avbd_settings* out);

/* Encode and submit `frames` physics frames asynchronously (`submitStep`,
 * GPUSolver.swift:3107-3136).  Errors latched during execution surface on
 * the next call or at avbd_sync.                                           */
int avbd_step(avbd_solver* solver, uint32_t frames);

/* Wait for every submitted frame and retire its counters (`synchronize`,
 * GPUSolver.swift:2924-2953).                                              */
int avbd_sync(avbd_solver* solver);

/* Read `n` body states by index (`bodyStates`, GPUSolver.swift:4471).
 * ids == NULL reads bodies [0, n).  Synchronises first.                   */
int avbd_get_body_states(avbd_solver* solver, const uint32_t* ids, uint32_t n,
                         avbd_body_state* out);

/* Overwrite `n` body states (`setBodyStates`, GPUSolver.swift:2409-2473):
 * clears the augmented-Lagrangian state of every incident joint, spring and
 * contact and restores the initial joint penalties.  ids == NULL writes
 * bodies [0, n).                                                          */
int avbd_set_body_states(avbd_solver* solver, const uint32_t* ids, uint32_t n,
                         const avbd_body_state* states);

/* Bulk position/orientation readback: xyzw position (w = mass) and xyzw
 * quaternion for bodies [0, n).  Either output may be NULL.                */
int avbd_get_positions(avbd_solver* solver, uint32_t n, float* pos_xyzw,
                       float* rot_xyzw);

/* Bulk position upload for bodies [0, n) from xyz triples, keeping the
 * velocity and the augmented-Lagrangian state (used to replay host input). */
int avbd_set_positions(avbd_solver* solver, uint32_t n, const float* pos_xyz);

/* Motor targets for hinge joints (`setMotorTargets`,
 * GPUSolver.swift:2496-2521).                                             */
int avbd_set_motor_targets(avbd_solver* solver, const uint32_t* joints,
                           uint32_t n, const float* targets);

/* World anchor of each listed joint (its rA, the world point of a joint to
 * the world) from xyz triples (`setJointWorldAnchors`,
 * GPUSolver.swift:2481-2494).                                             */
int avbd_set_joint_world_anchors(avbd_solver* solver, const uint32_t* joints,
                                 uint32_t n, const float* points_xyz);

/* Commands of velocity motors in rad/s (`setMotorVelocities`,
 * GPUSolver.swift:2534-2551); every listed joint must carry a velocity
 * motor.                                                                  */
int avbd_set_motor_velocities(avbd_solver* solver, const uint32_t* joints,
                              uint32_t n, const float* rad_per_s);

/* Effort limits of authored motors (`setMotorTorques`,
 * GPUSolver.swift:2564-2578): finite and non-negative.  Raising the limit
 * of a joint authored with zero stiffness and zero effort (a joint no stage
 * solves) returns AVBD_ERR_UNSUPPORTED.                                   */
int avbd_set_motor_torques(avbd_solver* solver, const uint32_t* joints,
                           uint32_t n, const float* torques);

/* Hinge twist angle and twist rate of each listed joint (`motorStates`,
 * GPUSolver.swift:2606-2637).                                             */
int avbd_get_motor_states(avbd_solver* solver, const uint32_t* joints,
                          uint32_t n, float* angles, float* velocities);

/* Largest joint violation / contact penetration (`maxConstraintErrorChecked`,
 * GPUSolver.swift:4819-4865; kernel 40_solver.metal:2189-2229).            */
int avbd_max_constraint_error(avbd_solver* solver, float* out);

/* Counters of the last retired frame (`lastNumPairs`, `lastColorCounts`,
 * `lastNumSoft`, GPUSolver.swift:313-328).                                */
int avbd_get_counters(avbd_solver* solver, avbd_counters* out);

/* Latched runtime failure kind (AVBD_FAIL_*) of this solver
 * (`runtimeFailure`, GPUSolver.swift:2219-2229).                           */
int avbd_runtime_failure(const avbd_solver* solver, int* kind);

/* Copy the last error message (NUL-terminated, truncated to len). A NULL
 * solver reads the last construction error of the calling thread.         */
int avbd_last_error(const avbd_solver* solver, char* buf, size_t len);

/* Bit-for-bit capture / restore of every solver buffer
 * (`captureRigidSpeculationSnapshot` / `restore…`, GPUSolver.swift:2955-3057),
 * extended to soft state.                                                  */
int avbd_snapshot_capture(avbd_solver* solver, avbd_snapshot** out);
int avbd_snapshot_restore(avbd_solver* solver, const avbd_snapshot* snap);
void avbd_snapshot_free(avbd_snapshot* snap);

/* Launch all subsequent solver work on a caller-owned CUDA stream (a
 * cudaStream_t passed as void*, e.g. the stream an application or benchmark
 * records its CUDA events on).  NULL restores the solver's own stream.  The
 * solver synchronises its previous stream before switching.               */
int avbd_set_stream(avbd_solver* solver, void* cuda_stream);

/* Per-stage GPU timing (the reference's `profiling` mode with encoder
 * timestamps, GPUSolver.swift:3081-3093, :3167-3216, :4377-4400): while
 * enabled, every frame records CUDA events at its stage boundaries, is
 * retired synchronously, and its stage durations are accumulated.        */
enum {
    AVBD_STAGE_BROADPHASE = 0, AVBD_STAGE_NARROWPHASE = 1, AVBD_STAGE_PERSISTENCE_MAP = 2,
    AVBD_STAGE_WARMSTART = 3, AVBD_STAGE_ADJACENCY = 4, AVBD_STAGE_COLORING = 5,
    AVBD_STAGE_PRIMAL = 6, AVBD_STAGE_DUAL = 7, AVBD_STAGE_FINALIZE = 8,
    AVBD_STAGE_ELEMENT_CONTACTS = 9,  /* element grid, pair streams, emission */
    AVBD_STAGE_TRUNCATION = 10,       /* per-color Planar-DAT passes          */
    AVBD_STAGE_LEARNED = 11,          /* features, MLP, trial sweeps          */
    AVBD_STAGE_COUNT_ = 12
};
typedef struct avbd_profile {
    uint64_t frames;
    uint64_t kernels_per_frame;   /* kernel nodes in one frame's graph      */
    double stage_ms[16];          /* summed GPU time per stage              */
    uint64_t stage_launches[16];  /* kernel launches per stage              */
    uint32_t color_lanes[64];     /* primal variant of each static color's
                                   * lean particles, as chosen by the
                                   * autotuner: 8, 16 or 32 lanes per body
                                   * or AVBD_PRIMAL_VARIANT_STAGED           */
    /* dynamic coloring: block shape of the rigid primal's grid-stride
     * launch, chosen per body-count bucket (floor(log2(dynamic bodies)))
     * by timing candidate shapes on the first frames of the first solver
     * of that bucket on the device; later solvers reuse the choice          */
    uint32_t dyn_blocks;
    uint32_t dyn_threads;
    uint32_t dyn_bucket;
    uint32_t dyn_candidates;      /* shapes timed (0: taken from the cache)  */
} avbd_profile;
/* Pin the per-color primal variant of a static-palette scene: 8, 16 or 32
 * lanes per body (grouped kernel), AVBD_PRIMAL_VARIANT_STAGED (block-wide
 * term evaluation into shared memory, then an 8-lane fold per body), or 0 to
 * re-run the autotuner, which times every variant on the next frames and
 * keeps the fastest per color (the default).  Every variant computes the
 * same floats.  No counterpart in the reference, whose primal has one
 * launch shape (primal_particles_split, 40_solver.metal:1544-1686).        */
enum { AVBD_PRIMAL_VARIANT_AUTO = 0, AVBD_PRIMAL_VARIANT_STAGED = 1 };
int avbd_set_primal_variant(avbd_solver* solver, uint32_t variant);
int avbd_set_profiling(avbd_solver* solver, int enabled);
int avbd_get_profile(avbd_solver* solver, avbd_profile* out);

/* Lower a contact capacity below the one sized at upload, to provoke the
 * capacity failures on small scenes (`planarDATSoftCapacityForTesting`,
 * `planarDATPairCapacityForTesting`, GPUSolver.swift:2117-2133, :2235-2236).
 * The value is clamped to the allocated capacity; takes effect from the next
 * frame.                                                                    */
enum { AVBD_CAPACITY_SOFT_CONTACTS = 0, AVBD_CAPACITY_PLANAR_DAT_PAIRS = 1 };
int avbd_set_capacity_for_testing(avbd_solver* solver, int which, uint32_t value);

/* ---- Learned warm start (no counterpart in the reference) -------------
 * A 32-128-128-128-16 MLP (BF16 weights/activations, FP32 accumulation)
 * predicts each dynamic particle's correction of the plain gamma warm start
 * from local features (outputs 0-2, in units of s = max(|g|, 1) dt^2) and,
 * after avbd_set_warm_start_rigid(solver, 1), each dynamic rigid body's
 * (outputs 3-5: the rotation as arc length at the body's bounding radius,
 * in the same units).  In AVBD_WARM_START_LEARNED mode every frame races
 * the plain and the predicted warm start for `trial_sweeps` primal sweeps and
 * keeps the prediction only when its augmented-Lagrangian residual is no
 * larger; plain AVBD stays the fallback.  trial_sweeps = 0 compares the
 * residuals of the two warm starts themselves (no trial sweep); 1 keeps the
 * winner's trial sweep as the first iteration's primal half; at most 16.  Parameters are the fp32 block of
 * avbd_mlp_param_count() floats (W1[128][32], b1, W2[128][128], b2,
 * W3[128][128], b3, W4[16][128], b4[16]); `norm` holds 96 floats: feature
 * mean[32], feature 1/std[32], target mean[16], target std[16].          */
enum { AVBD_WARM_START_PLAIN = 0, AVBD_WARM_START_LEARNED = 1 };
int avbd_set_warm_start_model(avbd_solver* solver, const float* params, const float* norm,
                              uint32_t trial_sweeps);
int avbd_set_warm_start_mode(avbd_solver* solver, int mode);
/* Learned rows: the dynamic particles (enabled = 0, the default) or the
 * particles followed by the dynamic rigid bodies (enabled = 1).  On a scene
 * without particles, learning and the learned mode need enabled = 1.      */
int avbd_set_warm_start_rigid(avbd_solver* solver, int enabled);
/* Record every frame's features [n][32] and training targets [n][6] (the
 * solve's correction of the plain warm start; the rotation part zero for
 * particles) in the LEARN_* debug buffers.                                */
int avbd_set_learning_capture(avbd_solver* solver, int enabled);
/* Per-frame residual trace: out[0] at the plain warm start, out[1] at the
 * warm start used, out[2 + k] after iteration k (sqrt of the summed squared
 * AL gradient over all dynamic DOFs).  Read after avbd_sync.              */
int avbd_set_residual_trace(avbd_solver* solver, int enabled);
int avbd_get_residual_trace(avbd_solver* solver, double* out, uint32_t n);

/* Training kernels (device pointers; stream may be null).  A batch is
 * features[batch][32] and targets[batch][6] (raw, normalised with `norm`);
 * the workspace holds avbd_mlp_workspace_bytes(batch) bytes.  The GEMMs run
 * on the tensor cores (tcgen05.mma, accumulators in tensor memory) and give
 * up a wait for their MMA completion after about one second, latching a
 * status word in the workspace.  avbd_mlp_gradients synchronises `stream`
 * and fails on it; avbd_mlp_train_step stays asynchronous (the word is
 * cleared at step 1 and sticky afterwards) and avbd_mlp_workspace_status
 * synchronises and reports it.                                             */
uint32_t avbd_mlp_param_count(void);
size_t avbd_mlp_workspace_bytes(uint32_t batch);
int avbd_mlp_gradients(const float* params, const float* norm, const float* features,
                       const float* targets, uint32_t batch, void* workspace, float* grad_out,
                       float* loss_out, void* stream);
int avbd_mlp_train_step(float* params, const float* norm, const float* features,
                        const float* targets, uint32_t batch, float* adam_m, float* adam_v,
                        uint32_t step, float lr, void* workspace, float* loss_out, void* stream);
int avbd_mlp_workspace_status(const void* workspace, uint32_t batch, void* stream);
/* Inference over n feature rows into out[n][6] on the tensor cores
 * (tcgen05.mma, accumulators in tensor memory); synchronises `stream` and
 * returns AVBD_ERR_RUNTIME_FAILURE if the kernel's bounded wait for its MMA
 * completion gave up (workspace >= 80 KiB).                               */
int avbd_mlp_infer(const float* params, const float* norm, const float* features, uint32_t n,
                   float* out, void* workspace, void* stream);
/* Test of the inference kernel's bounded wait: the same launch with no
 * tensor-core work issued, so its wait for the MMA completion barrier runs
 * out (after about one second), the CTA frees its tensor memory and the call
 * returns AVBD_ERR_RUNTIME_FAILURE with the device still usable.  No
 * counterpart in the reference.                                            */
int avbd_mlp_infer_wait_timeout_for_testing(const float* params, const float* norm, const float* features,
                                            uint32_t n, float* out, void* workspace, void* stream);

/* Read-only access to one internal buffer for parity checks and tools
 * (no counterpart in the reference's public API; its tests read the same
 * buffers through @testable imports).  `which` is an AVBD_BUF_* id; `bytes`
 * must not exceed avbd_debug_buffer_size().                                */
enum {
    AVBD_BUF_POS_LIN = 0, AVBD_BUF_POS_ANG = 1, AVBD_BUF_VEL_LIN = 2,
    AVBD_BUF_VEL_ANG = 3, AVBD_BUF_PAIRS = 4, AVBD_BUF_MANIFOLDS = 5,
    AVBD_BUF_ADJ_START = 6, AVBD_BUF_ADJ_COUNT = 7, AVBD_BUF_ADJ_LIST = 8,
    AVBD_BUF_COLORS = 9, AVBD_BUF_COLOR_START = 10, AVBD_BUF_COLOR_LIST = 11,
    AVBD_BUF_CELL_START = 12, AVBD_BUF_CELL_COUNT = 13,
    AVBD_BUF_CELL_BODIES = 14, AVBD_BUF_MAP_KEY_A = 15, AVBD_BUF_MAP_KEY_B = 16,
    AVBD_BUF_MAP_VAL = 17, AVBD_BUF_JOINTS = 18, AVBD_BUF_SPRINGS = 19,
    AVBD_BUF_TETS = 20, AVBD_BUF_INIT_LIN = 21, AVBD_BUF_INERT_LIN = 22,
    AVBD_BUF_EXCLUSIONS = 23, AVBD_BUF_HASHED_IDX = 24, AVBD_BUF_GLOBAL_IDX = 25,
    /* cloth: element topology, element contacts, Planar-DAT pair stream */
    AVBD_BUF_TRIS = 26, AVBD_BUF_EDGES = 27, AVBD_BUF_NBR_START = 28,
    AVBD_BUF_NBR_COUNT = 29, AVBD_BUF_NBR_LIST = 30, AVBD_BUF_PARTICLE_IDX = 31,
    AVBD_BUF_MEMBRANES = 32, AVBD_BUF_BENDS = 33, AVBD_BUF_SOFT = 34,
    AVBD_BUF_DAT_PAIRS = 35, AVBD_BUF_CLOTH_GROUP = 36, AVBD_BUF_OGC_PREV = 37,
    /* learned warm start: vertex ids, features [n][32], targets and
     * predictions [n][3] of the last frame                                  */
    AVBD_BUF_LEARN_IDX = 38, AVBD_BUF_LEARN_FEATURES = 39, AVBD_BUF_LEARN_TARGETS = 40,
    AVBD_BUF_LEARN_PREDICTIONS = 41,
    AVBD_BUF_COUNT_ = 42
};
size_t avbd_debug_buffer_size(avbd_solver* solver, int which);
int avbd_debug_read(avbd_solver* solver, int which, void* dst, size_t bytes);

/* ---- Batched worlds (vector environments) -------------------------------
 * The reference batches environments by packing N replicas into one scene,
 * one collision group per environment (RL/PushTEnv.swift:137-180), and
 * resets them through setBodyStates (GPUSolver.swift:2409-2473).  These entry
 * points make that layout explicit with ragged world offsets.
 *
 * avbd_create_batched: `scene` packs `num_worlds` worlds of uneven size;
 * world w owns bodies [world_offsets[w], world_offsets[w + 1]) (num_worlds + 1
 * non-decreasing offsets); bodies outside every world are shared (static
 * ground, fixtures).  Every collider of world w's bodies is put in collision
 * group w + 1 (whatever the description says), shared colliders in group 0,
 * so worlds never touch one another and all meet the shared bodies.  A
 * joint, spring, tet, triangle or exclusion that joins two different worlds
 * is refused (AVBD_ERR_INVALID_ARGUMENT).  Otherwise as avbd_create.       */
int avbd_create_batched(const avbd_scene_desc* scene, const uint32_t* world_offsets, uint32_t num_worlds,
                        avbd_solver** out);
/* Number of worlds (0 for a solver from avbd_create) and, when `offsets` is
 * non-null, its num_worlds + 1 offsets.                                    */
int avbd_get_world_offsets(avbd_solver* solver, uint32_t* num_worlds, uint32_t* offsets);
/* setBodyStates for bodies addressed inside one world (local index 0 = the
 * world's first body), with its AL-reset of incident constraints.          */
int avbd_set_world_body_states(avbd_solver* solver, uint32_t world, const uint32_t* local_ids, uint32_t n,
                               const avbd_body_state* states);
/* Put each listed world back to its state at creation: body poses and
 * velocities, motor targets, and the AL state of every joint, spring and
 * contact touching its bodies (reset as setBodyStates does).              */
int avbd_reset_worlds(avbd_solver* solver, const uint32_t* worlds, uint32_t n);
/* The motorized joints of one world, in joint order: up to `cap` ids in
 * `ids`, their number in *count.                                           */
int avbd_get_world_motor_joints(avbd_solver* solver, uint32_t world, uint32_t* ids, uint32_t cap,
                                uint32_t* count);

/* Allocation-free exclusive prefix sum of `n` uint32 words on the current
 * device: d_out[i] = d_in[0] + ... + d_in[i-1] (the scan the solver uses for
 * its hash grid, pair lists and adjacency).  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc: code that runs inside an arena or
 * memory pool that must own every device allocation, a real-time loop with
 * an allocation ban, or a host application whose allocator must see every
 * device allocation.  This call makes no cudaMalloc, cudaFree or other
 * allocating call.  Its only scratch, 4 KiB of block sums, is a fixed array
 * in the library's device image: every GPU that loads the library holds it
 * until the process exits.
 *
 * Limit: n <= 1,048,576; a larger n returns AVBD_ERR_INVALID_ARGUMENT and
 * leaves the message for avbd_last_error(NULL, ...).  d_in and d_out are
 * device pointers on the current device; they may be equal (an in-place
 * scan) or disjoint, and a partial overlap returns AVBD_ERR_INVALID_ARGUMENT.
 * `cuda_stream` is a cudaStream_t passed as void* (NULL = the default
 * stream).  The first call in a CUDA context (the device's primary context,
 * or one the caller made current with cuCtxSetCurrent) looks up that
 * context's scratch array address (cudaGetSymbolAddress); make that first
 * call before any stream capture.
 * All calls share the one scratch array, so calls that overlap on the GPU
 * (work on different streams running at the same time) race: serialise them.
 * Each call writes every scratch word it reads before reading it, so nothing
 * has to be cleared between calls.                                          */
int avbd_exclusive_scan_noalloc(const uint32_t* d_in, uint32_t* d_out, uint32_t n,
                                void* cuda_stream);

/* ---- Headless render and observation compute ---------------------------
 * The reference's render-side compute kernels (Shaders/50_render.metal,
 * Shaders/60_robotics.metal) as CUDA kernels on the solver's stream, ordered
 * after the frames already submitted.  No graphics API is involved: every
 * call writes plain buffers.  `out_on_device` = 1: `out` is a device pointer
 * on the solver's device and the call returns without waiting; 0: `out` is
 * host memory and the call waits for the result.                          */

/* One instance record per rendered collider (RenderInstance,
 * 50_render.metal:7-11).                                                  */
typedef struct avbd_render_instance {
    float model[16];   /* column-major 4x4; sizes scale boxes and spheres,
                        * tori, capsules and hulls keep unit scale         */
    float color[4];    /* rgb; w = shape kind (0 box .. 4 convex hull)    */
    float params[4];   /* size x, size y, signed bounding radius,
                        * 1 for dynamic bodies (shadow strength)           */
} avbd_render_instance;

/* Instance transforms and colours from the current poses (`build_instances`,
 * 50_render.metal:34-97; `encodeBuildInstancesChecked`,
 * GPUSolver.swift:4605-4646).  `colliders`: n collider ids (the reference
 * renders colliders with `isRendered` whose body is not part of a soft
 * surface, GPUSolver.swift:1942-1949); `colors_rgba`: n render colours (w > 0
 * overrides the palette) or NULL; `color_mode` 0: palette by body id, 1: by
 * the body's graph colour.  A static ground slab wider than 150 m gets an
 * all-zero record.                                                         */
int avbd_build_instances(avbd_solver* solver, const uint32_t* colliders, uint32_t n,
                         const float* colors_rgba, uint32_t color_mode,
                         avbd_render_instance* out, int out_on_device);

/* Smooth normals of the soft surface (tet boundary faces and authored
 * triangles): face normals, then an angle x area weighted gather per vertex
 * (`soft_face_normals`, `soft_normals`, 50_render.metal:104-180).  `out`
 * holds one float4 per body (xyz unit normal, w render thickness =
 * |radius| x (cloth_scale for cloth vertices) x a curvature factor); entries
 * of bodies off the surface are left untouched.  `cloth_scale` is
 * `clothRenderScale` (Scene.swift:542).                                   */
int avbd_soft_normals(avbd_solver* solver, float cloth_scale, float* out_xyzw,
                      int out_on_device);

/* A render-mesh vertex bound to four bodies (SkinBindingGPU,
 * GPUTypes.swift:104-111): position = sum of weights x body positions; the
 * normal follows the cofactor of the deformation gradient Ds * Dm^-1.      */
typedef struct avbd_skin_binding {
    uint32_t ids[4];
    float weights[4];
    float rest_normal[4];  /* xyz; normalised on upload, +z if zero        */
    float inv0[4], inv1[4], inv2[4];  /* rows of Dm^-1; all zero = the
                                         rest-pose inverse of the four
                                         bodies' scene positions          */
} avbd_skin_binding;

/* Uploads the skin bindings (GPUSolver.swift:1849-1907), replacing earlier
 * ones.  n = 0 clears them.                                                */
int avbd_set_skin_bindings(avbd_solver* solver, const avbd_skin_binding* bindings,
                           uint32_t n);

/* Deformed skin vertices (`skin_deform`, 50_render.metal:182-212): per
 * binding 8 floats, position (w = 1) then unit normal (w = 0).             */
int avbd_skin_deform(avbd_solver* solver, float* out, int out_on_device);

/* One Push-T environment of an observation batch (PushTEnvGPU,
 * RL/PushTEnv.swift:28-32).                                               */
typedef struct avbd_pusht_env {
    uint32_t ids[4];   /* pusher tip, block bar, block stem, unused        */
    float frame[4];    /* environment centre xy, goal position xy (local)  */
    float goal[4];     /* goal yaw, half window, unused, unused            */
} avbd_pusht_env;

/* Top-down RGB observations of a Push-T batch (`pusht_obs`,
 * 60_robotics.metal:21-69; `renderPushTObsChecked`, GPUSolver.swift:
 * 2296-2325): num_envs x res x res x 3 bytes, row-major per environment,
 * goal T green under the block T red under the pusher disc blue on a dark
 * background.  2 <= res <= 4096; a device `out` must be 16-byte aligned
 * when res is a multiple of 4.  The table is kept on the device while later
 * calls pass the same records.                                             */
int avbd_render_pusht_obs(avbd_solver* solver, const avbd_pusht_env* envs,
                          uint32_t num_envs, uint32_t res, uint8_t* out,
                          int out_on_device);

#ifdef __cplusplus
}
#endif
#endif /* AVBD_H */
