"""ctypes mirror of include/avbd.h (the C ABI of the solver step).

Every record here has the same field order and width as its C declaration;
tests/test_abi.py checks the sizes against the compiled library.
"""
import ctypes as C

ABI_VERSION = 3
CAPACITY_SOFT_CONTACTS, CAPACITY_PLANAR_DAT_PAIRS = 0, 1
PRIMAL_VARIANT_AUTO, PRIMAL_VARIANT_STAGED = 0, 1

# status codes
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_NO_DEVICE = 2
ERR_ALLOC_FAILED = 3
ERR_KERNEL_MISSING = 4
ERR_RUNTIME_FAILURE = 5
ERR_UNSUPPORTED = 6

STATUS_NAMES = {
    OK: "ok", ERR_INVALID_ARGUMENT: "invalid argument", ERR_NO_DEVICE: "no device",
    ERR_ALLOC_FAILED: "allocation failed", ERR_KERNEL_MISSING: "kernel missing",
    ERR_RUNTIME_FAILURE: "runtime failure", ERR_UNSUPPORTED: "unsupported scene feature",
}

# runtime failure kinds
FAIL_NONE = 0
FAIL_COMMAND_EXECUTION = 1
FAIL_RIGID_PAIR_CAPACITY = 2
FAIL_SOFT_CONTACT_CAPACITY = 3
FAIL_STATIC_COLOR_CAPACITY = 4
FAIL_UNRESOLVED_COLORING = 5
FAIL_PLANAR_DAT_PAIR_CAPACITY = 6
FAIL_PLANAR_DAT_GRID_SPAN = 7
FAIL_PLANAR_DAT_INVALID_ANCHOR = 8
FAIL_WAIT_TIMEOUT = 9

SHAPE_BOX, SHAPE_SPHERE, SHAPE_TORUS, SHAPE_CAPSULE = 0, 1, 2, 3
MOTOR_IMPLICIT_POSITION_PD, MOTOR_EXPLICIT_TORQUE_PD, MOTOR_VELOCITY = 0, 1, 2
TRUNCATION_AUTOMATIC, TRUNCATION_ISOTROPIC, TRUNCATION_PLANAR_DAT = 0, 1, 2

# debug buffer ids (AVBD_BUF_*)
BUF = dict(
    POS_LIN=0, POS_ANG=1, VEL_LIN=2, VEL_ANG=3, PAIRS=4, MANIFOLDS=5, ADJ_START=6,
    ADJ_COUNT=7, ADJ_LIST=8, COLORS=9, COLOR_START=10, COLOR_LIST=11, CELL_START=12,
    CELL_COUNT=13, CELL_BODIES=14, MAP_KEY_A=15, MAP_KEY_B=16, MAP_VAL=17, JOINTS=18,
    SPRINGS=19, TETS=20, INIT_LIN=21, INERT_LIN=22, EXCLUSIONS=23, HASHED_IDX=24,
    GLOBAL_IDX=25, TRIS=26, EDGES=27, NBR_START=28, NBR_COUNT=29, NBR_LIST=30,
    PARTICLE_IDX=31, MEMBRANES=32, BENDS=33, SOFT=34, DAT_PAIRS=35, CLOTH_GROUP=36,
    OGC_PREV=37, LEARN_IDX=38, LEARN_FEATURES=39, LEARN_TARGETS=40, LEARN_PREDICTIONS=41,
)

F3 = C.c_float * 3
F4 = C.c_float * 4


class Settings(C.Structure):
    _fields_ = [
        ("dt", C.c_float), ("gravity", C.c_float), ("iterations", C.c_int32),
        ("collision_margin", C.c_float), ("friction_combine_mode", C.c_uint32),
        ("alpha", C.c_float), ("beta_lin", C.c_float), ("beta_ang", C.c_float),
        ("gamma", C.c_float), ("lambda_max", C.c_float), ("rod_decay_pow", C.c_float),
        ("particle_damping", C.c_float), ("rigid_linear_damping", C.c_float),
        ("rigid_angular_damping", C.c_float), ("cloth_viscosity", C.c_float),
    ]


class BodyDesc(C.Structure):
    _fields_ = [
        ("size", F3), ("density", C.c_float), ("friction", C.c_float),
        ("dynamic_friction", C.c_float), ("position", F3), ("rotation", F4),
        ("velocity", F3), ("shape", C.c_uint32), ("is_particle", C.c_uint32),
        ("has_explicit_mass", C.c_uint32), ("mass", C.c_float),
        ("diagonal_inertia", F3), ("gravity_scale", C.c_float),
    ]


class ColliderDesc(C.Structure):
    _fields_ = [
        ("body", C.c_int32), ("size", F3), ("friction", C.c_float),
        ("dynamic_friction", C.c_float), ("local_position", F3),
        ("local_rotation", F4), ("shape", C.c_uint32), ("collision_group", C.c_uint32),
        ("collides_with_shared", C.c_uint32), ("collision_enabled", C.c_uint32),
        ("world_round_anchor", C.c_uint32), ("hull_offset", C.c_uint32),
        ("hull_count", C.c_uint32),
    ]


class JointDesc(C.Structure):
    _fields_ = [
        ("body_a", C.c_int32), ("body_b", C.c_int32), ("r_a", F3), ("r_b", F3),
        ("stiffness_lin", C.c_float), ("stiffness_ang", C.c_float),
        ("fracture", C.c_float), ("fracture_linear", C.c_uint32),
        ("has_hinge", C.c_uint32), ("hinge_axis", F3), ("motor_target", C.c_float),
        ("motor_torque", C.c_float), ("motor_rate", C.c_float),
        ("motor_stiffness", C.c_float), ("motor_damping", C.c_float),
        ("motor_mode", C.c_uint32), ("armature", C.c_float), ("limit_lo", C.c_float),
        ("limit_hi", C.c_float),
    ]


class SpringDesc(C.Structure):
    _fields_ = [
        ("body_a", C.c_int32), ("body_b", C.c_int32), ("r_a", F3), ("r_b", F3),
        ("stiffness", C.c_float), ("rest", C.c_float), ("hard", C.c_uint32),
    ]


class TetDesc(C.Structure):
    _fields_ = [("ids", C.c_int32 * 4), ("mu", C.c_float), ("lambda_", C.c_float),
                ("self_collision", C.c_uint32)]


class TriDesc(C.Structure):
    _fields_ = [("ids", C.c_int32 * 3), ("mu", C.c_float), ("lambda_", C.c_float),
                ("bend", C.c_float)]


class ExclusionDesc(C.Structure):
    _fields_ = [("body_a", C.c_int32), ("body_b", C.c_int32)]


class SpinnerDesc(C.Structure):
    _fields_ = [("body", C.c_int32), ("axis", F3), ("omega", C.c_float)]


class SceneDesc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_uint32),
        ("num_bodies", C.c_uint32), ("bodies", C.POINTER(BodyDesc)),
        ("num_colliders", C.c_uint32), ("colliders", C.POINTER(ColliderDesc)),
        ("num_hull_vertices", C.c_uint32), ("hull_vertices", C.POINTER(C.c_float)),
        ("num_joints", C.c_uint32), ("joints", C.POINTER(JointDesc)),
        ("num_springs", C.c_uint32), ("springs", C.POINTER(SpringDesc)),
        ("num_tets", C.c_uint32), ("tets", C.POINTER(TetDesc)),
        ("num_tris", C.c_uint32), ("tris", C.POINTER(TriDesc)),
        ("num_exclusions", C.c_uint32), ("exclusions", C.POINTER(ExclusionDesc)),
        ("num_spinners", C.c_uint32), ("spinners", C.POINTER(SpinnerDesc)),
        ("settings", Settings),
        ("max_pairs_per_body", C.c_uint32),
        ("truncation_selection", C.c_uint32),
        ("tet_inversion_prevention", C.c_uint32),
        ("device", C.c_int32),
    ]


class BodyState(C.Structure):
    _fields_ = [("position", F3), ("rotation", F4), ("velocity", F3),
                ("angular_velocity", F3)]


class Counters(C.Structure):
    _fields_ = [
        ("frame", C.c_uint64), ("num_pairs", C.c_uint32),
        ("pair_candidates", C.c_uint32), ("num_soft", C.c_uint32),
        ("soft_candidates", C.c_uint32), ("used_colors", C.c_uint32),
        ("color_conflicts", C.c_uint32), ("ogc_exceeded", C.c_uint32),
        ("color_counts", C.c_uint32 * 64),
        ("dat_pairs", C.c_uint32), ("dat_vt_pairs", C.c_uint32), ("dat_ee_pairs", C.c_uint32),
        ("dat_grid_overflows", C.c_uint32), ("dat_invalid_anchors", C.c_uint32),
        ("dat_truncations", C.c_uint32), ("dat_vt_degenerate", C.c_uint32),
        ("dat_ee_degenerate", C.c_uint32), ("dat_nonfinite", C.c_uint32),
        ("dat_tet_degenerate", C.c_uint32), ("learn_accepted", C.c_uint32),
        ("soft_rt", C.c_uint32), ("soft_vt", C.c_uint32), ("soft_ee", C.c_uint32),
    ]


class RenderInstance(C.Structure):
    """avbd_render_instance (RenderInstance, 50_render.metal:7-11)."""
    _fields_ = [("model", C.c_float * 16), ("color", C.c_float * 4), ("params", C.c_float * 4)]


class SkinBinding(C.Structure):
    """avbd_skin_binding (SkinBindingGPU, GPUTypes.swift:104-111)."""
    _fields_ = [("ids", C.c_uint32 * 4), ("weights", C.c_float * 4), ("rest_normal", C.c_float * 4),
                ("inv0", C.c_float * 4), ("inv1", C.c_float * 4), ("inv2", C.c_float * 4)]


class PushTEnv(C.Structure):
    """avbd_pusht_env (PushTEnvGPU, RL/PushTEnv.swift:28-32)."""
    _fields_ = [("ids", C.c_uint32 * 4), ("frame", C.c_float * 4), ("goal", C.c_float * 4)]


# Exported symbols declared in include/avbd.h (checked by the CPU tests).
EXPORTED = [
    "avbd_create", "avbd_destroy", "avbd_set_settings", "avbd_get_settings",
    "avbd_step", "avbd_sync", "avbd_get_body_states", "avbd_set_body_states",
    "avbd_get_positions", "avbd_set_positions", "avbd_set_motor_targets",
    "avbd_set_joint_world_anchors", "avbd_set_motor_velocities", "avbd_set_motor_torques",
    "avbd_get_motor_states",
    "avbd_max_constraint_error", "avbd_get_counters", "avbd_runtime_failure",
    "avbd_last_error", "avbd_snapshot_capture", "avbd_snapshot_restore",
    "avbd_snapshot_free", "avbd_debug_buffer_size", "avbd_debug_read", "avbd_set_stream",
    "avbd_set_profiling", "avbd_get_profile", "avbd_set_primal_variant", "avbd_exclusive_scan_noalloc", "avbd_set_capacity_for_testing",
    "avbd_set_warm_start_model", "avbd_set_warm_start_mode", "avbd_set_warm_start_rigid",
    "avbd_set_learning_capture",
    "avbd_set_residual_trace", "avbd_get_residual_trace", "avbd_mlp_param_count",
    "avbd_mlp_workspace_bytes", "avbd_mlp_gradients", "avbd_mlp_train_step", "avbd_mlp_workspace_status", "avbd_mlp_infer", "avbd_mlp_infer_wait_timeout_for_testing",
    "avbd_build_instances", "avbd_soft_normals", "avbd_set_skin_bindings", "avbd_skin_deform",
    "avbd_render_pusht_obs", "avbd_create_batched", "avbd_get_world_offsets", "avbd_set_world_body_states",
    "avbd_reset_worlds", "avbd_get_world_motor_joints",
]
WARM_START_PLAIN, WARM_START_LEARNED = 0, 1

STAGES = ["broadphase", "narrowphase", "persistence_map", "warmstart", "adjacency",
          "coloring", "primal", "dual", "finalize", "element_contacts", "truncation", "learned"]


class Profile(C.Structure):
    _fields_ = [("frames", C.c_uint64), ("kernels_per_frame", C.c_uint64),
                ("stage_ms", C.c_double * 16),
                ("stage_launches", C.c_uint64 * 16),
                ("color_lanes", C.c_uint32 * 64),
                ("dyn_blocks", C.c_uint32), ("dyn_threads", C.c_uint32),
                ("dyn_bucket", C.c_uint32), ("dyn_candidates", C.c_uint32)]
