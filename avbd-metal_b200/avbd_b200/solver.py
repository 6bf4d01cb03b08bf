"""`GPUSolver`: the Python host mirror of the reference's solver class
(Sources/PhysicsAVBD/GPU/GPUSolver.swift:17) over the C ABI of include/avbd.h.

The CUDA library is required: there is no CPU fallback.  Errors follow the
reference's convention — construction errors raise `AVBDError`, runtime
failures raise `RuntimeFailure` and are sticky (every later call raises).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import abi
from .scene import PhysicsScene, SimSettings

_LIB = None


class AVBDError(RuntimeError):
    """Construction error (AVBDError, GPUSolver.swift:640-661)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class RuntimeFailure(RuntimeError):
    """Latched runtime failure (RuntimeFailure, GPUSolver.swift:663-751)."""

    def __init__(self, kind: int, message: str):
        super().__init__(message or f"runtime failure {kind}")
        self.kind = kind


def library_path() -> str:
    here = os.path.dirname(os.path.abspath(__file__))
    return os.path.join(here, "_lib", "libavbd_b200.so")


def load_library() -> C.CDLL:
    """Load the in-tree CUDA library (fails loudly when it is missing)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not os.path.exists(path):
        raise ImportError(f"CUDA solver library not built: {path} (run avbd_b200.build.build())")
    lib = C.CDLL(path)
    vp, u32, i32, sz = C.c_void_p, C.c_uint32, C.c_int, C.c_size_t
    sig = {
        "avbd_create": ([vp, C.POINTER(vp)], i32),
        "avbd_destroy": ([vp], None),
        "avbd_set_settings": ([vp, vp], i32),
        "avbd_get_settings": ([vp, vp], i32),
        "avbd_step": ([vp, u32], i32),
        "avbd_sync": ([vp], i32),
        "avbd_get_body_states": ([vp, vp, u32, vp], i32),
        "avbd_set_body_states": ([vp, vp, u32, vp], i32),
        "avbd_get_positions": ([vp, u32, vp, vp], i32),
        "avbd_set_positions": ([vp, u32, vp], i32),
        "avbd_set_motor_targets": ([vp, vp, u32, vp], i32),
        "avbd_set_joint_world_anchors": ([vp, vp, u32, vp], i32),
        "avbd_set_motor_velocities": ([vp, vp, u32, vp], i32),
        "avbd_set_motor_torques": ([vp, vp, u32, vp], i32),
        "avbd_get_motor_states": ([vp, vp, u32, vp, vp], i32),
        "avbd_build_instances": ([vp, vp, u32, vp, u32, vp, i32], i32),
        "avbd_soft_normals": ([vp, C.c_float, vp, i32], i32),
        "avbd_set_skin_bindings": ([vp, vp, u32], i32),
        "avbd_skin_deform": ([vp, vp, i32], i32),
        "avbd_render_pusht_obs": ([vp, vp, u32, u32, vp, i32], i32),
        "avbd_max_constraint_error": ([vp, C.POINTER(C.c_float)], i32),
        "avbd_get_counters": ([vp, vp], i32),
        "avbd_runtime_failure": ([vp, C.POINTER(i32)], i32),
        "avbd_last_error": ([vp, C.c_char_p, sz], i32),
        "avbd_snapshot_capture": ([vp, C.POINTER(vp)], i32),
        "avbd_snapshot_restore": ([vp, vp], i32),
        "avbd_snapshot_free": ([vp], None),
        "avbd_debug_buffer_size": ([vp, i32], sz),
        "avbd_debug_read": ([vp, i32, vp, sz], i32),
        "avbd_set_stream": ([vp, vp], i32),
        "avbd_set_profiling": ([vp, i32], i32),
        "avbd_set_primal_variant": ([vp, u32], i32),
        "avbd_set_capacity_for_testing": ([vp, i32, u32], i32),
        "avbd_get_profile": ([vp, vp], i32),
        "avbd_set_warm_start_model": ([vp, vp, vp, u32], i32),
        "avbd_set_warm_start_mode": ([vp, i32], i32),
        "avbd_set_warm_start_rigid": ([vp, i32], i32),
        "avbd_set_learning_capture": ([vp, i32], i32),
        "avbd_set_residual_trace": ([vp, i32], i32),
        "avbd_get_residual_trace": ([vp, vp, u32], i32),
        "avbd_create_batched": ([vp, vp, u32, C.POINTER(vp)], i32),
        "avbd_get_world_offsets": ([vp, C.POINTER(u32), vp], i32),
        "avbd_set_world_body_states": ([vp, u32, vp, u32, vp], i32),
        "avbd_reset_worlds": ([vp, vp, u32], i32),
        "avbd_get_world_motor_joints": ([vp, u32, vp, u32, C.POINTER(u32)], i32),
        "avbd_mlp_param_count": ([], u32),
        "avbd_mlp_workspace_bytes": ([u32], sz),
        "avbd_mlp_gradients": ([vp, vp, vp, vp, u32, vp, vp, vp, vp], i32),
        "avbd_mlp_train_step": ([vp, vp, vp, vp, u32, vp, vp, u32, C.c_float, vp, vp, vp], i32),
        "avbd_mlp_workspace_status": ([vp, u32, vp], i32),
        "avbd_mlp_infer": ([vp, vp, vp, u32, vp, vp, vp], i32),
        "avbd_mlp_infer_wait_timeout_for_testing": ([vp, vp, vp, u32, vp, vp, vp], i32),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _LIB = lib
    return lib


def _last_error(h=None) -> str:
    buf = C.create_string_buffer(512)
    load_library().avbd_last_error(h, buf, 512)
    return buf.value.decode(errors="replace")


class GPUSolver:
    """AVBD solver step on one CUDA device (GPUSolver.swift:17)."""

    def __init__(self, scene: PhysicsScene, max_pairs_per_body: int = 16, device: int = -1,
                 truncation: int = abi.TRUNCATION_AUTOMATIC, tet_inversion_prevention: bool = False,
                 world_offsets=None):
        """world_offsets: batched worlds (avbd_create_batched) — world w owns
        bodies [world_offsets[w], world_offsets[w + 1]); each world gets its
        own collision group, bodies outside every world are shared."""
        lib = load_library()
        desc, self._keep = scene.to_desc(max_pairs_per_body=max_pairs_per_body,
                                         truncation=truncation,
                                         tet_inversion_prevention=tet_inversion_prevention,
                                         device=device)
        h = C.c_void_p()
        if world_offsets is None:
            rc = lib.avbd_create(C.byref(desc), C.byref(h))
        else:
            offs = np.ascontiguousarray(world_offsets, dtype=np.uint32)
            rc = lib.avbd_create_batched(C.byref(desc), offs.ctypes.data, max(0, len(offs) - 1), C.byref(h))
        if rc != abi.OK:
            raise AVBDError(rc, _last_error(None))
        self._h = h
        self.num_bodies = len(scene.bodies)
        self.num_joints = len(scene.joints)
        self._settings = scene.settings

    # -- lifetime ------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            load_library().avbd_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass

    def _check(self, rc: int):
        if rc == abi.OK:
            return
        if rc == abi.ERR_RUNTIME_FAILURE:
            raise RuntimeFailure(self.runtime_failure(), _last_error(self._h))
        raise AVBDError(rc, _last_error(self._h))

    # -- stepping (submitStep / synchronize) ----------------------------------
    @property
    def settings(self) -> SimSettings:
        return self._settings

    @settings.setter
    def settings(self, st: SimSettings):
        c = st.to_c()
        self._check(load_library().avbd_set_settings(self._h, C.byref(c)))
        self._settings = st

    def submit_step(self, frames: int = 1):
        self._check(load_library().avbd_step(self._h, frames))

    def step(self, frames: int = 1):
        self.submit_step(frames)

    def synchronize(self):
        self._check(load_library().avbd_sync(self._h))

    # -- state ---------------------------------------------------------------
    def positions(self):
        """(posLin xyzw with w = mass, posAng xyzw) for every body."""
        n = self.num_bodies
        pos = np.empty((n, 4), np.float32)
        rot = np.empty((n, 4), np.float32)
        self._check(load_library().avbd_get_positions(self._h, n, pos.ctypes.data, rot.ctypes.data))
        return pos, rot

    def read_positions_into(self, pos: np.ndarray):
        self._check(load_library().avbd_get_positions(self._h, pos.shape[0], pos.ctypes.data, None))

    def set_positions(self, xyz: np.ndarray):
        xyz = np.ascontiguousarray(xyz, dtype=np.float32)
        self._check(load_library().avbd_set_positions(self._h, xyz.shape[0], xyz.ctypes.data))

    def body_states(self, ids=None):
        n = self.num_bodies if ids is None else len(ids)
        out = (abi.BodyState * n)()
        idp = None
        if ids is not None:
            idarr = np.ascontiguousarray(ids, dtype=np.uint32)
            idp = idarr.ctypes.data
        self._check(load_library().avbd_get_body_states(self._h, idp, n, out))
        return out

    def body_position(self, i: int):
        return tuple(self.body_states([i])[0].position)

    def set_body_states(self, ids, states):
        idarr = np.ascontiguousarray(ids, dtype=np.uint32)
        arr = (abi.BodyState * len(states))(*states)
        self._check(load_library().avbd_set_body_states(self._h, idarr.ctypes.data, len(states), arr))

    def set_motor_targets(self, joints, targets):
        ids = np.ascontiguousarray(joints, dtype=np.uint32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        self._check(load_library().avbd_set_motor_targets(self._h, ids.ctypes.data, len(ids), t.ctypes.data))

    def set_joint_world_anchors(self, joints, points):
        """setJointWorldAnchors (GPUSolver.swift:2481-2494)."""
        ids = np.ascontiguousarray(joints, dtype=np.uint32)
        p = np.ascontiguousarray(points, dtype=np.float32).reshape(-1)
        if p.size != 3 * ids.size:
            raise ValueError("one xyz point per joint")
        self._check(load_library().avbd_set_joint_world_anchors(self._h, ids.ctypes.data, len(ids), p.ctypes.data))

    def set_motor_velocities(self, joints, rad_per_s):
        """setMotorVelocities (GPUSolver.swift:2534-2551)."""
        ids = np.ascontiguousarray(joints, dtype=np.uint32)
        v = np.ascontiguousarray(rad_per_s, dtype=np.float32)
        self._check(load_library().avbd_set_motor_velocities(self._h, ids.ctypes.data, len(ids), v.ctypes.data))

    def set_motor_torques(self, joints, torques):
        """setMotorTorques (GPUSolver.swift:2564-2578)."""
        ids = np.ascontiguousarray(joints, dtype=np.uint32)
        t = np.ascontiguousarray(torques, dtype=np.float32)
        self._check(load_library().avbd_set_motor_torques(self._h, ids.ctypes.data, len(ids), t.ctypes.data))

    # -- headless render and observation compute -------------------------------
    # Each call writes host arrays (returned) unless `device_out` gives a
    # device address (an int, e.g. a torch tensor's data_ptr()): then it only
    # enqueues the kernel on the solver's stream and returns None.
    def build_instances(self, colliders, colors=None, color_mode: int = 0, device_out=None):
        """encodeBuildInstancesChecked (GPUSolver.swift:4605-4646): (n, 24)
        float32 records (4x4 model column-major, rgba-kind colour, params)."""
        ids = np.ascontiguousarray(colliders, dtype=np.uint32)
        col = None if colors is None else np.ascontiguousarray(colors, dtype=np.float32).reshape(-1, 4)
        out = None if device_out is not None else np.zeros((len(ids), 24), np.float32)
        self._check(load_library().avbd_build_instances(
            self._h, ids.ctypes.data, len(ids), None if col is None else col.ctypes.data, color_mode,
            device_out if device_out is not None else out.ctypes.data, 1 if device_out is not None else 0))
        return out

    def soft_normals(self, cloth_scale: float = 0.0, out=None, device_out=None):
        """soft_face_normals + soft_normals (50_render.metal:104-180): one
        float4 per body (normal, render thickness); entries off the surface
        keep the values of `out` (zeros by default)."""
        if device_out is not None:
            self._check(load_library().avbd_soft_normals(self._h, cloth_scale, device_out, 1))
            return None
        res = np.zeros((self.num_bodies, 4), np.float32) if out is None else np.ascontiguousarray(out, np.float32)
        self._check(load_library().avbd_soft_normals(self._h, cloth_scale, res.ctypes.data, 0))
        return res

    def set_skin_bindings(self, bindings):
        """Skin bindings (GPUSolver.swift:1849-1907): a sequence of
        abi.SkinBinding or a ctypes array of them."""
        arr = (abi.SkinBinding * len(bindings))(*bindings)
        self._num_skin = len(bindings)
        self._check(load_library().avbd_set_skin_bindings(self._h, arr, len(bindings)))

    def skin_deform(self, device_out=None):
        """skin_deform (50_render.metal:182-212): (n, 8) float32 = position
        (w 1) and normal (w 0) per binding."""
        n = getattr(self, "_num_skin", 0)
        if device_out is not None:
            self._check(load_library().avbd_skin_deform(self._h, device_out, 1))
            return None
        out = np.zeros((n, 8), np.float32)
        self._check(load_library().avbd_skin_deform(self._h, out.ctypes.data if n else out.ctypes.data, 0))
        return out

    def render_pusht_obs(self, envs, res: int = 64, device_out=None):
        """renderPushTObsChecked (GPUSolver.swift:2296-2325): uint8 array
        (num_envs, res, res, 3)."""
        arr = envs if isinstance(envs, C.Array) else (abi.PushTEnv * len(envs))(*envs)
        if device_out is not None:
            self._check(load_library().avbd_render_pusht_obs(self._h, arr, len(envs), res, device_out, 1))
            return None
        out = np.zeros((len(envs), res, res, 3), np.uint8)
        self._check(load_library().avbd_render_pusht_obs(self._h, arr, len(envs), res, out.ctypes.data, 0))
        return out

    def motor_states(self, joints):
        """motorStates (GPUSolver.swift:2606-2637): (angles, velocities)."""
        ids = np.ascontiguousarray(joints, dtype=np.uint32)
        a = np.zeros(len(ids), np.float32)
        v = np.zeros(len(ids), np.float32)
        self._check(load_library().avbd_get_motor_states(self._h, ids.ctypes.data, len(ids), a.ctypes.data,
                                                         v.ctypes.data))
        return a, v

    # -- diagnostics -----------------------------------------------------------
    # -- batched worlds (vector environments) ---------------------------------
    def world_offsets(self) -> np.ndarray:
        n = C.c_uint32()
        self._check(load_library().avbd_get_world_offsets(self._h, C.byref(n), None))
        out = np.zeros(n.value + 1 if n.value else 0, np.uint32)
        if n.value:
            self._check(load_library().avbd_get_world_offsets(self._h, C.byref(n), out.ctypes.data))
        return out

    def set_world_body_states(self, world: int, local_ids, states):
        ids = np.ascontiguousarray(local_ids, dtype=np.uint32)
        arr = (abi.BodyState * len(states))(*states)
        self._check(load_library().avbd_set_world_body_states(self._h, world, ids.ctypes.data, len(ids), arr))

    def reset_worlds(self, worlds):
        w = np.ascontiguousarray(worlds, dtype=np.uint32)
        self._check(load_library().avbd_reset_worlds(self._h, w.ctypes.data, len(w)))

    def world_motor_joints(self, world: int) -> np.ndarray:
        n = C.c_uint32()
        self._check(load_library().avbd_get_world_motor_joints(self._h, world, None, 0, C.byref(n)))
        out = np.zeros(n.value, np.uint32)
        if n.value:
            self._check(load_library().avbd_get_world_motor_joints(self._h, world, out.ctypes.data, n.value,
                                                                   C.byref(n)))
        return out

    def max_constraint_error(self) -> float:
        v = C.c_float()
        self._check(load_library().avbd_max_constraint_error(self._h, C.byref(v)))
        return v.value

    def counters(self) -> abi.Counters:
        c = abi.Counters()
        load_library().avbd_get_counters(self._h, C.byref(c))
        return c

    def runtime_failure(self) -> int:
        k = C.c_int()
        load_library().avbd_runtime_failure(self._h, C.byref(k))
        return k.value

    def last_error(self) -> str:
        return _last_error(self._h)

    def snapshot(self):
        s = C.c_void_p()
        self._check(load_library().avbd_snapshot_capture(self._h, C.byref(s)))
        return _Snapshot(s)

    def restore(self, snap):
        self._check(load_library().avbd_snapshot_restore(self._h, snap._h))

    def set_stream(self, cuda_stream_handle):
        """Launch on a caller-owned stream (an integer cudaStream_t handle, e.g.
        torch.cuda.Stream().cuda_stream); None restores the solver's stream."""
        self._check(load_library().avbd_set_stream(self._h, cuda_stream_handle or None))

    def set_capacity_for_testing(self, which: int, value: int):
        """Lower the soft-contact or Planar-DAT pair capacity (abi.CAPACITY_*)
        to provoke its capacity failure on a small scene."""
        self._check(load_library().avbd_set_capacity_for_testing(self._h, int(which), int(value)))

    def set_primal_variant(self, variant: int):
        """Pin every static color's primal to one variant: 8, 16 or 32 lanes
        per body, abi.PRIMAL_VARIANT_STAGED, or abi.PRIMAL_VARIANT_AUTO to
        re-run the autotuner.  All variants compute the same floats."""
        self._check(load_library().avbd_set_primal_variant(self._h, int(variant)))

    def set_profiling(self, enabled: bool):
        self._check(load_library().avbd_set_profiling(self._h, 1 if enabled else 0))

    def profile(self) -> dict:
        p = abi.Profile()
        self._check(load_library().avbd_get_profile(self._h, C.byref(p)))
        return {"frames": p.frames, "kernels_per_frame": p.kernels_per_frame,
                "stage_ms": {n: p.stage_ms[i] for i, n in enumerate(abi.STAGES)},
                "stage_launches": {n: p.stage_launches[i] for i, n in enumerate(abi.STAGES)},
                "color_lanes": list(p.color_lanes),
                "dynamic_primal_shape": {"blocks": p.dyn_blocks, "threads": p.dyn_threads,
                                         "body_count_bucket": p.dyn_bucket, "candidates_timed": p.dyn_candidates}}

    # ---- learned warm start ------------------------------------------------
    def set_warm_start_model(self, params, norm, trial_sweeps: int = 1, rigid: Optional[bool] = None) -> None:
        """Upload an MLP (fp32 parameter block and 96-float normalisation);
        `rigid` (when given) sets whether it predicts the rigid bodies too."""
        p = np.ascontiguousarray(params, np.float32)
        n = np.ascontiguousarray(norm, np.float32)
        self._check(load_library().avbd_set_warm_start_model(self._h, p.ctypes.data, n.ctypes.data,
                                                             int(trial_sweeps)))
        if rigid is not None:
            self.set_warm_start_rigid(rigid)

    def set_warm_start_rigid(self, enabled: bool) -> None:
        """Learned rows: the particles (False) or the particles and the
        dynamic rigid bodies (True)."""
        self._check(load_library().avbd_set_warm_start_rigid(self._h, 1 if enabled else 0))

    def set_warm_start_mode(self, mode: int) -> None:
        self._check(load_library().avbd_set_warm_start_mode(self._h, int(mode)))

    def set_learning_capture(self, enabled: bool) -> None:
        self._check(load_library().avbd_set_learning_capture(self._h, 1 if enabled else 0))

    def set_residual_trace(self, enabled: bool) -> None:
        self._check(load_library().avbd_set_residual_trace(self._h, 1 if enabled else 0))

    def residual_trace(self, n: int) -> np.ndarray:
        """[r(plain warm start), r(warm start used), r after iteration 1..n-2]."""
        out = np.zeros(n, np.float64)
        self._check(load_library().avbd_get_residual_trace(self._h, out.ctypes.data, n))
        return out

    def learning_sample(self):
        """(features [n][32], targets [n][6]) of the last captured frame:
        particle rows first, then the rigid bodies when they are learned."""
        f = self.debug_read("LEARN_FEATURES", np.float32).reshape(-1, 32)
        t = self.debug_read("LEARN_TARGETS", np.float32).reshape(-1, 6)
        return f, t

    def debug_read(self, name: str, dtype=np.uint8):
        lib = load_library()
        which = abi.BUF[name]
        n = lib.avbd_debug_buffer_size(self._h, which)
        buf = np.zeros(n, np.uint8)
        if n:
            self._check(lib.avbd_debug_read(self._h, which, buf.ctypes.data, n))
        return buf.view(dtype)


class _Snapshot:
    def __init__(self, h):
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.avbd_snapshot_free(self._h)
            self._h = None
