"""CPU oracle of the AVBD solver step — TEST INFRASTRUCTURE.

A serial C++ restatement of the reference solver path (see avbd_oracle.cpp).
Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
import this package; the product library never calls it.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "build", "liboracle.so")
SRC = [os.path.join(HERE, "avbd_oracle.cpp"), os.path.join(HERE, "oracle_cloth.cpp"),
       os.path.join(HERE, "oracle_render.cpp"),
       os.path.join(HERE, "oracle_solver.h"), os.path.join(HERE, "oracle_math.h"),
       os.path.join(HERE, "..", "include", "avbd.h")]


def build(force: bool = False) -> str:
    """Compile the oracle with IEEE float32 semantics (no FMA contraction)."""
    if not force and os.path.exists(LIB) and all(
            os.path.getmtime(LIB) >= os.path.getmtime(s) for s in SRC):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
           "-fPIC", "-shared", "-o", LIB, SRC[0], SRC[1], SRC[2]]
    subprocess.check_call(cmd)
    return LIB


_lib = None


def bind(cdll):
    """Declare the oracle's C entry points on a loaded library (the oracle
    alone, or the oracle linked with the reference kernels, oracle/ref.py)."""
    _lib = cdll
    _lib.oracle_create.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
    _lib.oracle_destroy.argtypes = [C.c_void_p]
    _lib.oracle_set_threads.argtypes = [C.c_void_p, C.c_int]
    _lib.oracle_set_settings.argtypes = [C.c_void_p, C.c_void_p]
    _lib.oracle_step.argtypes = [C.c_void_p, C.c_uint32]
    _lib.oracle_runtime_failure.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    _lib.oracle_get_positions.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
    _lib.oracle_get_body_states.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
    _lib.oracle_set_motor_targets.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
    for name in ("oracle_set_joint_world_anchors", "oracle_set_motor_velocities", "oracle_set_motor_torques"):
        getattr(_lib, name).argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
    _lib.oracle_get_motor_states.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
    _lib.oracle_build_instances.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32,
                                            C.c_void_p]
    _lib.oracle_soft_normals.argtypes = [C.c_void_p, C.c_float, C.c_void_p]
    _lib.oracle_set_skin_bindings.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
    _lib.oracle_skin_deform.argtypes = [C.c_void_p, C.c_void_p]
    _lib.oracle_render_pusht_obs.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p]
    _lib.oracle_max_constraint_error.argtypes = [C.c_void_p, C.POINTER(C.c_float)]
    _lib.oracle_set_residual_trace.argtypes = [C.c_void_p, C.c_int]
    _lib.oracle_get_residual_trace.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
    _lib.oracle_residual.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    _lib.oracle_get_counters.argtypes = [C.c_void_p, C.c_void_p]
    _lib.oracle_debug_buffer_size.argtypes = [C.c_void_p, C.c_int]
    _lib.oracle_debug_buffer_size.restype = C.c_size_t
    _lib.oracle_debug_read.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]
    _lib.oracle_atan2.argtypes = [C.c_float, C.c_float]
    _lib.oracle_set_capacity_for_testing.argtypes = [C.c_void_p, C.c_int, C.c_uint32]
    _lib.oracle_atan2.restype = C.c_float
    return _lib


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = bind(C.CDLL(LIB))
    return _lib


class OracleSolver:
    """Same surface as avbd_b200.GPUSolver, backed by the CPU oracle."""

    def __init__(self, scene, threads: int = 1, _library=None, **desc_kw):
        from avbd_b200 import abi  # noqa: WPS433 (package path set by caller)
        self._abi = abi
        self._L = _library if _library is not None else lib()
        self.scene = scene
        desc, self._keep = scene.to_desc(**desc_kw)
        self._desc = desc
        h = C.c_void_p()
        rc = self._L.oracle_create(C.byref(desc), C.byref(h))
        if rc != 0:
            raise RuntimeError(f"oracle_create failed: status {rc}")
        self._h = h
        self.num_bodies = scene and len(scene.bodies)
        self._L.oracle_set_threads(self._h, threads)

    def close(self):
        if getattr(self, "_h", None):
            self._L.oracle_destroy(self._h)
            self._h = None

    __del__ = close

    def step(self, frames: int = 1) -> int:
        return self._L.oracle_step(self._h, frames)

    def set_settings(self, settings):
        st = settings.to_c()
        self._L.oracle_set_settings(self._h, C.byref(st))

    def runtime_failure(self) -> int:
        k = C.c_int()
        self._L.oracle_runtime_failure(self._h, C.byref(k))
        return k.value

    def positions(self):
        n = self.num_bodies
        pos = np.zeros((n, 4), np.float32)
        rot = np.zeros((n, 4), np.float32)
        self._L.oracle_get_positions(self._h, n, pos.ctypes.data, rot.ctypes.data)
        return pos, rot

    def body_states(self):
        n = self.num_bodies
        out = (self._abi.BodyState * n)()
        self._L.oracle_get_body_states(self._h, n, out)
        return out

    def set_capacity_for_testing(self, which: int, value: int):
        return self._L.oracle_set_capacity_for_testing(self._h, which, value)

    def set_motor_targets(self, joints, targets):
        ids = np.ascontiguousarray(joints, dtype=np.uint32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        self._L.oracle_set_motor_targets(self._h, ids.ctypes.data, len(ids), t.ctypes.data)

    def set_joint_world_anchors(self, joints, points):
        ids = np.ascontiguousarray(joints, dtype=np.uint32)
        p = np.ascontiguousarray(points, dtype=np.float32).reshape(-1)
        self._L.oracle_set_joint_world_anchors(self._h, ids.ctypes.data, len(ids), p.ctypes.data)

    def set_motor_velocities(self, joints, rad_per_s):
        ids = np.ascontiguousarray(joints, dtype=np.uint32)
        v = np.ascontiguousarray(rad_per_s, dtype=np.float32)
        self._L.oracle_set_motor_velocities(self._h, ids.ctypes.data, len(ids), v.ctypes.data)

    def set_motor_torques(self, joints, torques):
        ids = np.ascontiguousarray(joints, dtype=np.uint32)
        t = np.ascontiguousarray(torques, dtype=np.float32)
        self._L.oracle_set_motor_torques(self._h, ids.ctypes.data, len(ids), t.ctypes.data)

    def build_instances(self, colliders, colors=None, color_mode: int = 0):
        ids = np.ascontiguousarray(colliders, dtype=np.uint32)
        col = None if colors is None else np.ascontiguousarray(colors, dtype=np.float32).reshape(-1, 4)
        out = np.zeros((len(ids), 24), np.float32)
        self._L.oracle_build_instances(self._h, ids.ctypes.data, len(ids), None if col is None else col.ctypes.data,
                                     color_mode, out.ctypes.data)
        return out

    def soft_normals(self, cloth_scale: float = 0.0, out=None):
        res = np.zeros((self.num_bodies, 4), np.float32) if out is None else np.ascontiguousarray(out, np.float32)
        self._L.oracle_soft_normals(self._h, cloth_scale, res.ctypes.data)
        return res

    def set_skin_bindings(self, bindings):
        arr = (self._abi.SkinBinding * len(bindings))(*bindings)
        self._num_skin = len(bindings)
        rc = self._L.oracle_set_skin_bindings(self._h, arr, len(bindings))
        if rc != 0:
            raise RuntimeError(f"oracle_set_skin_bindings failed: {rc}")

    def skin_deform(self):
        out = np.zeros((getattr(self, "_num_skin", 0), 8), np.float32)
        self._L.oracle_skin_deform(self._h, out.ctypes.data)
        return out

    def render_pusht_obs(self, envs, res: int = 64):
        arr = envs if isinstance(envs, C.Array) else (self._abi.PushTEnv * len(envs))(*envs)
        out = np.zeros((len(envs), res, res, 3), np.uint8)
        self._L.oracle_render_pusht_obs(self._h, arr, len(envs), res, out.ctypes.data)
        return out

    def motor_states(self, joints):
        ids = np.ascontiguousarray(joints, dtype=np.uint32)
        a = np.zeros(len(ids), np.float32)
        v = np.zeros(len(ids), np.float32)
        self._L.oracle_get_motor_states(self._h, ids.ctypes.data, len(ids), a.ctypes.data, v.ctypes.data)
        return a, v

    def max_constraint_error(self) -> float:
        v = C.c_float()
        self._L.oracle_max_constraint_error(self._h, C.byref(v))
        return v.value

    def set_residual_trace(self, enabled: bool) -> None:
        self._L.oracle_set_residual_trace(self._h, 1 if enabled else 0)

    def residual_trace(self, n: int) -> np.ndarray:
        out = np.zeros(n, np.float64)
        self._L.oracle_get_residual_trace(self._h, out.ctypes.data, n)
        return out

    def residual(self) -> float:
        v = C.c_double()
        self._L.oracle_residual(self._h, C.byref(v))
        return v.value

    def counters(self):
        c = self._abi.Counters()
        self._L.oracle_get_counters(self._h, C.byref(c))
        return c

    def debug_read(self, name: str, dtype=np.uint8):
        which = self._abi.BUF[name]
        n = self._L.oracle_debug_buffer_size(self._h, which)
        buf = np.zeros(n, np.uint8)
        if n:
            rc = self._L.oracle_debug_read(self._h, which, buf.ctypes.data, n)
            if rc != 0:
                raise RuntimeError(f"oracle_debug_read({name}) failed: {rc}")
        return buf.view(dtype)
