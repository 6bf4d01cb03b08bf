"""Oracle B: the reference's CPU solver restated in C++ — TEST INFRASTRUCTURE
and the CPU baseline of the rigid-stack workload.

The reference's rigid-only CPU solver (Sources/PhysicsAVBD/CPU/CPUSolver.swift,
the "ground truth" of its Metal solver) differs from the GPU path by design
(O(n^2) broadphase, body-order Gauss-Seidel, unpreconditioned LDL^T, no
speculative margin), so it is not the CUDA path's parity oracle; see
cpu_solver.cpp.  Only tests/ and bench.py's CPU legs use it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from . import HERE

SRC = os.path.join(HERE, "cpu_solver.cpp")
LIB = os.path.join(HERE, "build", "libcpu_solver.so")


def build(force: bool = False) -> str:
    deps = [SRC, os.path.join(HERE, "..", "include", "avbd.h")]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
                           "-o", LIB, SRC])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        L.cpu_solver_create.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
        L.cpu_solver_destroy.argtypes = [C.c_void_p]
        L.cpu_solver_step.argtypes = [C.c_void_p, C.c_uint32]
        L.cpu_solver_get_body_states.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
        L.cpu_solver_max_constraint_error.argtypes = [C.c_void_p]
        L.cpu_solver_max_constraint_error.restype = C.c_float
        L.cpu_solver_num_forces.argtypes = [C.c_void_p]
        L.cpu_solver_num_forces.restype = C.c_uint32
        _lib = L
    return _lib


class CPUSolver:
    """PhysicsScene.makeCPUSolver() (CPU/PhysicsScene+CPUSolver.swift:5-62)."""

    def __init__(self, scene):
        from avbd_b200 import abi
        self._abi = abi
        desc, self._keep = scene.to_desc()
        h = C.c_void_p()
        rc = lib().cpu_solver_create(C.byref(desc), C.byref(h))
        if rc != 0:
            raise RuntimeError(f"cpu_solver_create: status {rc} (only box/sphere rigid scenes are restated)")
        self._h = h
        self.num_bodies = len(scene.bodies)

    def close(self):
        if getattr(self, "_h", None):
            lib().cpu_solver_destroy(self._h)
            self._h = None

    __del__ = close

    def step(self, frames: int = 1) -> int:
        return lib().cpu_solver_step(self._h, frames)

    def set_motor_targets(self, joints, targets):
        raise NotImplementedError("the reference CPU solver has no joint motors")

    def body_states(self):
        out = (self._abi.BodyState * self.num_bodies)()
        lib().cpu_solver_get_body_states(self._h, self.num_bodies, out)
        return out

    def positions(self):
        st = self.body_states()
        pos = np.array([list(s.position) for s in st], np.float32)
        rot = np.array([list(s.rotation) for s in st], np.float32)
        return pos, rot

    def max_constraint_error(self) -> float:
        return lib().cpu_solver_max_constraint_error(self._h)

    def num_forces(self) -> int:
        return lib().cpu_solver_num_forces(self._h)
