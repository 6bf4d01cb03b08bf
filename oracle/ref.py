"""The reference's own kernels beside the oracle — TEST INFRASTRUCTURE.

`build()` compiles, in this container only (where the reference's sources
are present), one shared library into `oracle/_ref/`: the oracle's sources
plus `ref_pin.cpp`, which includes the reference's shader files
`Sources/PhysicsAVBD/Shaders/*.metal` unchanged, from where they lie, as C++
through the Metal stand-in header `msl/metal_stdlib`.  Nothing of the
reference is copied into this repository; the library is git-ignored.

`PinnedOracle` is an oracle solver whose every frame is also computed stage by
stage by the reference's kernels on the same state (warm start, narrowphase,
persistence map, adjacency, the split primal of every color, the dual,
finalize) and compared word for word; `stats()` reports per stage how many
records were compared and how many differed.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from . import HERE, OracleSolver, bind

REFERENCE_SHADERS = "/root/reference/Sources/PhysicsAVBD/Shaders"
OUT = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT, "liboracle_ref.so")
SRC = [os.path.join(HERE, f) for f in ("avbd_oracle.cpp", "oracle_cloth.cpp", "oracle_render.cpp", "ref_pin.cpp")]
DEPS = SRC + [os.path.join(HERE, f) for f in ("oracle_solver.h", "oracle_math.h", os.path.join("msl", "metal_stdlib"))]
STAGES = ["broadphase", "narrowphase", "map", "warm_joints", "warm_bodies", "adjacency", "coloring", "primal",
          "dual", "finalize"]


def available() -> bool:
    """The reference's shader sources are readable (this container only)."""
    return os.path.isdir(REFERENCE_SHADERS)


def build(force: bool = False) -> str:
    if os.path.exists(LIB) and not force and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in DEPS):
        return LIB
    if not available():
        raise FileNotFoundError(f"reference shader sources not found at {REFERENCE_SHADERS}")
    os.makedirs(OUT, exist_ok=True)
    cmd = ["g++", "-O2", "-std=c++20", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared",
           "-Wno-attributes", "-I", os.path.join(HERE, "msl"), "-I", REFERENCE_SHADERS, "-o", LIB] + SRC
    subprocess.check_call(cmd)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = bind(C.CDLL(LIB))
        _lib.ref_pin_attach.argtypes = [C.c_void_p, C.c_uint32]
        _lib.ref_pin_attach.restype = C.c_void_p
        _lib.ref_pin_detach.argtypes = [C.c_void_p, C.c_void_p]
        _lib.ref_pin_stats.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
        _lib.ref_pin_diag_error.argtypes = [C.c_void_p]
        _lib.ref_pin_diag_error.restype = C.c_float
        _lib.ref_pin_perturb_for_testing.argtypes = [C.c_void_p, C.c_int]
    return _lib


class PinnedOracle(OracleSolver):
    """An oracle solver whose stages are re-run by the reference's kernels."""

    def __init__(self, scene, threads: int = 1, primal_every: int = 1, **desc_kw):
        super().__init__(scene, threads=threads, _library=lib(), **desc_kw)
        self._pin = self._L.ref_pin_attach(self._h, primal_every)

    def close(self):
        if getattr(self, "_pin", None):
            self._L.ref_pin_detach(self._h, self._pin)
            self._pin = None
        super().close()

    __del__ = close

    def stats(self) -> dict:
        out = np.zeros(6 * len(STAGES), np.float64)
        self._L.ref_pin_stats(self._pin, out.ctypes.data, len(out))
        return {name: {"calls": int(out[6 * k]), "compared": int(out[6 * k + 1]),
                       "mismatched": int(out[6 * k + 2]), "max_rel": float(out[6 * k + 3]),
                       "first_bad_frame": int(out[6 * k + 4]), "first_bad_index": int(out[6 * k + 5])}
                for k, name in enumerate(STAGES)}

    def perturb_for_testing(self, stage: str) -> None:
        self._L.ref_pin_perturb_for_testing(self._pin, STAGES.index(stage))

    def reference_diag_error(self) -> float:
        return self._L.ref_pin_diag_error(self._pin)
