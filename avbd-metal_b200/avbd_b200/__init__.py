"""avbd_b200 — the AVBD solver step (augmented vertex block descent) on
NVIDIA B200 (sm_100a CUDA kernels behind a C ABI, include/avbd.h).

Python host mirror of the reference's scene/step API:
  PhysicsScene / SimSettings  (Sources/SimCore/Scenes/Scene.swift)
  GPUSolver                   (Sources/PhysicsAVBD/GPU/GPUSolver.swift)
"""
from . import abi, demos
from .scene import (PhysicsScene, SceneBody, SceneCollider, SceneJoint, SceneSpinner,
                    SceneSpring, SceneTet, SceneTri, SimSettings)
from .solver import AVBDError, GPUSolver, RuntimeFailure, library_path, load_library

__all__ = [
    "abi", "demos", "PhysicsScene", "SceneBody", "SceneCollider", "SceneJoint", "SceneSpinner",
    "SceneSpring", "SceneTet", "SceneTri", "SimSettings", "GPUSolver", "AVBDError",
    "RuntimeFailure", "library_path", "load_library",
]
