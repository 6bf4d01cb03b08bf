"""Oracle B — the reference's CPU solver restated (oracle/cpu_solver.cpp) —
against the reference's own CPU known-answer gates, and against Oracle A (the
GPU-path restatement) with the tolerance the reference itself uses between
its CPU and GPU solvers.

Gates restated from Tests/PhysicsAVBDTests/CPUSolverTests.swift:35-98 and the
CPU/GPU parity test GPUSolverTests.swift:831-846 (3-box stack, 120 frames,
per-body |dx| < 0.05 m); the two solvers differ by design (broadphase,
Gauss-Seidel order, preconditioning, speculative margin).
"""
import numpy as np
import pytest

from avbd_b200 import demos
from avbd_b200.scene import PhysicsScene, SceneJoint

cs = pytest.importorskip("oracle.cpu_solver")


def cpu(scene, frames):
    o = cs.CPUSolver(scene)
    assert o.step(frames) == 0
    return o


def test_box_rests_on_ground():
    s = PhysicsScene("rest")
    s.add_body((100, 100, 1), 0.0, 0.5, (0, 0, -0.5))
    b = s.add_body((1, 1, 1), 1.0, 0.5, (0, 0, 0.6))
    st = cpu(s, 120).body_states()[b]
    assert abs(st.position[2] - 0.5) < 0.03
    assert np.linalg.norm(st.velocity[:]) < 0.05


def test_free_fall_matches_implicit_euler():
    s = PhysicsScene("fall")
    b = s.add_body((1, 1, 1), 1.0, 0.5, (0, 0, 100))
    o = cpu(s, 30)
    v, z = 0.0, 100.0
    for _ in range(30):
        v += s.settings.gravity * s.settings.dt
        z += v * s.settings.dt
    assert abs(o.body_states()[b].position[2] - z) < 0.01


def test_pendulum_joint_error():
    s = PhysicsScene("pendulum")
    bob = s.add_body((0.5, 0.5, 0.5), 1.0, 0.5, (1, 0, 0))
    s.add_joint(SceneJoint(-1, bob, (0, 0, 0), (-1, 0, 0)))
    assert cpu(s, 120).max_constraint_error() < 0.01


def test_small_stack_stability():
    s = PhysicsScene("stack5")
    s.settings.iterations = 10
    s.add_body((100, 100, 1), 0.0, 0.7, (0, 0, -0.5))
    ids = [s.add_body((1, 1, 1), 1.0, 0.7, (0, 0, 0.5 + i)) for i in range(5)]
    st = cpu(s, 300).body_states()
    for i, b in enumerate(ids):
        assert abs(st[b].position[2] - (0.5 + i)) < 0.08


def test_rigid_stack_20_stands():
    """The rigid-stack benchmark scene (20 unit cubes, 10 iterations) over
    its 300 frames: every cube stays within 0.1 m of its column and rests at
    its stack height within the reference's 0.08 m stack gate per level."""
    s = demos.rigid_stack_scene(seed=1)
    st = cpu(s, 300).body_states()
    for i in range(20):
        p = st[1 + i].position
        assert abs(p[0]) < 0.1 and abs(p[1]) < 0.1
        assert abs(p[2] - (0.5 + i * (1.0 + 1e-3))) < 0.08 * (i + 1)


def test_cpu_and_gpu_path_agree_to_the_references_tolerance(oracle_lib):
    """GPUSolverTests.swift:831-846: 3-box stack, 120 frames, per-body
    position difference below 5 cm between the CPU solver and the GPU path."""
    s = demos.stack(3)
    a = cs.CPUSolver(s)
    b = oracle_lib.OracleSolver(s)
    for _ in range(120):
        a.step(1)
        b.step(1)
    pa, _ = a.positions()
    pb, _ = b.positions()
    assert np.max(np.linalg.norm(pa[:, :3] - pb[:, :3], axis=1)) < 0.05
