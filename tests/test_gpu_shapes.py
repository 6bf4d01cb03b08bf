"""Tori, capsules and convex hulls: the CUDA solver against the CPU oracle,
through the C ABI.  Trajectories are compared every frame (bit-identical in
practice; the tolerance is 1e-4 relative), the contact records of the round
shapes bitwise, and the reference's known-answer gates are rerun on the GPU
path."""
import numpy as np
import pytest

from avbd_b200 import abi, demos
from avbd_b200.solver import AVBDError, GPUSolver

from test_gpu_parity import compare_state, pair

pytestmark = pytest.mark.gpu


def _oracle_scenes():
    import test_oracle_shapes
    return test_oracle_shapes


def manifolds_equal(g, o):
    gm = g.debug_read("MANIFOLDS", np.uint32).reshape(-1, 176)
    om = o.debug_read("MANIFOLDS", np.uint32).reshape(-1, 176)
    assert gm.shape == om.shape
    active = 0
    for r in range(gm.shape[0]):
        n = gm[r, 2]
        assert np.array_equal(gm[r, :8], om[r, :8]), f"manifold {r} header"
        if n:
            active += 1
            assert np.array_equal(gm[r, :16 + 20 * n], om[r, :16 + 20 * n]), f"manifold {r}"
    return active


@pytest.mark.parametrize("name,make,frames", [
    ("torus-rest", demos.torus_rest_scene, 400),
    ("linked-tori", demos.linked_tori_scene, 420),
    ("ring-catch", demos.ring_catch_scene, 240),
    ("bearing", demos.bearing_scene, 300),
    ("hull-box", demos.hull_box_scene, 360),
    ("chainmail-5", lambda: demos.chainmail_scene(rings=5, drops=3), 300),
    ("shapes-64", lambda: demos.shapes_scene(count=64), 200),
    ("drape-capsule", lambda: demos.drape_scene(res=16, obstacle="capsule"), 90),
    ("drape-torus", lambda: demos.drape_scene(res=16, obstacle="torus"), 90),
    ("capsule-rest", lambda: _oracle_scenes().capsule_rest_scene(), 240),
    ("crossed-capsules", lambda: _oracle_scenes().crossed_capsules_scene(), 240),
    ("ball-on-capsule", lambda: _oracle_scenes().ball_on_capsule_scene(), 180),
    ("hull-stack", lambda: _oracle_scenes().hull_stack_scene(), 240),
])
def test_shape_trajectory_parity(cuda_lib, oracle_lib, name, make, frames):
    g, o = pair(make(), oracle_lib)
    exact = 0
    for f in range(frames):
        g.step(1)
        assert o.step(1) == 0
        exact += compare_state(g, o, f + 1)
        if (f + 1) % 50 == 0 or f + 1 == frames:
            manifolds_equal(g, o)
            gc, oc = g.counters(), o.counters()
            assert (gc.num_pairs, gc.num_soft) == (oc.num_pairs, oc.num_soft), f"frame {f + 1}"
    print(f"{name}: {exact}/{frames} frames bit-identical")
    assert g.runtime_failure() == 0


def test_round_contacts_bitwise(cuda_lib, oracle_lib):
    """Every torus/capsule/hull pair kind with contacts at once: the records
    (feature keys, anchors, warm-started duals) match bit for bit."""
    g, o = pair(demos.shapes_scene(count=96), oracle_lib)
    g.step(120)
    assert o.step(120) == 0
    g.synchronize()
    assert manifolds_equal(g, o) > 50
    types = g.debug_read("PAIRS", np.uint32)
    assert types.size > 0


def test_capsule_foot_holds_on_gpu(cuda_lib, oracle_lib):
    """GPUSolverTests.swift:577-620 on the CUDA path, with the joint anchor
    moved every frame through the C ABI; the oracle follows the same
    commands and the trajectories agree."""
    g, o = pair(demos.capsule_foot_scene(), oracle_lib)
    g.step(600)
    assert o.step(600) == 0
    compare_state(g, o, 600)
    settled = g.positions()[0][1, :3].copy()
    for f in range(1200):
        p = g.positions()[0][1]
        pt = [float(p[0]) + 0.04, float(p[1]), float(p[2])]
        g.set_joint_world_anchors([0], pt)
        o.set_joint_world_anchors([0], pt)
        g.step(1)
        assert o.step(1) == 0
    compare_state(g, o, 1800)
    pos, _ = g.positions()
    v = np.asarray(g.body_states()[1].velocity)
    assert abs(pos[1, 0] - settled[0]) < 0.001
    assert np.linalg.norm(v) < 0.03


def test_chainmail_hangs_on_gpu(cuda_lib):
    # TorusAndMachineTests.swift:45-57
    s = demos.chainmail_scene(rings=5, drops=3)
    rings = [i for i, b in enumerate(s.bodies) if b.shape == abi.SHAPE_TORUS]
    g = GPUSolver(s)
    g.step(700)
    pos, _ = g.positions()
    assert (pos[rings, 2] > 4.5).all()
    assert int((pos[-3:, 2] > 4.0).sum()) >= 2


def test_motor_setters_parity(cuda_lib, oracle_lib):
    """Velocity commands, effort limits and motor states through the C ABI
    follow the oracle."""
    from test_oracle_shapes import hinge_scene
    g, o = pair(hinge_scene(abi.MOTOR_VELOCITY), oracle_lib)
    for solver in (g, o):
        solver.set_motor_velocities([0], [2.0])
    for f in range(90):
        g.step(1)
        assert o.step(1) == 0
        if f == 59:
            for solver in (g, o):
                solver.set_motor_torques([0], [0.5])
    compare_state(g, o, 90)
    ga, gv = g.motor_states([0])
    oa, ov = o.motor_states([0])
    assert np.array_equal(ga.view(np.uint32), oa.view(np.uint32))
    assert np.array_equal(gv.view(np.uint32), ov.view(np.uint32))
    assert abs(gv[0] - 2.0) < 0.3


def test_setter_validation(cuda_lib):
    g = GPUSolver(demos.torus_rest_scene())
    with pytest.raises(AVBDError):
        g.set_motor_velocities([0], [1.0])  # no joints at all
    from test_oracle_shapes import hinge_scene
    h = GPUSolver(hinge_scene(abi.MOTOR_IMPLICIT_POSITION_PD))
    with pytest.raises(AVBDError):
        h.set_motor_velocities([0], [1.0])  # not a velocity motor
    with pytest.raises(AVBDError):
        h.set_motor_torques([0], [-1.0])
    with pytest.raises(AVBDError):
        h.set_joint_world_anchors([0], [float("nan"), 0.0, 0.0])
    h.set_motor_torques([0], [1.0])
    h.step(2)


def test_invalid_hulls_refused(cuda_lib):
    s = demos.hull_box_scene()
    s.colliders[-1].hull_vertices = s.colliders[-1].hull_vertices[:3]
    with pytest.raises(AVBDError):
        GPUSolver(s)
    s = demos.hull_box_scene()
    s.colliders[-1].hull_vertices[0] = (float("inf"), 0.0, 0.0)
    with pytest.raises(AVBDError):
        GPUSolver(s)
