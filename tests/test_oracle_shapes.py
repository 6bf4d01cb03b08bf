"""Tori, capsules and convex hulls on the CPU oracle, against the
reference's own known-answer tests for them (TorusAndMachineTests.swift,
GPUSolverTests.swift:537-620).  Each test restates one gate: its scene, frame
count, expectation and tolerance."""
import math

import numpy as np
import pytest

from avbd_b200 import abi, demos
from avbd_b200.scene import PhysicsScene, SceneJoint


def run(oracle_lib, scene, frames):
    o = oracle_lib.OracleSolver(scene, threads=1)
    for f in range(frames):
        assert o.step(1) == 0, f"frame {f + 1}: failure {o.runtime_failure()}"
    return o


def rotate(q, v):
    u = np.asarray(q[:3], np.float64)
    t = 2.0 * np.cross(u, v)
    return np.asarray(v, np.float64) + q[3] * t + np.cross(u, t)


def test_torus_rests_flat(oracle_lib):
    # TorusAndMachineTests.swift:7-15
    o = run(oracle_lib, demos.torus_rest_scene(), 400)
    pos, rot = o.positions()
    assert abs(pos[1, 2] - 0.12) <= 0.1, pos[1]
    assert abs(rotate(rot[1], (0, 0, 1))[2]) > 0.95


def test_interlocked_tori_hold_weight(oracle_lib):
    # TorusAndMachineTests.swift:17-30
    o = run(oracle_lib, demos.linked_tori_scene(), 420)
    pos, _ = o.positions()
    assert pos[-1, 2] > 3.0, "linked tori must carry 1 kg"


def test_sphere_caught_in_ring(oracle_lib):
    # TorusAndMachineTests.swift:32-41
    o = run(oracle_lib, demos.ring_catch_scene(), 240)
    pos, _ = o.positions()
    assert pos[2, 2] > 0.8, "ball should rest inside the ring"


def test_capsule_torus_bearing(oracle_lib):
    # TorusAndMachineTests.swift:88-102: hang offset (0.27 - 0.115) - 0.11
    o = run(oracle_lib, demos.bearing_scene(), 300)
    pos, _ = o.positions()
    assert abs(pos[1, 2] - (3.0 - 0.045)) <= 0.02, pos[1]


def test_chainmail_hangs_on_pegs(oracle_lib):
    # TorusAndMachineTests.swift:45-57
    s = demos.chainmail_scene(rings=5, drops=3)
    rings = [i for i, b in enumerate(s.bodies) if b.shape == abi.SHAPE_TORUS]
    o = run(oracle_lib, s, 700)
    pos, _ = o.positions()
    assert (pos[rings, 2] > 4.5).all(), "a ring fell out of the sheet"
    assert int((pos[-3:, 2] > 4.0).sum()) >= 2, "mail should catch the dropped objects"


def test_convex_hull_rests_on_box_terrain(oracle_lib):
    # GPUSolverTests.swift:537-571
    s = demos.hull_box_scene()
    c = s.colliders[-1]
    assert len(c.hull_vertices) == 8 and c.size == (1.0, 1.0, 1.0)
    o = run(oracle_lib, s, 360)
    pos, rot = o.positions()
    assert abs(pos[1, 2] - 0.5) <= 0.06, pos[1]
    assert abs(rot[1, 0]) < 0.05 and abs(rot[1, 1]) < 0.05
    m = o.debug_read("MANIFOLDS", np.uint32).reshape(-1, 176)
    active = {(int(r[0]), int(r[1])) for r in m if r[2] > 0}
    assert (0, 1) in active or (1, 0) in active


def test_compound_capsule_foot_holds(oracle_lib):
    # GPUSolverTests.swift:577-620: a 20 N pull below the ~55 N Coulomb
    # limit; the anchor of the spring follows the foot 4 cm ahead
    o = run(oracle_lib, demos.capsule_foot_scene(), 600)
    settled = o.positions()[0][1, :3].copy()
    for _ in range(1200):
        p = o.positions()[0][1]
        o.set_joint_world_anchors([0], [p[0] + 0.04, p[1], p[2]])
        assert o.step(1) == 0
    pos, _ = o.positions()
    v = np.asarray(o.body_states()[1].velocity)
    assert abs(pos[1, 0] - settled[0]) < 0.001, "compound capsule foot crept under a sub-Coulomb load"
    assert np.linalg.norm(v) < 0.03


def test_hull_contacts_only_boxes(oracle_lib):
    """A hull meets boxes only (30_narrowphase.metal:433-440): a hull body
    dropped on a static sphere passes through it and lands on the ground."""
    s = PhysicsScene("hull-sphere")
    demos.add_ground(s)
    s.add_sphere(0.6, 0.0, 0.5, (0, 0, 0.3))
    b = s.add_body((1, 1, 1), 0.0, 0.5, (0, 0, 1.5), mass=1.0, diagonal_inertia=(0.2, 0.2, 0.2),
                   collision_enabled=False)
    s.add_convex_collider(b, [(0.3, 0, 0), (-0.3, 0, 0), (0, 0.3, 0), (0, -0.3, 0), (0, 0, 0.3), (0, 0, -0.3)])
    o = run(oracle_lib, s, 240)
    pos, _ = o.positions()
    assert abs(pos[b, 2] - 0.3) < 0.05, pos[b]


@pytest.mark.parametrize("obstacle", ["capsule", "torus"])
def test_drape_over_round_obstacles(oracle_lib, obstacle):
    """Cloth over a static capsule (its three feature spheres meet the
    triangles) and over a flat ring (particle-torus contacts only): the
    sheet stays finite and parts of it rest on the obstacle."""
    o = run(oracle_lib, demos.drape_scene(res=16, obstacle=obstacle), 90)
    pos, _ = o.positions()
    cloth = pos[2:, 2]
    assert np.isfinite(pos).all()
    assert cloth.max() > 0.9 and cloth.min() > -0.05
    if obstacle == "capsule":
        assert o.counters().num_soft > 0


def test_shapes_pile_settles(oracle_lib):
    o = run(oracle_lib, demos.shapes_scene(count=48), 150)
    pos, _ = o.positions()
    assert np.isfinite(pos).all()
    assert pos[1:, 2].min() > -0.1
    assert o.counters().num_pairs > 40


def test_hull_vertex_count_and_shape_refusals(oracle_lib):
    s = demos.hull_box_scene()
    s.colliders[-1].hull_vertices = s.colliders[-1].hull_vertices[:3]
    with pytest.raises(RuntimeError):
        oracle_lib.OracleSolver(s)
    s = demos.hull_box_scene()
    s.colliders[-1].hull_vertices[0] = (float("nan"), 0.0, 0.0)
    with pytest.raises(RuntimeError):
        oracle_lib.OracleSolver(s)
    s = demos.torus_rest_scene()
    s.bodies[1].shape = 7
    with pytest.raises(RuntimeError):
        oracle_lib.OracleSolver(s)
    with pytest.raises(ValueError):
        demos.hull_box_scene().add_convex_collider(1, [(0, 0, 0)] * 65)


def hinge_scene(mode):
    s = PhysicsScene("hinge")
    s.settings.gravity = 0.0
    s.add_body((0.2, 0.2, 0.2), 0.0, 0.5, (0, 0, 1))
    b = s.add_body((0.6, 0.1, 0.1), 100.0, 0.5, (0.3, 0, 1))
    s.add_joint(SceneJoint(0, b, (0, 0, 0), (-0.3, 0, 0), stiffness_lin=float("inf"), stiffness_ang=float("inf"),
                           hinge_axis=(0, 0, 1), motor_torque=2.0, motor_stiffness=5.0, motor_damping=0.5,
                           motor_mode=mode))
    s.add_collision_exclusion(0, b)
    return s


def test_motor_velocity_torque_and_states(oracle_lib):
    """Velocity motor commands, effort limits and the hinge state read back
    (GPUSolver.swift:2534-2637): a commanded 2 rad/s spins the hinge at
    about that rate; zero effort stops driving it."""
    o = oracle_lib.OracleSolver(hinge_scene(abi.MOTOR_VELOCITY), threads=1)
    o.set_motor_velocities([0], [2.0])
    assert o.step(60) == 0
    a0, v0 = o.motor_states([0])
    assert abs(v0[0] - 2.0) < 0.2, v0
    assert o.step(30) == 0
    a1, _ = o.motor_states([0])
    d = math.remainder(float(a1[0] - a0[0]), 2 * math.pi)
    assert abs(d - 1.0) < 0.15, d
    o.set_motor_torques([0], [0.0])
    o.set_motor_velocities([0], [-3.0])
    assert o.step(30) == 0
    _, v2 = o.motor_states([0])
    assert v2[0] > 0.0, "with zero effort the motor no longer drives the hinge"



def capsule_rest_scene():
    s = PhysicsScene("capsule-rest")
    demos.add_ground(s, friction=0.6)
    s.add_capsule(0.8, 0.15, 1.0, 0.6, (0, 0, 0.6), rotation=demos.quat_axis_angle(math.pi / 2, (0, 1, 0)))
    return s


def crossed_capsules_scene():
    s = PhysicsScene("capsule-cross")
    demos.add_ground(s)
    s.add_capsule(1.0, 0.1, 0.0, 0.6, (0, 0, 0.1), rotation=demos.quat_axis_angle(math.pi / 2, (0, 1, 0)))
    s.add_capsule(1.0, 0.12, 1.0, 0.6, (0, 0, 0.6), rotation=demos.quat_axis_angle(math.pi / 2, (1, 0, 0)))
    return s


def ball_on_capsule_scene():
    s = PhysicsScene("ball-on-capsule")
    demos.add_ground(s)
    s.add_capsule(1.2, 0.2, 0.0, 0.8, (0, 0, 1.0), rotation=demos.quat_axis_angle(math.pi / 2, (0, 1, 0)))
    s.add_sphere(0.3, 1.0, 0.8, (0.0, 0.0, 1.6))
    return s


def hull_stack_scene():
    s = PhysicsScene("hull-hull")
    demos.add_ground(s)
    octa = [(0.3, 0, 0), (-0.3, 0, 0), (0, 0.3, 0), (0, -0.3, 0), (0, 0, 0.3), (0, 0, -0.3)]
    base = s.add_body((1, 1, 1), 0.0, 0.5, (0, 0, 0.3), collision_enabled=False)
    s.add_convex_collider(base, octa)
    b = s.add_body((1, 1, 1), 0.0, 0.5, (0, 0, 1.2), mass=1.0, diagonal_inertia=(0.2, 0.2, 0.2),
                   collision_enabled=False)
    s.add_convex_collider(b, octa)
    return s


def test_capsule_rests_on_its_side(oracle_lib):
    """A horizontal capsule dropped on the ground settles with its axis one
    radius above it and stays horizontal (capsule-box three-seed contact)."""
    o = run(oracle_lib, capsule_rest_scene(), 240)
    pos, rot = o.positions()
    assert abs(pos[1, 2] - 0.15) < 0.01, pos[1]
    assert abs(rotate(rot[1], (0, 0, 1))[2]) < 0.05  # axis stays horizontal


def test_crossed_capsules_stack(oracle_lib):
    """A capsule dropped crosswise on a static one rests with the axes two
    radii apart (capsule-capsule closest points)."""
    o = run(oracle_lib, crossed_capsules_scene(), 240)
    pos, _ = o.positions()
    assert abs(pos[2, 2] - (0.1 + 0.1 + 0.12)) < 0.015, pos[2]
    assert abs(pos[2, 0]) < 0.05 and abs(pos[2, 1]) < 0.05


def test_sphere_rests_on_capsule(oracle_lib):
    """A ball on top of a static horizontal capsule: centre at the capsule
    axis height plus both radii (capsule-sphere)."""
    o = run(oracle_lib, ball_on_capsule_scene(), 180)
    pos, _ = o.positions()
    assert abs(pos[2, 2] - (1.0 + 0.2 + 0.15)) < 0.01, pos[2]


def test_hulls_do_not_collide_with_each_other(oracle_lib):
    """Hull-hull pairs produce no contact (30_narrowphase.metal:433-440): a
    hull body falls through a static hull onto the ground."""
    o = run(oracle_lib, hull_stack_scene(), 240)
    pos, _ = o.positions()
    assert abs(pos[2, 2] - 0.3) < 0.05, pos[2]
