"""The oracle against the reference's own known-answer tests.

The reference ships no golden data files or stored trajectories; its pins
are analytic gates in its test suite.  Each test below restates one of them
(expectation and tolerance) and checks the CPU oracle against it.  This is
what pins the oracle to the reference's behaviour.
"""
import math

import numpy as np
import pytest

from avbd_b200 import abi, demos
from avbd_b200.scene import PhysicsScene, SceneJoint, SceneSpring, SceneTet


def run(oracle_lib, scene, frames, **kw):
    o = oracle_lib.OracleSolver(scene, **kw)
    assert o.step(frames) == 0, o.runtime_failure()
    return o


def test_friction_combine_modes(oracle_lib):
    # CPUSolverTests.swift:7-15: geometric, multiply, min, max, average
    for mode, want in [(0, math.sqrt(0.4)), (1, 0.4), (2, 0.5), (3, 0.8), (4, 0.65)]:
        s = PhysicsScene("friction")
        demos.add_ground(s, friction=0.8)
        s.add_body((1, 1, 1), 1.0, 0.5, (0, 0, 0.5))
        s.settings.friction_combine_mode = mode
        o = run(oracle_lib, s, 1)
        m = o.debug_read("MANIFOLDS", np.float32).reshape(-1, 176)
        active = [r for r in m if r.view(np.uint32)[2] > 0]
        assert active, "box on ground must produce a manifold"
        # basisT1.w = static friction (combined)
        assert abs(active[0][11] - want) < 1e-6


def test_box_rests_on_ground(oracle_lib):
    # CPUSolverTests.swift:35-47: z = 0.5 +- 0.03, |v| < 0.05 after 120 frames
    s = PhysicsScene("rest")
    s.add_body((100, 100, 1), 0.0, 0.5, (0, 0, -0.5))
    b = s.add_body((1, 1, 1), 1.0, 0.5, (0, 0, 0.6))
    o = run(oracle_lib, s, 120)
    st = o.body_states()[b]
    assert abs(st.position[2] - 0.5) < 0.03
    assert np.linalg.norm(st.velocity[:]) < 0.05


def test_free_fall_matches_implicit_euler(oracle_lib):
    # CPUSolverTests.swift:50-64 / GPUSolverTests.swift:470: v += g dt; z += v dt
    s = PhysicsScene("fall")
    b = s.add_body((1, 1, 1), 1.0, 0.5, (0, 0, 100))
    o = run(oracle_lib, s, 30)
    v, z = 0.0, 100.0
    for _ in range(30):
        v += s.settings.gravity * s.settings.dt
        z += v * s.settings.dt
    assert abs(o.body_states()[b].position[2] - z) < 0.01


def test_pendulum_joint_error(oracle_lib):
    # CPUSolverTests.swift:66-76: world-anchored 1 m arm, error < 1 cm
    s = PhysicsScene("pendulum")
    bob = s.add_body((0.5, 0.5, 0.5), 1.0, 0.5, (1, 0, 0))
    s.add_joint(SceneJoint(-1, bob, (0, 0, 0), (-1, 0, 0)))
    o = run(oracle_lib, s, 120)
    assert o.max_constraint_error() < 0.01


def test_small_stack_stability(oracle_lib):
    # CPUSolverTests.swift:79-98: 5 boxes, 10 iterations, 300 frames, +-0.08
    s = PhysicsScene("stack5")
    s.settings.iterations = 10
    s.add_body((100, 100, 1), 0.0, 0.7, (0, 0, -0.5))
    ids = [s.add_body((1, 1, 1), 1.0, 0.7, (0, 0, 0.5 + i)) for i in range(5)]
    o = run(oracle_lib, s, 300)
    st = o.body_states()
    for i, b in enumerate(ids):
        p = st[b].position
        assert abs(p[2] - (0.5 + i)) < 0.08
        assert math.hypot(p[0], p[1]) < 0.15


def test_tet_volume_preservation(oracle_lib):
    # SoftBodyTests.swift:53-69: 6V / 0.125 = 1 +- 0.05 after 300 frames
    o = run(oracle_lib, demos.single_tet_scene(), 300)
    pos, _ = o.positions()
    p = pos[:4, :3].astype(np.float64)
    v6 = abs(np.dot(p[1] - p[0], np.cross(p[2] - p[0], p[3] - p[0])))
    assert abs(v6 / 0.125 - 1.0) < 0.05


def test_particle_rod_chain_inextensible(oracle_lib):
    # SoftBodyTests.swift:27-51: rods stay 0.25 +- 0.01; particles keep identity rotation
    o = run(oracle_lib, demos.particle_rod_chain_scene(), 300)
    pos, rot = o.positions()
    d = np.linalg.norm(pos[1:12, :3] - pos[:11, :3], axis=1)
    assert np.all(np.abs(d - 0.25) < 0.01)
    assert abs(rot[5, 3] - 1.0) < 1e-4


def test_gravity_scale(oracle_lib):
    # GPUSolverTests.swift:7-30: gravityScale 0 holds z = 2 +- 1e-5; scale 1 falls below 1.95
    s = PhysicsScene("gravity-scale")
    s.settings.dt = 1 / 100
    s.settings.iterations = 4
    a = s.add_body((0.1, 0.1, 0.1), 1000.0, 0.0, (0, 0, 2), shape=abi.SHAPE_SPHERE)
    b = s.add_body((0.1, 0.1, 0.1), 1000.0, 0.0, (2, 0, 2), shape=abi.SHAPE_SPHERE)
    s.bodies[a].gravity_scale = 0.0
    o = run(oracle_lib, s, 10)
    st = o.body_states()
    assert abs(st[a].position[2] - 2.0) < 1e-5
    assert st[b].position[2] < 1.95


def test_rigid_linear_damping(oracle_lib):
    # GPUSolverTests.swift:32-53: v = exp(-2) +- 1e-4 after 1 s at damping 2
    s = PhysicsScene("damping")
    s.settings.gravity = 0.0
    s.settings.dt = 1 / 120
    s.settings.rigid_linear_damping = 2.0
    b = s.add_body((0.2, 0.2, 0.2), 1000.0, 0.0, (0, 0, 0), velocity=(1, 0, 0), shape=abi.SHAPE_SPHERE)
    o = run(oracle_lib, s, 120)
    assert abs(o.body_states()[b].velocity[0] - math.exp(-2)) < 1e-4


def test_rigid_damping_does_not_damp_particles(oracle_lib):
    # GPUSolverTests.swift:83-104
    s = PhysicsScene("particle-damping")
    s.settings.gravity = 0.0
    s.settings.dt = 1 / 120
    s.settings.rigid_linear_damping = 2.0
    s.settings.rigid_angular_damping = 2.0
    p = s.add_particle(0.04, 0.01, 0.0, (0, 0, 0), velocity=(1, 0, 0))
    o = run(oracle_lib, s, 120)
    assert abs(o.body_states()[p].velocity[0] - 1.0) < 1e-4


def test_bitwise_determinism(oracle_lib):
    # GPUSolverTests.swift:777-828: two instances, identical trajectories
    s = demos.rigid_stack_scene(seed=7, count=8)
    a = run(oracle_lib, s, 60)
    b = run(oracle_lib, s, 60)
    pa, ra = a.positions()
    pb, rb = b.positions()
    assert np.array_equal(pa.view(np.uint32), pb.view(np.uint32))
    assert np.array_equal(ra.view(np.uint32), rb.view(np.uint32))


def test_soft_cube_settles_on_ground(oracle_lib):
    # scaled soft cube: rests on the ground without tunnelling or collapse
    s = demos.soft_cube_scene(seed=3, n=6)
    o = run(oracle_lib, s, 240)
    pos, _ = o.positions()
    z = pos[1:, 2]
    assert z.min() > -0.02
    assert 0.8 < z.max() - z.min() < 1.2


def test_unsupported_features_are_refused(oracle_lib):
    # Planar-DAT truncation of tet surfaces is refused, not approximated
    s = demos.two_cubes_scene(n=3)
    with pytest.raises(RuntimeError):
        oracle_lib.OracleSolver(s, truncation=abi.TRUNCATION_PLANAR_DAT)


def test_atan2_series_accuracy(oracle_lib):
    """The fixed-sequence atan2 shared by the oracle and the kernels (hinge
    twist angles) stays within a few ulp of the float64 value, keeps the
    quadrant and signed-zero conventions of atan2."""
    import math
    lib = oracle_lib.lib()
    rng = np.random.default_rng(3)
    ys = np.concatenate([rng.normal(size=4000), rng.uniform(-1e-3, 1e-3, 500), [0.0, -0.0, 1.0, -1.0]])
    xs = np.concatenate([rng.normal(size=4000), rng.uniform(-1e-3, 1e-3, 500), [1.0, 1.0, 0.0, 0.0]])
    worst = 0.0
    for y, x in zip(ys.astype(np.float32), xs.astype(np.float32)):
        got = lib.oracle_atan2(float(y), float(x))
        want = math.atan2(float(y), float(x))
        ulp = np.spacing(np.float32(abs(want))) if want != 0 else np.float32(1e-45)
        worst = max(worst, abs(got - want) / float(ulp))
    assert worst <= 4.0, worst
    assert lib.oracle_atan2(0.0, -0.0) == np.float32(math.pi)
    assert math.copysign(1.0, lib.oracle_atan2(-0.0, 1.0)) < 0
    assert lib.oracle_atan2(1.0, 0.0) == np.float32(math.pi / 2)
