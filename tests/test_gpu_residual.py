"""The solver's convergence metrics against the oracle, through the C ABI.

* `avbd_max_constraint_error` — the reference's `diag_error`
  (Shaders/40_solver.metal:2189-2229, host GPUSolver.swift:4829-4864): the
  largest hard-joint violation and contact penetration of the last frame.
  Both sides take the maximum of the same float32 values, so they must agree
  bit for bit.
* the AL residual trace — r = ||gradient of the augmented-Lagrangian
  objective||_2 over every dynamic DOF (the primal's right-hand side with the
  inertial term), at the warm start and after every iteration.  The kernels
  sum per-body float32 squares in double in a fixed order, the oracle in body
  order; the traces must agree within 1e-5 relative.
"""
import numpy as np
import pytest

from avbd_b200 import demos
from avbd_b200.solver import GPUSolver

from test_gpu_parity import pair

pytestmark = pytest.mark.gpu

RESID_REL_TOL = 1e-5


def small_mixed():
    return demos.mixed_scene(seed=7, cubes=4, cube_n=4, boxes=4, cloth_n=10, pitch=0.5)


def hinge_worlds():
    s, motors, _ = demos.batched_worlds_scene(worlds=24, seed=5)
    return s, np.array(motors, np.uint32)


@pytest.mark.parametrize("name,make,frames,penetrates", [
    ("rigid-stack-20", lambda: demos.rigid_stack_scene(seed=1), 60, True),
    ("soft-cube-24", lambda: demos.soft_cube_scene(seed=2, n=24), 40, True),
    # contacts held inside the speculative margin: the metric stays 0
    ("mixed-small", small_mixed, 60, False),
    ("box-field-700", lambda: demos.box_field_scene(700), 30, False),
])
def test_max_constraint_error_matches_oracle(cuda_lib, oracle_lib, name, make, frames, penetrates):
    g, o = pair(make(), oracle_lib)
    seen = 0.0
    for f in range(frames):
        g.step(1)
        assert o.step(1) == 0
        if f % 5 == 4 or f + 1 == frames:
            a, b = g.max_constraint_error(), o.max_constraint_error()
            assert np.float32(a).view(np.uint32) == np.float32(b).view(np.uint32), \
                f"{name} frame {f + 1}: diag {a!r} vs oracle {b!r}"
            seen = max(seen, a)
    if penetrates:
        assert seen > 0.0, f"{name}: no contact penetration or joint error was ever measured"


def test_max_constraint_error_hinge_worlds(cuda_lib, oracle_lib):
    s, motors = hinge_worlds()
    g, o = pair(s, oracle_lib)
    rng = np.random.default_rng(3)
    for f in range(40):
        t = rng.uniform(-0.5, 0.5, size=len(motors)).astype(np.float32)
        g.set_motor_targets(motors, t)
        o.set_motor_targets(motors, t)
        g.step(1)
        o.step(1)
        a, b = g.max_constraint_error(), o.max_constraint_error()
        # joint errors pass through the hinge twist (atan2 series, shared) and
        # agree bit for bit whenever the poses do
        gp, _ = g.positions()
        op, _ = o.positions()
        if np.array_equal(gp.view(np.uint32), op.view(np.uint32)):
            assert a == b, f"frame {f + 1}: {a} vs {b}"
        else:
            assert abs(a - b) <= 1e-4 * max(1.0, abs(b))


def trace_len(scene):
    return 2 + scene.settings.iterations


@pytest.mark.parametrize("name,make,frames", [
    ("soft-cube-24", lambda: demos.soft_cube_scene(seed=2, n=24), 30),
    ("rigid-stack-20", lambda: demos.rigid_stack_scene(seed=1), 40),
    ("mixed-small", small_mixed, 40),
    ("cloth-sphere-24", lambda: demos.cloth_sphere_scene(n=24, iterations=10), 30),
])
def test_residual_trace_matches_oracle(cuda_lib, oracle_lib, name, make, frames):
    scene = make()
    g, o = pair(scene, oracle_lib)
    g.set_residual_trace(True)
    o.set_residual_trace(True)
    n = trace_len(scene)
    worst = 0.0
    for f in range(frames):
        g.step(1)
        assert o.step(1) == 0
        g.synchronize()
        a, b = g.residual_trace(n), o.residual_trace(n)
        assert np.all(np.isfinite(a)) and np.all(b >= 0.0)
        scale = np.maximum(np.abs(b), 1e-30)
        err = float(np.max(np.abs(a - b) / scale))
        worst = max(worst, err)
        assert err <= RESID_REL_TOL, f"{name} frame {f + 1}: trace {a} vs oracle {b} (rel {err:.2e})"
    print(f"{name}: residual traces agree to {worst:.2e} relative over {frames} frames")


def test_residual_trace_hinge_worlds(cuda_lib, oracle_lib):
    s, motors = hinge_worlds()
    g, o = pair(s, oracle_lib)
    g.set_residual_trace(True)
    o.set_residual_trace(True)
    n = trace_len(s)
    rng = np.random.default_rng(8)
    for f in range(30):
        t = rng.uniform(-0.5, 0.5, size=len(motors)).astype(np.float32)
        g.set_motor_targets(motors, t)
        o.set_motor_targets(motors, t)
        g.step(1)
        o.step(1)
        g.synchronize()
        a, b = g.residual_trace(n), o.residual_trace(n)
        err = float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-30)))
        assert err <= 1e-4, f"frame {f + 1}: {a} vs {b}"


def test_residual_falls_over_iterations(cuda_lib):
    """The AL residual of the soft cube falls from the warm start to the last
    iteration on contact frames (a sanity check of what the trace measures)."""
    s = demos.soft_cube_scene(seed=2, n=24)
    g = GPUSolver(s)
    g.set_residual_trace(True)
    n = trace_len(s)
    drops = 0
    for f in range(60):
        g.step(1)
        g.synchronize()
        t = g.residual_trace(n)
        if f >= 30:
            drops += t[-1] < t[0]
    assert drops >= 25
