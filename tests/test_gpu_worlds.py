"""Batched worlds through avbd_create_batched (ragged world offsets).

The reference packs vector environments into one scene with one collision
group per environment (RL/PushTEnv.swift:137-180) and resets them through
setBodyStates (GPUSolver.swift:2409-2473).  Here the same 4096 articulated
worlds are built with every collider in group 0 and handed to
avbd_create_batched with their ragged body offsets: the frames must be bit
for bit those of the collision-group packing built by hand.  World-addressed
state setters, world resets and the motor-joint lists are checked too, as is
the block-shape autotuner of the dynamic-coloring primal.
"""
import numpy as np
import pytest

from avbd_b200 import abi, demos
from avbd_b200.solver import GPUSolver

pytestmark = pytest.mark.gpu


def worlds(n=4096, seed=4, groups=True):
    return demos.batched_worlds_scene(worlds=n, seed=seed, collision_groups=groups)


def offsets_of(scene, offs):
    return np.array(list(offs) + [len(scene.bodies)], np.uint32)


def test_batched_create_matches_collision_group_packing(cuda_lib):
    s_ref, motors, offs = worlds()
    s_bat, motors_b, offs_b = worlds(groups=False)
    assert offs == offs_b and motors == motors_b
    ref = GPUSolver(s_ref)
    bat = GPUSolver(s_bat, world_offsets=offsets_of(s_bat, offs))
    assert np.array_equal(bat.world_offsets(), offsets_of(s_bat, offs))
    assert np.array_equal(ref.world_offsets(), np.zeros(0, np.uint32))
    rng = np.random.default_rng(5)
    ids = np.array(motors, np.uint32)
    for f in range(60):
        t = rng.uniform(-0.5, 0.5, size=len(ids)).astype(np.float32)
        ref.set_motor_targets(ids, t)
        bat.set_motor_targets(ids, t)
        ref.step(1)
        bat.step(1)
        a, ra = ref.positions()
        b, rb = bat.positions()
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f"frame {f + 1}"
        assert np.array_equal(ra.view(np.uint32), rb.view(np.uint32)), f"frame {f + 1}"
    # every world's motors, in joint order
    per_world = {}
    for j in motors:
        b = s_ref.joints[j].body_b
        w = int(np.searchsorted(np.array(offs), b, side="right") - 1)
        per_world.setdefault(w, []).append(j)
    for w in (0, 1, 2047, 4095):
        assert list(bat.world_motor_joints(w)) == per_world[w]


def test_world_setters_and_resets(cuda_lib):
    s, motors, offs = worlds(n=64, seed=7, groups=False)
    o = offsets_of(s, offs)
    a = GPUSolver(s, world_offsets=o)
    b = GPUSolver(s, world_offsets=o)
    ids = np.array(motors, np.uint32)
    rng = np.random.default_rng(2)
    targets = [rng.uniform(-0.5, 0.5, size=len(ids)).astype(np.float32) for _ in range(60)]
    for f in range(30):
        for g in (a, b):
            g.set_motor_targets(ids, targets[f])
            g.step(1)
    # world-addressed states equal global ones
    w = 9
    st = a.body_states([int(o[w]) + 1])[0]
    st.velocity[:] = (0.0, 0.0, 1.0)
    a.set_world_body_states(w, [1], [st])
    b.set_body_states([int(o[w]) + 1], [st])
    pa, _ = a.positions()
    pb, _ = b.positions()
    assert np.array_equal(pa.view(np.uint32), pb.view(np.uint32))
    # reset world 5 of `a` only: its bodies return to their creation state,
    # the other worlds do not notice
    a.reset_worlds([5])
    init = [(bd.position, bd.rotation) for bd in s.bodies]
    sa = a.body_states(list(range(int(o[5]), int(o[6]))))
    for k, stt in enumerate(sa):
        p0, q0 = init[int(o[5]) + k]
        assert np.allclose(stt.position[:], p0, atol=0) and np.allclose(stt.rotation[:], q0, atol=0)
        assert np.allclose(stt.velocity[:], 0.0)
    others = np.ones(len(s.bodies), bool)
    others[int(o[5]):int(o[6])] = False
    for f in range(30, 60):
        for g in (a, b):
            g.set_motor_targets(ids, targets[f])
            g.step(1)
        pa, _ = a.positions()
        pb, _ = b.positions()
        assert np.array_equal(pa[others].view(np.uint32), pb[others].view(np.uint32)), f"frame {f + 1}"
    assert not np.array_equal(pa[~others], pb[~others])


def test_dynamic_primal_shape_is_tuned_once_per_bucket(cuda_lib):
    s, _, offs = worlds(n=512, seed=3)
    g1 = GPUSolver(s)
    g1.step(10)
    p1 = g1.profile()["dynamic_primal_shape"]
    shapes = {(148 * k, t) for k, t in [(1, 128), (2, 128), (3, 128), (4, 128), (4, 64), (6, 64), (8, 64)]}
    assert (p1["blocks"], p1["threads"]) in shapes
    n_dyn = sum(1 for b in s.bodies if b.is_dynamic)
    assert 2 ** p1["body_count_bucket"] <= n_dyn < 2 ** (p1["body_count_bucket"] + 1)
    g2 = GPUSolver(s)
    g2.step(10)
    p2 = g2.profile()["dynamic_primal_shape"]
    assert (p2["blocks"], p2["threads"]) == (p1["blocks"], p1["threads"])
    assert p2["candidates_timed"] == 0
    # tuning frames compute the same floats as the tuned graph frames
    a, _ = g1.positions()
    b, _ = g2.positions()
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    print("dynamic primal shape", p1)
