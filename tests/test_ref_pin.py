"""The oracle pinned to the reference's own solver kernels.

The reference's shader sources (Sources/PhysicsAVBD/Shaders/*.metal) compile
unchanged as C++ through the Metal stand-in header oracle/msl/metal_stdlib
(oracle/ref.py builds them, where they lie, into oracle/_ref/).  Every frame
of each scene below is computed by the oracle and, stage by stage on the same
input state, by the reference's kernels: the spatial hash and candidate pairs
(bp_count / bp_scatter / bp_sort_cells / bp_count_pairs_deterministic /
bp_emit_pairs_deterministic), the narrowphase (np_collide), the persistence
map (pm_insert), the joint and body warm start, the adjacency lists, the
dynamic coloring, the 8-lane split primal of every color of every iteration
(primal_particles_split, its SIMD lanes run in lockstep), the dual (dual_all)
and finalize_velocities — and the two outputs are compared word for word.
The bar is bit-exact for every stage, integers and floats alike.

These tests need the reference's sources and so run where they are present
(skipped elsewhere); tests/golden/ holds trajectories recorded from this
pinned oracle, which the CUDA tests and every machine can check against.
"""
import numpy as np
import pytest

from avbd_b200 import demos

ref = pytest.importorskip("oracle.ref")
if not ref.available():
    pytest.skip("the reference's shader sources are not present on this machine", allow_module_level=True)


@pytest.fixture(scope="module")
def pinned():
    ref.build()
    return ref


def small_mixed():
    return demos.mixed_scene(seed=7, cubes=4, cube_n=4, boxes=4, cloth_n=10, pitch=0.5)


SCENES = [
    ("stack-5", lambda: demos.stack(5), 40, 1),
    ("rigid-stack-20", lambda: demos.rigid_stack_scene(seed=1), 60, 1),
    ("soft-cube-6", lambda: demos.soft_cube_scene(seed=5, n=6), 40, 1),
    ("hinge-worlds-8", lambda: demos.batched_worlds_scene(worlds=8, seed=5)[0], 40, 1),
    ("box-field-200", lambda: demos.box_field_scene(200), 30, 1),
    ("shapes-512", lambda: demos.shapes_scene(seed=1), 30, 2),
    ("drape-12", lambda: demos.drape_scene(res=12), 40, 1),
    ("mixed-small", small_mixed, 40, 2),
]


@pytest.mark.parametrize("name,make,frames,primal_every", SCENES, ids=[s[0] for s in SCENES])
def test_every_stage_matches_the_reference_kernels(pinned, name, make, frames, primal_every):
    o = pinned.PinnedOracle(make(), primal_every=primal_every)
    assert o.step(frames) == 0
    st = o.stats()
    for stage in ("narrowphase", "map", "warm_bodies", "adjacency", "primal", "dual", "finalize"):
        assert st[stage]["compared"] > 0, f"{name}: stage {stage} compared nothing"
    bad = {k: v for k, v in st.items() if v["mismatched"]}
    assert not bad, f"{name}: stages differing from the reference's kernels: {bad}"
    print(name, {k: v["compared"] for k, v in st.items() if v["compared"]})
    o.close()


def test_dynamic_coloring_and_pairs_are_compared(pinned):
    o = pinned.PinnedOracle(demos.rigid_stack_scene(seed=3), primal_every=4)
    o.step(30)
    st = o.stats()
    assert st["coloring"]["compared"] > 0 and st["broadphase"]["compared"] > 0
    assert st["coloring"]["mismatched"] == 0 and st["broadphase"]["mismatched"] == 0


def test_joint_warm_start_is_compared(pinned):
    o = pinned.PinnedOracle(demos.batched_worlds_scene(worlds=4, seed=2)[0], primal_every=4)
    o.step(20)
    st = o.stats()
    assert st["warm_joints"]["compared"] > 0 and st["warm_joints"]["mismatched"] == 0


@pytest.mark.parametrize("stage", ["primal", "dual"])
def test_harness_reports_a_planted_difference(pinned, stage):
    """Self-check: one perturbed input in the reference's run of a stage
    must show up as mismatched records of that stage and no other."""
    o = pinned.PinnedOracle(demos.stack(5))
    o.perturb_for_testing(stage)
    o.step(10)
    st = o.stats()
    assert st[stage]["mismatched"] > 0
    assert all(v["mismatched"] == 0 for k, v in st.items() if k != stage)


def test_reference_diag_error_matches_oracle(pinned):
    o = pinned.PinnedOracle(demos.soft_cube_scene(seed=5, n=6), primal_every=10)
    seen = 0.0
    for _ in range(30):
        o.step(1)
        a, b = o.reference_diag_error(), o.max_constraint_error()
        assert np.float32(a).view(np.uint32) == np.float32(b).view(np.uint32)
        seen = max(seen, a)
    assert seen > 0.0
