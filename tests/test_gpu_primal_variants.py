"""Every variant of the static-palette primal against the oracle, bit for bit.

The autotuner picks per color between the grouped kernel (8, 16 or 32 lanes
per body) and the staged kernel (the block's adjacency entries evaluated
densely into shared memory, then folded per body by 8 lanes).  Each variant
folds the entries of a body in the order of the reference's 8-lane SIMD
group (primal_particles_split, 40_solver.metal:1544-1686), so each must
reproduce the oracle's frames exactly; here every variant is pinned for
the whole run instead of only for the tuner's timing frame.
"""
import math

import numpy as np
import pytest

from avbd_b200 import abi, demos
from avbd_b200.scene import PhysicsScene, SceneJoint, SceneTet
from avbd_b200.solver import GPUSolver

pytestmark = pytest.mark.gpu

VARIANTS = [abi.PRIMAL_VARIANT_STAGED, 8, 16, 32]


def tet_fan_scene(tets: int = 600, pinned: bool = False) -> PhysicsScene:
    """One hub particle shared by `tets` tets (600 adjacency entries: more
    than a staged block holds, so the fold also evaluates entries inline)."""
    s = PhysicsScene("tet-fan")
    s.settings.iterations = 10
    hub = s.add_particle(0.02, 0.05, position=(0.0, 0.0, 2.0))
    for k in range(tets):
        # direction on a Fibonacci sphere, a small right-handed tet out there
        z = 1.0 - 2.0 * (k + 0.5) / tets
        r = math.sqrt(max(0.0, 1.0 - z * z))
        phi = k * 2.399963229728653
        d = np.array([r * math.cos(phi), r * math.sin(phi), z])
        u = np.cross(d, [0.0, 0.0, 1.0] if abs(z) < 0.9 else [1.0, 0.0, 0.0])
        u /= np.linalg.norm(u)
        v = np.cross(d, u)
        c = np.array([0.0, 0.0, 2.0]) + 0.5 * d
        ids = [s.add_particle(0.01, 0.02, position=tuple(c + 0.04 * w)) for w in (u, v, d)]
        s.add_tet(SceneTet((hub, ids[0], ids[1], ids[2]), 500.0, 2000.0))
    if pinned:
        s.add_joint(SceneJoint(-1, hub, (0.0, 0.0, 2.0), (0, 0, 0)))
    return s


def run_pinned_variant(scene, oracle_lib, variant, frames):
    g = GPUSolver(scene)
    o = oracle_lib.OracleSolver(scene, threads=8)
    g.set_primal_variant(variant)
    for f in range(frames):
        g.step(1)
        assert o.step(1) == 0
        gp, gr = g.positions()
        op, orr = o.positions()
        assert np.array_equal(gp.view(np.uint32), op.view(np.uint32)), f"frame {f + 1}: positions differ"
        assert np.array_equal(gr.view(np.uint32), orr.view(np.uint32)), f"frame {f + 1}: rotations differ"
    lanes = g.profile()["color_lanes"]
    return lanes


SCENES = [
    ("soft-cube-10", lambda: demos.soft_cube_scene(seed=5, n=10, iterations=10), 20),
    ("pinned-soft-block-10", lambda: demos.pinned_soft_block_scene(10), 20),
    ("mixed-small", lambda: demos.mixed_scene(seed=7, cubes=4, cube_n=4, boxes=4, cloth_n=10, pitch=0.5), 40),
    # 40 boxes: more than 32 global colliders, so the rigid-triangle
    # emission takes its warp path over the global chunks
    ("mixed-40-boxes", lambda: demos.mixed_scene(seed=9, cubes=4, cube_n=4, boxes=40, cloth_n=16, pitch=0.5), 40),
    ("drape-20", lambda: demos.drape_scene(res=20), 30),
    ("tet-fan", lambda: tet_fan_scene(), 10),
    ("tet-fan-pinned", lambda: tet_fan_scene(pinned=True), 10),
]


@pytest.mark.parametrize("name,make,frames", SCENES, ids=[s[0] for s in SCENES])
@pytest.mark.parametrize("variant", VARIANTS, ids=["staged", "lanes8", "lanes16", "lanes32"])
def test_primal_variant_bitwise(cuda_lib, oracle_lib, name, make, frames, variant):
    lanes = run_pinned_variant(make(), oracle_lib, variant, frames)
    assert variant in lanes


def test_primal_variant_rejects_unknown(cuda_lib):
    g = GPUSolver(demos.soft_cube_scene(seed=5, n=10, iterations=4))
    with pytest.raises(Exception):
        g.set_primal_variant(12)
    g.set_primal_variant(abi.PRIMAL_VARIANT_AUTO)
    g.step(6)                                   # four tuning frames, then graphs
    assert all(v in (1, 8, 16, 32) for v in g.profile()["color_lanes"][:4])
