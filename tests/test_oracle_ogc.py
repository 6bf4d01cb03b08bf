"""Isotropic-OGC gates on the CPU oracle: soft surfaces that touch each
other, rigid boxes and cloth landing on soft bodies, cloth under isotropic
truncation.  They check the behaviour the element contacts exist for
(surfaces stay apart, every contact kind is produced, nothing blows up) and
the topology the trackers use."""
import numpy as np

from avbd_b200 import abi, demos


def test_two_cubes_stay_apart(oracle_lib):
    """The upper cube lands on the lower one and rests there: vertex-triangle
    contacts keep the two surfaces separated."""
    n = 5
    o = oracle_lib.OracleSolver(demos.two_cubes_scene(n=n), threads=1)
    seen_vt = 0
    for _ in range(150):
        assert o.step(1) == 0
        seen_vt = max(seen_vt, o.counters().soft_vt)
    pos, _ = o.positions()
    lower = pos[1:1 + n ** 3, 2]
    upper = pos[1 + n ** 3:1 + 2 * n ** 3, 2]
    radius = 0.3 / (n - 1) * 0.32
    assert np.isfinite(pos).all() and o.runtime_failure() == 0
    assert seen_vt > 0
    assert upper.min() > lower.max() - 2 * radius, (upper.min(), lower.max())


def test_mixed_scene_produces_every_contact_kind(oracle_lib):
    """Soft cubes, boxes and a cloth: rigid-triangle, vertex-triangle and
    edge-edge records all appear, bounds clamp some steps, and the state
    stays finite."""
    o = oracle_lib.OracleSolver(demos.mixed_scene(seed=7, cubes=4, cube_n=4, boxes=4, cloth_n=10, pitch=0.5),
                                threads=1)
    rt = vt = ee = clamped = 0
    for _ in range(120):
        assert o.step(1) == 0
        c = o.counters()
        rt, vt, ee = max(rt, c.soft_rt), max(vt, c.soft_vt), max(ee, c.soft_ee)
        clamped += c.ogc_exceeded
    pos, _ = o.positions()
    assert np.isfinite(pos).all() and o.runtime_failure() == 0
    assert rt > 0 and vt > 0 and ee > 0 and clamped > 0


def test_isotropic_cloth_drape(oracle_lib):
    """A cloth draped over a box under isotropic truncation (instead of the
    automatic Planar-DAT): element contacts form and the sheet stays finite
    and above the ground."""
    o = oracle_lib.OracleSolver(demos.drape_scene(res=14), threads=1, truncation=abi.TRUNCATION_ISOTROPIC)
    for _ in range(90):
        assert o.step(1) == 0
    c = o.counters()
    pos, _ = o.positions()
    assert np.isfinite(pos).all() and o.runtime_failure() == 0
    assert c.soft_vt + c.soft_rt > 0
    assert pos[1:, 2].min() > -0.05


def test_two_cube_topology(oracle_lib):
    """Collision surfaces of two tet blocks: boundary triangles of each
    block, every surface vertex on exactly one surface group."""
    n = 5
    o = oracle_lib.OracleSolver(demos.two_cubes_scene(n=n), threads=1)
    tris = o.debug_read("TRIS").view(np.uint32).reshape(-1, 4)
    assert len(tris) == 2 * 6 * 2 * (n - 1) ** 2
    group = o.debug_read("CLOTH_GROUP").view(np.uint32)
    surf = o.debug_read("PARTICLE_IDX").view(np.uint32)
    assert len(surf) == 2 * (n ** 3 - (n - 2) ** 3)
    assert set(np.unique(group[surf])) == {1, 2}
