"""Scene builders on the host (no solver): convex colliders are centred on
their tight box without moving the geometry, capsules and tori carry the
reference's size convention, the Push-T batch is laid out and seeded as the
reference's vector environment and its tables and anchors are well formed."""
import numpy as np

from avbd_b200 import abi, demos
from avbd_b200.scene import PhysicsScene


def test_convex_collider_is_centred_on_its_box():
    s = PhysicsScene("hull")
    b = s.add_body((1, 1, 1), 0.0, 0.5, (0, 0, 0), collision_enabled=False)
    verts = [(0.0, 0.0, 0.0), (2.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 0.5)]
    q = demos.quat_axis_angle(0.7, (0, 0, 1))
    c = s.add_convex_collider(b, verts, local_position=(0.1, 0.2, 0.3), local_rotation=q)
    col = s.colliders[c]
    assert np.allclose(col.size, (2.0, 1.0, 0.5))
    v = np.asarray(col.hull_vertices)
    assert np.allclose(v.min(axis=0), -v.max(axis=0))
    # world-frame vertices are unchanged: local_position + R(local_rotation) v
    def rot(qq, x):
        u = np.asarray(qq[:3]); t = 2 * np.cross(u, x)
        return x + qq[3] * t + np.cross(u, t)
    before = np.array([np.array((0.1, 0.2, 0.3)) + rot(q, np.array(p)) for p in verts])
    after = np.array([np.asarray(col.local_position) + rot(q, p) for p in v])
    assert np.allclose(before, after, atol=1e-6)
    desc, keep = s.to_desc()
    assert desc.num_hull_vertices == 4 and desc.colliders[c].hull_count == 4


def test_capsule_and_torus_size_convention():
    s = PhysicsScene("round")
    a = s.add_capsule(0.8, 0.1, 1.0, 0.5, (0, 0, 1))
    t = s.add_torus(0.45, 0.12, 1.0, 0.5, (0, 0, 2))
    assert np.allclose(s.bodies[a].size, (0.8, 0.1, 0.0)) and s.bodies[a].shape == abi.SHAPE_CAPSULE
    assert np.allclose(s.bodies[t].size, (0.45, 0.12, 0.0)) and s.bodies[t].shape == abi.SHAPE_TORUS
    # their own colliders anchor contacts in world space (round anchors)
    assert s.colliders[-1].world_round_anchor and s.colliders[-2].world_round_anchor


def test_pusht_batch_layout_and_tables():
    s, envs = demos.pusht_scene(9, seed=3)
    s2, envs2 = demos.pusht_scene(9, seed=3)
    assert [b.position for b in s.bodies] == [b.position for b in s2.bodies]
    centers = np.array([e["center"] for e in envs])
    assert len({tuple(c) for c in centers}) == 9
    assert np.allclose(np.sort(np.unique(centers[:, 0])), [-7.0, 0.0, 7.0])
    for e_i, e in enumerate(envs):
        assert s.bodies[e["tip"]].shape == abi.SHAPE_CAPSULE
        assert s.joints[e["drag_joint"]].body_a == -1 and s.joints[e["drag_joint"]].body_b == e["tip"]
        g = e_i + 1
        assert all(c.collision_group == g for c in s.colliders if c.body in (e["tip"], e["bar"], e["stem"]))
    table = demos.pusht_env_table(envs)
    assert len(table) == 9 and table[4].goal[1] == 3.25 and list(table[0].ids)[:3] == [envs[0]["tip"], envs[0]["bar"], envs[0]["stem"]]
    ids, pts = demos.pusht_tip_anchors(envs, [(5.0, -5.0)] * 9)
    assert ids == [e["drag_joint"] for e in envs]
    assert np.allclose(pts[:, :2] - centers, [3.02, -3.02])
    assert np.allclose(pts[:, 2], demos.PUSHT_TIP_HEIGHT)


def test_skin_bindings_cover_every_tet():
    s = demos.soft_cube_scene(seed=1, n=3)
    b = demos.skin_bindings_for_tets(s, per_tet=2)
    assert len(b) == 2 * len(s.tets)
    w = np.array([list(x.weights) for x in b])
    assert np.allclose(w.sum(axis=1), 1.0, atol=1e-6) and (w >= 0).all()
