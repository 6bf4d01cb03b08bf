"""Headless render and observation compute on the CPU oracle
(50_render.metal, 60_robotics.metal): Push-T pixel observations, rigid
instance records, soft-surface normals and skinned vertices, checked
against what the geometry says they must be."""
import math

import numpy as np

from avbd_b200 import abi, demos

BG, GOAL, BLOCK, TIP = (15, 15, 15), (25, 140, 30), (216, 38, 30), (51, 102, 242)


def pixel_of(x, y, center, res, half=3.25):
    f = lambda w, c: int(round(((w - c) / (2 * half) + 0.5) * (res - 1)))  # noqa: E731
    return f(x, center[0]), f(y, center[1])


def test_pusht_observation_layout(oracle_lib):
    """Goal T green, block T red, pusher disc blue on the dark background,
    at the pixels their world positions map to (60_robotics.metal:21-69)."""
    s, envs = demos.pusht_scene(4, seed=3)
    o = oracle_lib.OracleSolver(s, threads=1)
    res = 64
    img = o.render_pusht_obs(demos.pusht_env_table(envs), res)
    assert img.shape == (4, res, res, 3)
    pos, _ = o.positions()
    pix_area = (6.5 / (res - 1)) ** 2
    for e, r in enumerate(envs):
        flat = img[e].reshape(-1, 3)
        kinds = {c: int((flat == np.array(c)).all(1).sum()) for c in (BG, GOAL, BLOCK, TIP)}
        assert sum(kinds.values()) == res * res
        # T area 0.25 + 0.1625 m^2; the goal may be partly covered by the block
        assert 0.6 < kinds[BLOCK] * pix_area / 0.4125 < 1.4, kinds
        assert kinds[GOAL] > 0 and kinds[TIP] > 0
        px, py = pixel_of(pos[r["tip"], 0], pos[r["tip"], 1], r["center"], res)
        assert tuple(img[e, py, px]) == TIP
        gx, gy = r["center"][0] + 0.85, r["center"][1] + 0.85 + 0.125  # goal bar centre (yaw 0)
        px, py = pixel_of(gx, gy, r["center"], res)
        assert tuple(img[e, py, px]) in (GOAL, BLOCK, TIP)
        assert tuple(img[e, 0, 0]) == BG


def test_pusht_tip_follows_anchor(oracle_lib):
    """The drag joint's world anchor moves the pusher; the observation
    shows the disc where the tip went."""
    s, envs = demos.pusht_scene(1, seed=5)
    o = oracle_lib.OracleSolver(s, threads=1)
    target = (-1.5, 1.0)
    for _ in range(90):
        ids, pts = demos.pusht_tip_anchors(envs, [target])
        o.set_joint_world_anchors(ids, pts)
        assert o.step(1) == 0
    pos, _ = o.positions()
    r = envs[0]
    tip = pos[r["tip"], :2] - np.asarray(r["center"])
    assert np.linalg.norm(tip - target) < 0.1, tip
    img = o.render_pusht_obs(demos.pusht_env_table(envs), 48)
    px, py = pixel_of(pos[r["tip"], 0], pos[r["tip"], 1], r["center"], 48)
    assert tuple(img[0, py, px]) == TIP


def test_build_instances_records(oracle_lib):
    """Model matrices are the collider's world rotation scaled by its size
    (unit scale for round shapes), translated to its centre; dynamic bodies
    get palette colours, statics grey, a ground slab over 150 m a zero record
    (50_render.metal:34-97)."""
    s = demos.stack(3)
    s.add_torus(0.4, 0.1, 1.0, 0.5, (3, 0, 1), rotation=demos.quat_axis_angle(0.3, (1, 0, 0)))
    o = oracle_lib.OracleSolver(s, threads=1)
    assert o.step(5) == 0
    recs = o.build_instances(list(range(len(s.colliders))), colors=None)
    assert not recs[0].any()  # 200 m ground slab
    pos, rot = o.positions()
    for c in (1, 2, 3):
        m = recs[c, :16].reshape(4, 4).T  # rows of the column-major matrix
        q = rot[c]
        u = np.asarray(q[:3], np.float64)
        R = np.eye(3) + 2 * q[3] * np.array([[0, -u[2], u[1]], [u[2], 0, -u[0]], [-u[1], u[0], 0]]) \
            + 2 * np.array([[0, -u[2], u[1]], [u[2], 0, -u[0]], [-u[1], u[0], 0]]) @ \
            np.array([[0, -u[2], u[1]], [u[2], 0, -u[0]], [-u[1], u[0], 0]])
        assert np.allclose(m[:3, :3], R * np.asarray(s.bodies[c].size), atol=1e-5)
        assert np.allclose(m[:3, 3], pos[c, :3], atol=1e-6)
        assert recs[c, 19] == 0.0 and recs[c, 23] == 1.0
    torus = recs[4]
    assert torus[19] == 2.0  # kind
    assert np.allclose(np.linalg.norm(torus[:12].reshape(3, 4)[:, :3], axis=1), 1.0, atol=1e-5)
    over = o.build_instances([1], colors=[(0.1, 0.2, 0.3, 1.0)])
    assert np.allclose(over[0, 16:19], (0.1, 0.2, 0.3))


def test_soft_normals_of_a_resting_block(oracle_lib):
    """Smooth normals of a soft block's boundary: face-interior vertices of
    the top face point up, of the side faces sideways; the render thickness
    is the particle radius where the surface is flat."""
    s = demos.soft_cube_scene(seed=3, n=6)
    o = oracle_lib.OracleSolver(s, threads=1)
    nrm = o.soft_normals(0.0)
    pos, _ = o.positions()
    verts = pos[1:, :3]
    zmax, xmax = verts[:, 2].max(), verts[:, 0].max()
    interior = lambda a, b: (a > verts[:, 0].min() + 0.1) & (a < xmax - 0.1) & \
        (b > verts[:, 1].min() + 0.1) & (b < verts[:, 1].max() - 0.1)  # noqa: E731
    top = np.where((np.abs(verts[:, 2] - zmax) < 1e-3) & interior(verts[:, 0], verts[:, 1]))[0] + 1
    assert len(top) > 0
    assert np.allclose(nrm[top, :3], (0, 0, 1), atol=2e-2)
    side = np.where(np.abs(verts[:, 0] - xmax) < 1e-3)[0] + 1
    assert (nrm[side, 0] > 0.5).all()
    radius = abs(s.bodies[top[0]].size[0]) / 2
    assert np.allclose(nrm[top, 3], radius, rtol=1e-3)
    assert not nrm[0].any()  # the ground is not on the surface


def test_skin_at_rest_reproduces_bindings(oracle_lib):
    """At the rest pose F = I: each skinned vertex is its weighted rest
    position and keeps its (normalised) rest normal."""
    s = demos.soft_cube_scene(seed=3, n=4)
    o = oracle_lib.OracleSolver(s, threads=1)
    binds = demos.skin_bindings_for_tets(s)
    o.set_skin_bindings(binds)
    out = o.skin_deform()
    pos = np.array([b.position for b in s.bodies], np.float64)
    for i in range(0, len(binds), 7):
        b = binds[i]
        want = sum(b.weights[k] * pos[b.ids[k]] for k in range(4))
        assert np.allclose(out[i, :3], want, atol=1e-5)
        n = np.array(b.rest_normal[:3])
        assert np.allclose(out[i, 4:7], n / np.linalg.norm(n), atol=1e-4)
        assert out[i, 3] == 1.0 and out[i, 7] == 0.0
