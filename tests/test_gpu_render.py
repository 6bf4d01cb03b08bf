"""Headless render and observation compute: the CUDA kernels against the
CPU oracle through the C ABI.  Push-T observations are bytes and must be
identical; instance records and skinned vertices are computed with the same
IEEE operations and must be bit-identical; smooth normals go through acosf
(CUDA) against std::acos (oracle) and must agree within 2e-6."""
import numpy as np
import pytest

from avbd_b200 import demos
from avbd_b200.solver import AVBDError, GPUSolver

from test_gpu_parity import compare_state, pair

pytestmark = pytest.mark.gpu


def drive_pusht(g, o, envs, frames, seed=0):
    rng = np.random.default_rng(seed)
    targets = rng.uniform(-2.5, 2.5, size=(len(envs), 2))
    for f in range(frames):
        if f % 20 == 0:
            targets = rng.uniform(-2.5, 2.5, size=(len(envs), 2))
        ids, pts = demos.pusht_tip_anchors(envs, targets)
        g.set_joint_world_anchors(ids, pts)
        o.set_joint_world_anchors(ids, pts)
        g.step(1)
        assert o.step(1) == 0


@pytest.mark.parametrize("res", [64, 50])
def test_pusht_obs_bytes(cuda_lib, oracle_lib, res):
    s, envs = demos.pusht_scene(16, seed=2)
    g, o = pair(s, oracle_lib)
    drive_pusht(g, o, envs, 120)
    compare_state(g, o, 120)
    table = demos.pusht_env_table(envs)
    a, b = g.render_pusht_obs(table, res), o.render_pusht_obs(table, res)
    assert a.shape == (16, res, res, 3)
    assert np.array_equal(a, b), f"{int((a != b).any(-1).sum())} pixels differ"
    assert len(np.unique(a.reshape(-1, 3), axis=0)) == 4


def test_pusht_obs_device_output(cuda_lib):
    """The device-output form writes the same bytes into caller memory."""
    torch = pytest.importorskip("torch")
    s, envs = demos.pusht_scene(8, seed=4)
    g = GPUSolver(s)
    g.step(10)
    table = demos.pusht_env_table(envs)
    host = g.render_pusht_obs(table, 64)
    dev = torch.zeros((8, 64, 64, 3), dtype=torch.uint8, device="cuda")
    g.render_pusht_obs(table, 64, device_out=dev.data_ptr())
    g.synchronize()
    torch.cuda.synchronize()
    assert np.array_equal(dev.cpu().numpy(), host)
    with pytest.raises(AVBDError):
        g.render_pusht_obs(table, 1)


def test_build_instances_bitwise(cuda_lib, oracle_lib):
    s = demos.shapes_scene(count=48)
    g, o = pair(s, oracle_lib)
    g.step(60)
    assert o.step(60) == 0
    ids = list(range(len(s.colliders)))
    colors = np.zeros((len(ids), 4), np.float32)
    colors[::5] = (0.2, 0.3, 0.4, 1.0)
    for mode in (0, 1):
        a = g.build_instances(ids, colors, color_mode=mode)
        b = o.build_instances(ids, colors, color_mode=mode)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f"mode {mode}"
    assert not a[0].any()  # the ground slab


def test_soft_normals_match(cuda_lib, oracle_lib):
    for scene in (demos.soft_cube_scene(seed=5, n=8), demos.drape_scene(res=16)):
        g, o = pair(scene, oracle_lib)
        g.step(40)
        assert o.step(40) == 0
        compare_state(g, o, 40)
        a, b = g.soft_normals(0.5), o.soft_normals(0.5)
        assert np.abs(a - b).max() <= 2e-6, np.abs(a - b).max()
        on = np.linalg.norm(a[:, :3], axis=1) > 0
        assert on.sum() > 0 and np.allclose(np.linalg.norm(a[on, :3], axis=1), 1.0, atol=1e-5)


def test_skin_deform_bitwise(cuda_lib, oracle_lib):
    s = demos.soft_cube_scene(seed=6, n=6)
    g, o = pair(s, oracle_lib)
    binds = demos.skin_bindings_for_tets(s, per_tet=2)
    g.set_skin_bindings(binds)
    o.set_skin_bindings(binds)
    g.step(30)
    assert o.step(30) == 0
    a, b = g.skin_deform(), o.skin_deform()
    assert a.shape == (len(binds), 8)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
