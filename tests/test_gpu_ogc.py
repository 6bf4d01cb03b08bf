"""Isotropic-OGC parity of the CUDA solver with the CPU oracle, through the
C ABI: soft bodies touching each other, rigid boxes and cloth meeting soft
surfaces, and cloth under isotropic truncation (vertex-triangle / edge-edge
trackers, conservative bounds and their refresh, rigid-triangle contacts,
color-Jacobi commits).

Contact records and adjacency must be bit-exact; positions and velocities
within 1e-4 relative per frame (in practice the frames agree bit for bit and
the tests print how many did).
"""
import numpy as np
import pytest

from avbd_b200 import abi, demos

from test_gpu_parity import compare_state, pair

pytestmark = pytest.mark.gpu


def small_mixed():
    return demos.mixed_scene(seed=7, cubes=4, cube_n=4, boxes=4, cloth_n=10, pitch=0.5)


def iso_drape():
    return demos.drape_scene(res=14)


def run_ogc(scene, oracle_lib, frames, check_every=1, **kw):
    g, o = pair(scene, oracle_lib, **kw)
    exact = 0
    for f in range(frames):
        g.step(1)
        assert o.step(1) == 0
        if (f + 1) % check_every == 0 or f + 1 == frames:
            exact += compare_state(g, o, f + 1)
            gc, oc = g.counters(), o.counters()
            assert (gc.num_soft, gc.soft_rt, gc.soft_vt, gc.soft_ee, gc.ogc_exceeded) == \
                   (oc.num_soft, oc.soft_rt, oc.soft_vt, oc.soft_ee, oc.ogc_exceeded), f"frame {f + 1}"
    return g, o, exact


@pytest.mark.parametrize("name,make,frames,kw", [
    ("two-cubes", lambda: demos.two_cubes_scene(), 90, {}),
    ("mixed-small", small_mixed, 120, {}),
    ("iso-drape-14", iso_drape, 90, {"truncation": abi.TRUNCATION_ISOTROPIC}),
])
def test_ogc_trajectory_parity(cuda_lib, oracle_lib, name, make, frames, kw):
    g, o, exact = run_ogc(make(), oracle_lib, frames, **kw)
    c = g.counters()
    print(f"{name}: {exact}/{frames} frames bit-identical; soft rt/vt/ee {c.soft_rt}/{c.soft_vt}/{c.soft_ee}")
    assert g.runtime_failure() == 0


def test_ogc_contacts_bitwise(cuda_lib, oracle_lib):
    """Once the cloth has landed on the soft cubes and boxes: element-contact
    records (order included), the merged adjacency and the bound anchors."""
    g, o, _ = run_ogc(small_mixed(), oracle_lib, 100, check_every=25)
    c = g.counters()
    assert c.soft_vt > 0 and c.soft_rt > 0
    gs, os_ = g.debug_read("SOFT"), o.debug_read("SOFT")
    assert gs.size > 0 and np.array_equal(gs, os_)
    for name in ["ADJ_START", "ADJ_COUNT", "ADJ_LIST", "OGC_PREV", "PARTICLE_IDX", "TRIS", "EDGES"]:
        a, b = g.debug_read(name), o.debug_read(name)
        assert np.array_equal(a, b), name


def test_two_cubes_stay_apart(cuda_lib):
    """The upper cube rests on the lower one: vertex-triangle contacts keep
    the surfaces separated (no vertex of the upper cube below the lower
    cube's top layer by more than a contact radius)."""
    s = demos.two_cubes_scene()
    n = 5
    from avbd_b200.solver import GPUSolver
    g = GPUSolver(s)
    g.step(180)
    pos, _ = g.positions()
    lower = pos[1:1 + n ** 3, 2]
    upper = pos[1 + n ** 3:1 + 2 * n ** 3, 2]
    radius = 0.3 / (n - 1) * 0.32
    assert np.isfinite(pos).all()
    assert upper.min() > lower.max() - 2 * radius, (upper.min(), lower.max())
    assert g.counters().soft_vt > 0


def test_mixed_full_size_runs(cuda_lib):
    """The mixed scene at full size (64 soft cubes of 10^3 vertices, 256
    boxes, a 128^2 cloth): 60 frames without a runtime failure and with
    element contacts of every kind."""
    from avbd_b200.solver import GPUSolver
    g = GPUSolver(demos.mixed_scene())
    g.step(60)
    pos, _ = g.positions()
    c = g.counters()
    print(f"mixed: soft {c.num_soft} (rt {c.soft_rt}, vt {c.soft_vt}, ee {c.soft_ee}), ogc {c.ogc_exceeded}")
    assert g.runtime_failure() == 0 and np.isfinite(pos).all()
    assert c.soft_vt > 0


def test_snapshot_restore_mixed_bitwise(cuda_lib):
    """Snapshots cover the element-contact state (soft contacts and their map,
    tracked sets, bound anchors): replaying from one repeats the frames bit
    for bit (the reference's snapshots refuse soft scenes,
    GPUSolver.swift:2985-2986)."""
    from avbd_b200.solver import GPUSolver
    g = GPUSolver(small_mixed())
    g.step(70)
    snap = g.snapshot()
    g.step(20)
    a, ra = g.positions()
    ca = g.counters()
    g.restore(snap)
    g.step(20)
    b, rb = g.positions()
    cb = g.counters()
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(ra.view(np.uint32), rb.view(np.uint32))
    assert (ca.num_soft, ca.soft_vt, ca.soft_ee, ca.soft_rt) == (cb.num_soft, cb.soft_vt, cb.soft_ee, cb.soft_rt)
