"""Full-size parity of the benchmark scenes over their first 60 frames.

The four solver configurations at the sizes the benchmark runs them — the
24^3 soft cube, the 256^2 cloth over a sphere (Planar-DAT), 4096 batched
articulated worlds with new motor targets every frame, and the mixed scene
(64 soft cubes, 256 boxes, a 128^2 cloth; isotropic OGC) — stepped by the
CUDA solver and the CPU oracle side by side.

Every frame: positions, rotations and velocities within 1e-4 relative.
At frames 30 and 60: the spatial hash, the candidate pairs (order included),
the adjacency lists, the palette, the persistence map as a key -> value set,
the active manifolds and the element-contact records bit for bit.
"""
import os

import numpy as np
import pytest

from avbd_b200 import demos
from avbd_b200.solver import GPUSolver

from test_gpu_parity import assert_close

pytestmark = pytest.mark.gpu

FRAMES = 60
CHECK_AT = (30, 60)


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def compare_frame(g, o, frame):
    gp, gr = g.positions()
    op, orr = o.positions()
    assert_close(f"frame {frame} posLin", gp, op)
    assert_close(f"frame {frame} posAng", gr, orr)
    gs, os_ = g.body_states(), o.body_states()
    gv = np.array([list(s.velocity) + list(s.angular_velocity) for s in gs])
    ov = np.array([list(s.velocity) + list(s.angular_velocity) for s in os_])
    assert_close(f"frame {frame} velocity", gv, ov)
    return bool(np.array_equal(gp.view(np.uint32), op.view(np.uint32))
                and np.array_equal(gr.view(np.uint32), orr.view(np.uint32)))


def mapset(s):
    ka, kb, v = (s.debug_read(k, np.uint32) for k in ("MAP_KEY_A", "MAP_KEY_B", "MAP_VAL"))
    return {(int(a), int(b)): int(c) for a, b, c in zip(ka, kb, v) if a}


def compare_streams(g, o, frame, dynamic_palette, soft=False, dat=False):
    g.synchronize()
    gc, oc = g.counters(), o.counters()
    assert gc.num_pairs == oc.num_pairs, f"frame {frame}: pair count"
    assert gc.pair_candidates == oc.pair_candidates, f"frame {frame}: pair candidates"
    names = ["CELL_COUNT", "CELL_START", "CELL_BODIES", "ADJ_START", "ADJ_COUNT", "ADJ_LIST", "COLOR_START"]
    for name in names:
        a, b = g.debug_read(name, np.uint32), o.debug_read(name, np.uint32)
        assert a.size == b.size and np.array_equal(a, b), f"frame {frame}: {name}"
    n = int(gc.num_pairs)
    gpairs, opairs = g.debug_read("PAIRS", np.uint32), o.debug_read("PAIRS", np.uint32)
    assert np.array_equal(gpairs[:2 * n], opairs[:2 * n]), f"frame {frame}: PAIRS"
    lg, lo = g.debug_read("COLOR_LIST", np.uint32), o.debug_read("COLOR_LIST", np.uint32)
    if dynamic_palette:
        cs = g.debug_read("COLOR_START", np.uint32)
        for c in range(64):
            assert sorted(lg[cs[c]:cs[c + 1]]) == sorted(lo[cs[c]:cs[c + 1]]), f"frame {frame}: color {c}"
    else:
        assert np.array_equal(lg, lo), f"frame {frame}: static palette"
    assert mapset(g) == mapset(o), f"frame {frame}: persistence map"
    gm = g.debug_read("MANIFOLDS", np.uint32).reshape(-1, 176)
    om = o.debug_read("MANIFOLDS", np.uint32).reshape(-1, 176)
    for r in range(n):
        k = gm[r, 2]
        assert gm[r, 2] == om[r, 2], f"frame {frame}: manifold {r} contact count"
        assert np.array_equal(gm[r, :16 + 20 * k], om[r, :16 + 20 * k]), f"frame {frame}: manifold {r}"
    if soft:
        assert (gc.num_soft, gc.soft_candidates) == (oc.num_soft, oc.soft_candidates), f"frame {frame}: soft"
        ns = int(gc.num_soft)
        gs, os_ = g.debug_read("SOFT", np.uint32), o.debug_read("SOFT", np.uint32)
        assert np.array_equal(gs[:28 * ns], os_[:28 * ns]), f"frame {frame}: element contacts"
    if dat:
        assert (gc.dat_pairs, gc.dat_vt_pairs, gc.dat_ee_pairs, gc.dat_truncations) == \
               (oc.dat_pairs, oc.dat_vt_pairs, oc.dat_ee_pairs, oc.dat_truncations), f"frame {frame}: DAT"
        np_ = int(gc.dat_pairs)
        gd, od = g.debug_read("DAT_PAIRS", np.uint32), o.debug_read("DAT_PAIRS", np.uint32)
        assert np.array_equal(gd[:4 * np_], od[:4 * np_]), f"frame {frame}: DAT pair stream"


def run_full(scene, oracle_lib, *, dynamic_palette=False, soft=False, dat=False, motors=None, seed=0):
    g = GPUSolver(scene)
    o = oracle_lib.OracleSolver(scene, threads=host_threads())
    rng = np.random.default_rng(seed)
    exact = 0
    for f in range(1, FRAMES + 1):
        if motors is not None:
            t = rng.uniform(-0.5, 0.5, size=len(motors)).astype(np.float32)
            g.set_motor_targets(motors, t)
            o.set_motor_targets(motors, t)
        g.step(1)
        assert o.step(1) == 0, f"oracle failure at frame {f}"
        exact += compare_frame(g, o, f)
        if f in CHECK_AT:
            compare_streams(g, o, f, dynamic_palette, soft=soft, dat=dat)
    assert g.runtime_failure() == 0
    return g, o, exact


def test_soft_cube_24_sixty_frames(cuda_lib, oracle_lib):
    _, _, exact = run_full(demos.soft_cube_scene(seed=2, n=24), oracle_lib)
    print(f"soft-cube-24: {exact}/{FRAMES} frames bit-identical")


def test_batched_worlds_4096_sixty_frames(cuda_lib, oracle_lib):
    scene, motors, _ = demos.batched_worlds_scene(worlds=4096, seed=4)
    _, _, exact = run_full(scene, oracle_lib, dynamic_palette=True, motors=np.array(motors, np.uint32), seed=11)
    print(f"batched-worlds-4096: {exact}/{FRAMES} frames bit-identical")


def test_mixed_sixty_frames(cuda_lib, oracle_lib):
    _, _, exact = run_full(demos.mixed_scene(seed=5), oracle_lib, soft=True)
    print(f"mixed-64: {exact}/{FRAMES} frames bit-identical")


def test_cloth_sphere_256_sixty_frames(cuda_lib, oracle_lib):
    _, _, exact = run_full(demos.cloth_sphere_scene(seed=3, n=256), oracle_lib, soft=True, dat=True)
    print(f"cloth-sphere-256: {exact}/{FRAMES} frames bit-identical")
