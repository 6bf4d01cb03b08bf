"""Record golden trajectories from the oracle pinned to the reference's kernels.

Run in a checkout where the reference's sources are present (they are read,
unchanged and where they lie, by oracle/ref.py):

    python tests/golden/make_golden.py

For each scene below the oracle steps the frames while the reference's own
kernels recompute every stage on the same state (oracle/ref_pin.cpp); the
script refuses to write a fixture unless every stage of every frame matched
word for word.  It stores, every `every` frames, the positions and rotations
(float32 bit patterns) in tests/golden/<scene>.npz, plus the per-stage
comparison counts.  These files let any machine — the GPU box included, where
the reference is absent — check the oracle and the CUDA path against
trajectories the reference's kernels produced.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "avbd-metal_b200")]

from avbd_b200 import demos  # noqa: E402
from oracle import ref  # noqa: E402


def small_mixed():
    return demos.mixed_scene(seed=7, cubes=4, cube_n=4, boxes=4, cloth_n=10, pitch=0.5)


# name -> (scene builder, frames, record every, primal check every k-th iteration)
SCENES = {
    "stack5": (lambda: demos.stack(5), 60, 5, 1),
    "rigid_stack20": (lambda: demos.rigid_stack_scene(seed=1), 90, 5, 1),
    "soft_cube6": (lambda: demos.soft_cube_scene(seed=5, n=6), 60, 5, 1),
    "hinge_worlds8": (lambda: demos.batched_worlds_scene(worlds=8, seed=5)[0], 60, 5, 1),
    "drape12": (lambda: demos.drape_scene(res=12), 60, 5, 1),
    "mixed_small": (small_mixed, 60, 5, 2),
}


def record(name):
    make, frames, every, primal_every = SCENES[name]
    o = ref.PinnedOracle(make(), primal_every=primal_every)
    pos, rot = [], []
    for f in range(1, frames + 1):
        assert o.step(1) == 0
        if f % every == 0:
            p, r = o.positions()
            pos.append(p.view(np.uint32).copy())
            rot.append(r.view(np.uint32).copy())
    st = o.stats()
    bad = {k: v for k, v in st.items() if v["mismatched"]}
    if bad:
        raise SystemExit(f"{name}: stages differ from the reference's kernels: {bad}")
    compared = np.array([st[k]["compared"] for k in ref.STAGES], np.int64)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), frames=np.int32(frames), every=np.int32(every),
                        pos_bits=np.stack(pos), rot_bits=np.stack(rot), stages=np.array(ref.STAGES),
                        compared=compared)
    print(name, dict(zip(ref.STAGES, compared.tolist())))


if __name__ == "__main__":
    ref.build()
    for n in (sys.argv[1:] or SCENES):
        record(n)
