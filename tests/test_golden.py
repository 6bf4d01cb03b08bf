"""The oracle against trajectories recorded while the reference's own kernels
recomputed every stage (tests/golden/make_golden.py, oracle/ref_pin.cpp).

Each fixture holds the float32 bit patterns of every body's position and
rotation every few frames; the oracle must reproduce them bit for bit.  The
fixtures travel with the repository, so this pin holds on machines where the
reference's sources are absent.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_golden import SCENES  # noqa: E402

GOLDEN = os.path.join(HERE, "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


def replay(solver, name):
    g = load(name)
    frames, every = int(g["frames"]), int(g["every"])
    k = 0
    for f in range(1, frames + 1):
        solver.step(1)
        if f % every == 0:
            p, r = solver.positions()
            yield f, p.view(np.uint32), r.view(np.uint32), g["pos_bits"][k], g["rot_bits"][k]
            k += 1


@pytest.mark.parametrize("name", sorted(SCENES))
def test_oracle_reproduces_reference_kernel_trajectory(oracle_lib, name):
    make = SCENES[name][0]
    o = oracle_lib.OracleSolver(make(), threads=4)
    for f, p, r, gp, gr in replay(o, name):
        assert np.array_equal(p, gp), f"{name} frame {f}: positions differ from the fixture"
        assert np.array_equal(r, gr), f"{name} frame {f}: rotations differ from the fixture"
    assert load(name)["compared"].sum() > 0
