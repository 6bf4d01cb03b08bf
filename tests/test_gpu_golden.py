"""The CUDA solver against trajectories recorded while the reference's own
kernels recomputed every stage of the oracle (tests/golden/make_golden.py).

Bit-exact is the expectation (the kernels evaluate the same float32
expressions in the same order); the bar is 1e-4 relative per recorded frame.
"""
import numpy as np
import pytest

from avbd_b200.solver import GPUSolver

from test_golden import SCENES, replay
from test_gpu_parity import assert_close

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(SCENES))
def test_cuda_reproduces_reference_kernel_trajectory(cuda_lib, name):
    g = GPUSolver(SCENES[name][0]())
    exact = total = 0
    for f, p, r, gp, gr in replay(g, name):
        assert_close(f"{name} frame {f} pos", p.view(np.float32), gp.view(np.float32))
        assert_close(f"{name} frame {f} rot", r.view(np.float32), gr.view(np.float32))
        exact += bool(np.array_equal(p, gp) and np.array_equal(r, gr))
        total += 1
    print(f"{name}: {exact}/{total} recorded frames bit-identical to the reference-kernel trajectory")
