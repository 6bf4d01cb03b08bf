"""Capacity failures of the element-contact pipelines, provoked on small
scenes by lowering a capacity (the reference's `*CapacityForTesting`
overrides, GPUSolver.swift:2117-2133): the CUDA solver latches the same
failure on the same frame as the oracle, the frames before it agree with the
oracle, and the failure is sticky — every later call, state reads included,
raises it again (counters stay readable).  Nothing here faults or stalls a
GPU: the failures are counters read back on the host."""
import pytest

from avbd_b200 import abi, demos
from avbd_b200.solver import RuntimeFailure

from test_gpu_parity import compare_state, pair

pytestmark = pytest.mark.gpu


def run_until_failure(scene, oracle_lib, which, value, frames, **kw):
    g, o = pair(scene, oracle_lib, **kw)
    g.set_capacity_for_testing(which, value)
    o.set_capacity_for_testing(which, value)
    for f in range(frames):
        g.step(1)
        rc = o.step(1)
        try:
            g.synchronize()
        except RuntimeFailure as e:
            assert rc != 0, f"the CUDA solver failed at frame {f + 1}, the oracle did not"
            return g, o, f + 1, e
        assert rc == 0, f"the oracle failed at frame {f + 1}, the CUDA solver did not"
        compare_state(g, o, f + 1)
    pytest.fail(f"no failure within {frames} frames")


def assert_sticky(g, kind):
    assert g.runtime_failure() == kind
    with pytest.raises(RuntimeFailure) as again:
        g.step(1)
    assert again.value.kind == kind
    with pytest.raises(RuntimeFailure):
        g.synchronize()
    with pytest.raises(RuntimeFailure):
        g.positions()


@pytest.mark.parametrize("name,make,kw", [
    ("drape-planar-dat", lambda: demos.drape_scene(res=16), {}),
    ("two-cubes-isotropic", lambda: demos.two_cubes_scene(), {}),
])
def test_soft_contact_capacity(cuda_lib, oracle_lib, name, make, kw):
    g, o, frame, e = run_until_failure(make(), oracle_lib, abi.CAPACITY_SOFT_CONTACTS, 6, 150, **kw)
    print(f"{name}: soft-contact capacity failure at frame {frame}: {e}")
    assert e.kind == abi.FAIL_SOFT_CONTACT_CAPACITY
    assert o.runtime_failure() == abi.FAIL_SOFT_CONTACT_CAPACITY
    assert g.counters().soft_candidates > 6
    assert_sticky(g, abi.FAIL_SOFT_CONTACT_CAPACITY)


def test_planar_dat_pair_capacity(cuda_lib, oracle_lib):
    g, o, frame, e = run_until_failure(demos.drape_scene(res=16), oracle_lib, abi.CAPACITY_PLANAR_DAT_PAIRS, 4, 150)
    print(f"Planar-DAT pair capacity failure at frame {frame}: {e}")
    assert e.kind == abi.FAIL_PLANAR_DAT_PAIR_CAPACITY
    assert o.runtime_failure() == abi.FAIL_PLANAR_DAT_PAIR_CAPACITY
    assert g.counters().dat_pairs > 4
    assert_sticky(g, abi.FAIL_PLANAR_DAT_PAIR_CAPACITY)
