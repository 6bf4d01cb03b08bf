"""The C ABI boundary on the CPU: the library builds for sm_100a, loads,
exports every entry point declared in include/avbd.h, its records have the
C layout, and construction without a GPU fails cleanly (no compute call)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from avbd_b200 import abi, build, demos
from avbd_b200.solver import AVBDError, GPUSolver, load_library

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "avbd.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(avbd_[a-z_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return load_library()


def test_header_declarations_match_python_list():
    assert declared_functions() == sorted(abi.EXPORTED)


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.check_output(["nm", "-D", "--defined-only", build.LIB], text=True)
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [f for f in declared_functions() if f not in exported]
    assert not missing, missing
    for f in declared_functions():
        assert hasattr(lib, f)


def test_record_layouts_match_c(tmp_path):
    structs = ["avbd_settings", "avbd_body_desc", "avbd_collider_desc", "avbd_joint_desc",
               "avbd_spring_desc", "avbd_tet_desc", "avbd_tri_desc", "avbd_exclusion_desc",
               "avbd_spinner_desc", "avbd_scene_desc", "avbd_body_state", "avbd_counters"]
    src = tmp_path / "sizes.c"
    src.write_text('#include <stdio.h>\n#include "avbd.h"\nint main(void){\n' + "".join(
        f'printf("%zu\\n", sizeof({s}));\n' for s in structs) + "return 0;}\n")
    exe = tmp_path / "sizes"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    sizes = [int(x) for x in subprocess.check_output([str(exe)], text=True).split()]
    py = [abi.Settings, abi.BodyDesc, abi.ColliderDesc, abi.JointDesc, abi.SpringDesc, abi.TetDesc,
          abi.TriDesc, abi.ExclusionDesc, abi.SpinnerDesc, abi.SceneDesc, abi.BodyState, abi.Counters]
    assert sizes == [C.sizeof(t) for t in py]


def test_build_targets_sm100a():
    # the library is compiled for exactly one target: sm_100a
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_create_without_device_fails_cleanly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(AVBDError) as e:
        GPUSolver(demos.stack(2))
    assert e.value.status == abi.ERR_NO_DEVICE


def test_invalid_scene_is_rejected(lib):
    s = demos.stack(1)
    s.colliders[0].body = 99          # owner out of range
    with pytest.raises(AVBDError) as e:
        GPUSolver(s)
    assert e.value.status == abi.ERR_INVALID_ARGUMENT


def test_null_arguments_are_rejected(lib):
    assert lib.avbd_create(None, None) == abi.ERR_INVALID_ARGUMENT
    assert lib.avbd_step(None, 1) == abi.ERR_INVALID_ARGUMENT
    assert lib.avbd_sync(None) == abi.ERR_INVALID_ARGUMENT


def test_batched_create_refuses_a_joint_between_worlds(lib):
    """avbd_create_batched validates the world partition before touching a
    device: a joint joining two worlds is an invalid argument."""
    from avbd_b200.scene import SceneJoint
    s, motors, offs = demos.batched_worlds_scene(worlds=3, seed=1, collision_groups=False)
    a, b = offs[0], offs[1]
    s.add_joint(SceneJoint(a, b, (0, 0, 0), (0, 0, 0)))
    with pytest.raises(AVBDError) as e:
        GPUSolver(s, world_offsets=list(offs) + [len(s.bodies)])
    assert e.value.status == abi.ERR_INVALID_ARGUMENT
    assert "joins two worlds" in str(e.value)


def test_batched_create_refuses_decreasing_offsets(lib):
    s, motors, offs = demos.batched_worlds_scene(worlds=3, seed=1, collision_groups=False)
    with pytest.raises(AVBDError) as e:
        GPUSolver(s, world_offsets=[offs[1], offs[0], len(s.bodies)])
    assert e.value.status == abi.ERR_INVALID_ARGUMENT
