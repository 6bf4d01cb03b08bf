"""The allocation-free scan entry point, through the C ABI.

`avbd_exclusive_scan_noalloc` serves callers that cannot call cudaMalloc (an
arena or pool that owns every device allocation, a real-time loop with an
allocation ban): its block-sum scratch is a fixed device array in the
library, not memory the call allocates.  Here two calls in a row are checked
word for word against the scan computed by the existing entry points — the
solver's own exclusive scan of its hash-bucket counts (avbd_step, read back
with avbd_debug_read) — and against numpy's exclusive cumulative sum (uint32
wraparound) of random words at ragged sizes up to the 1,048,576-word limit,
in place and out of place.  This file sorts last so that a run stopping at
the first failure has already run every other test; it also passes alone.
"""
import ctypes as C

import numpy as np
import pytest

from avbd_b200 import abi, demos
from avbd_b200.solver import GPUSolver, load_library

pytestmark = pytest.mark.gpu


def noalloc_scan(lib, host_words):
    import torch
    dev_in = torch.from_numpy(host_words.astype(np.int64).astype(np.int32)).cuda()
    dev_out = torch.empty_like(dev_in)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.avbd_exclusive_scan_noalloc(C.c_void_p(dev_in.data_ptr()), C.c_void_p(dev_out.data_ptr()),
                                         len(host_words), C.c_void_p(stream))
    torch.cuda.synchronize()
    return rc, dev_out.cpu().numpy().view(np.uint32)


def test_noalloc_scan_matches_solver_scan_twice(cuda_lib):
    lib = load_library()
    lib.avbd_exclusive_scan_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
    lib.avbd_exclusive_scan_noalloc.restype = C.c_int
    # two different scenes: a one-block scan (small hash table) and a
    # multi-block scan (32,768 buckets), called back to back
    for scene in (demos.soft_cube_scene(seed=21, n=6), demos.soft_cube_scene(seed=22, n=24)):
        solver = GPUSolver(scene)
        solver.step(2)
        solver.synchronize()
        counts = solver.debug_read("CELL_COUNT", np.uint32)
        want = solver.debug_read("CELL_START", np.uint32)
        rc, got = noalloc_scan(lib, counts)
        assert rc == abi.OK
        assert got.shape == want.shape and np.array_equal(got, want)
        solver.close()


def bind(lib):
    lib.avbd_exclusive_scan_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
    lib.avbd_exclusive_scan_noalloc.restype = C.c_int
    return lib


def exclusive_cumsum_u32(words):
    out = np.zeros(len(words), np.uint64)
    if len(words) > 1:
        out[1:] = np.cumsum(words[:-1].astype(np.uint64))
    return (out & 0xFFFFFFFF).astype(np.uint32)


@pytest.mark.parametrize("n", [1, 1023, 1025, 1_048_575, 1_048_576])
def test_noalloc_scan_matches_numpy(cuda_lib, n):
    """Random words (large values, so the sums wrap around 2^32): a partial
    last block, one word past a block, and the largest n (1024 blocks, every
    scratch word used); out of place, then in place on the same buffer."""
    import torch
    lib = bind(load_library())
    rng = np.random.default_rng(n)
    words = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
    want = exclusive_cumsum_u32(words)
    dev_in = torch.from_numpy(words.view(np.int32).copy()).cuda()
    dev_out = torch.empty_like(dev_in)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.avbd_exclusive_scan_noalloc(C.c_void_p(dev_in.data_ptr()), C.c_void_p(dev_out.data_ptr()), n, stream)
    torch.cuda.synchronize()
    assert rc == abi.OK
    assert np.array_equal(dev_out.cpu().numpy().view(np.uint32), want)
    assert np.array_equal(dev_in.cpu().numpy().view(np.uint32), words)    # input untouched
    rc = lib.avbd_exclusive_scan_noalloc(C.c_void_p(dev_in.data_ptr()), C.c_void_p(dev_in.data_ptr()), n, stream)
    torch.cuda.synchronize()
    assert rc == abi.OK
    assert np.array_equal(dev_in.cpu().numpy().view(np.uint32), want)


def test_noalloc_scan_rejects_partial_overlap(cuda_lib):
    import torch
    lib = bind(load_library())
    buf = torch.zeros(4096, dtype=torch.int32, device="cuda")
    rc = lib.avbd_exclusive_scan_noalloc(C.c_void_p(buf.data_ptr()), C.c_void_p(buf.data_ptr() + 4 * 16), 2048,
                                         None)
    assert rc == abi.ERR_INVALID_ARGUMENT


def test_noalloc_scan_rejects_oversize(cuda_lib):
    lib = load_library()
    lib.avbd_exclusive_scan_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
    lib.avbd_exclusive_scan_noalloc.restype = C.c_int
    rc = lib.avbd_exclusive_scan_noalloc(C.c_void_p(16), C.c_void_p(16), (1 << 20) + 1, None)
    assert rc == abi.ERR_INVALID_ARGUMENT
    buf = C.create_string_buffer(256)
    lib.avbd_last_error(None, buf, 256)
    assert b"1,048,576" in buf.value
