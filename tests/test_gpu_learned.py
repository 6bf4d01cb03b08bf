"""Learned warm start on the GPU: the BF16 tensor-core training kernels'
gradients against the float64 oracle, fused inference against the oracle,
the solver integration (a model that predicts no correction reproduces the
plain trajectory bit for bit) and that training lowers the loss."""
import numpy as np
import pytest

from avbd_b200 import abi, demos, learned
from avbd_b200.solver import GPUSolver

pytestmark = pytest.mark.gpu


def _random_batch(rng, B):
    X = rng.normal(size=(B, learned.DIN)).astype(np.float32)
    X[:, 15] = 1.0
    T = rng.normal(size=(B, learned.USED)).astype(np.float32)
    return X, T


def _norm(rng):
    n = np.zeros(learned.NNORM, np.float32)
    n[learned.XM:learned.XM + learned.DIN] = rng.normal(0, 0.1, learned.DIN)
    n[learned.XI:learned.XI + learned.DIN] = rng.uniform(0.5, 2.0, learned.DIN)
    n[learned.YM:learned.YM + learned.USED] = rng.normal(0, 0.1, learned.USED)
    n[learned.YS:learned.NNORM] = 1.0
    n[learned.YS:learned.YS + learned.USED] = rng.uniform(0.5, 2.0, learned.USED)
    return n


@pytest.mark.parametrize("B", [192, 4096])
def test_gradients_match_float64_oracle(cuda_lib, oracle_lib, B):
    from oracle import mlp_oracle as M
    rng = np.random.default_rng(B)
    p = learned.init_params(seed=B)
    p[M.OB1:M.OW2] = rng.normal(0, 0.1, M.HID)       # nonzero biases exercise every term
    p[M.OB3:M.OW4] = rng.normal(0, 0.1, M.HID)
    norm = _norm(rng)
    X, T = _random_batch(rng, B)
    loss, g = learned.gradients(p, norm, X, T)
    wl, wg = M.forward_backward(p, norm, X, T, rounded=True)
    assert abs(loss - wl) <= 1e-4 * max(1.0, abs(wl)), (loss, wl)
    for name, (a, b) in {"W1": (M.OW1, M.OB1), "b1": (M.OB1, M.OW2), "W2": (M.OW2, M.OB2),
                         "b2": (M.OB2, M.OW3), "W3": (M.OW3, M.OB3), "b3": (M.OB3, M.OW4),
                         "W4": (M.OW4, M.OB4), "b4": (M.OB4, M.NPARAM)}.items():
        err = np.linalg.norm(g[a:b] - wg[a:b]) / max(np.linalg.norm(wg[a:b]), 1e-12)
        assert err <= 5e-3, (name, err)


@pytest.mark.parametrize("n", [1, 127, 1000, 128 * 296 + 37])
def test_inference_matches_oracle(cuda_lib, oracle_lib, n):
    """The tcgen05 inference kernel (128-row tiles, persistent CTAs) against
    the float64 network with BF16-rounded weights and activations: a single
    row, a partial tile, several tiles, and more tiles than CTAs."""
    from oracle import mlp_oracle as M
    rng = np.random.default_rng(7)
    p = learned.init_params(seed=3)
    p[M.OB4:M.OB4 + 6] = [0.1, -0.2, 0.3, 0.05, -0.05, 0.15]
    norm = _norm(rng)
    X, _ = _random_batch(rng, n)
    y = learned.infer(p, norm, X)
    want = M.predict(p, norm, X, rounded=True)
    scale = np.abs(want).max()
    # the activations are rounded to BF16 (8-bit mantissa) between layers;
    # a different FP32 accumulation order can move a rounding by one BF16
    # ulp, so over tens of thousands of rows the largest deviation reaches a
    # few 1e-3 of the output scale while the typical one stays far below
    err = np.abs(y - want)
    assert err.max() <= 3e-3 * scale + 1e-6
    assert err.mean() <= 1e-4 * scale + 1e-7


def test_inference_wait_gives_up_and_leaves_the_device_usable(cuda_lib):
    """The inference kernel's wait for its MMA completion barrier is bounded:
    with no tensor-core work issued nothing ever arrives, the wait gives up
    after about a second, the call reports a runtime failure, and the next
    inference on the same device is correct."""
    import ctypes as C
    import torch
    from avbd_b200.solver import load_library
    rng = np.random.default_rng(1)
    p = learned.init_params(seed=2)
    norm = _norm(rng)
    X, _ = _random_batch(rng, 256)
    dev = torch.device("cuda", 0)
    prm = torch.from_numpy(p.astype(np.float32)).to(dev)
    nrm = torch.from_numpy(norm.astype(np.float32)).to(dev)
    Xd = torch.from_numpy(X.astype(np.float32)).to(dev)
    out = torch.zeros((256, learned.USED), dtype=torch.float32, device=dev)
    ws = torch.empty(1 << 17, dtype=torch.uint8, device=dev)
    rc = load_library().avbd_mlp_infer_wait_timeout_for_testing(
        prm.data_ptr(), nrm.data_ptr(), Xd.data_ptr(), 256, out.data_ptr(), ws.data_ptr(),
        C.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    assert rc == abi.ERR_RUNTIME_FAILURE
    from oracle import mlp_oracle as M
    y = learned.infer(p, norm, X)
    want = M.predict(p, norm, X, rounded=True)
    assert np.abs(y - want).max() <= 1e-3 * np.abs(want).max() + 1e-6


def _mixed_small():
    return demos.mixed_scene(seed=7, cubes=4, cube_n=4, boxes=4, cloth_n=10, pitch=0.5)


@pytest.mark.parametrize("name,make,trials,frames,rigid", [
    ("soft-cube-6, 2 trial sweeps", lambda: demos.soft_cube_scene(seed=3, n=6), 2, 40, False),
    ("soft-cube-6, kept trial sweep", lambda: demos.soft_cube_scene(seed=3, n=6), 1, 40, False),
    ("soft-cube-6, no trial sweep", lambda: demos.soft_cube_scene(seed=3, n=6), 0, 40, False),
    ("mixed-small, kept trial sweep", _mixed_small, 1, 80, False),
    ("mixed-small, rigid rows", _mixed_small, 1, 80, True),
    ("rigid-stack-20, rigid rows", lambda: demos.rigid_stack_scene(seed=1), 1, 60, True),
    ("batched-worlds-16, rigid rows, no trial sweep", lambda: demos.batched_worlds_scene(worlds=16, seed=4)[0],
     0, 40, True),
])
def test_zero_correction_model_reproduces_plain_frames(cuda_lib, name, make, trials, frames, rigid):
    """A model whose every prediction is zero: x_learned == x_plain, the
    race is a tie that the prediction wins, and the trajectory is the plain
    one bit for bit — with the trial sweeps undone, with the winner's sweep
    kept as the first iteration (its OGC bound count included), without a
    trial sweep, in a color-Jacobi scene whose predicted branch has its own
    pending-solve buffers, and with rigid-body rows (positions and
    orientations)."""
    s = make()
    plain, learn = GPUSolver(s), GPUSolver(s)
    norm = np.zeros(learned.NNORM, np.float32)
    norm[learned.XI:learned.XI + learned.DIN] = 1.0
    norm[learned.YS:learned.NNORM] = 1.0
    learn.set_warm_start_model(np.zeros(learned.NPARAM, np.float32), norm, trials, rigid=rigid)
    learn.set_warm_start_mode(abi.WARM_START_LEARNED)
    for f in range(frames):
        plain.step(1)
        learn.step(1)
        a, qa = plain.positions()
        b, qb = learn.positions()
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f
        assert np.array_equal(qa.view(np.uint32), qb.view(np.uint32)), f
    # every raced frame is a tie the prediction wins; the first frames of a
    # scene whose color launches are tuned (four primal variants, or up to
    # seven dynamic-coloring block shapes) time the launches instead of racing
    assert frames - (7 if rigid else 4) <= learn.counters().learn_accepted <= frames
    assert learn.counters().ogc_exceeded == plain.counters().ogc_exceeded


def test_training_learns_the_correction(cuda_lib):
    """Trained on the solver's own rollouts, the network explains most of the
    variance of the solve's correction of the plain warm start."""
    X, T = learned.collect(lambda seed: demos.soft_cube_scene(seed=seed, n=10), seeds=[1, 2], frames=60)
    assert X.shape[1] == learned.DIN and T.shape[1] == learned.USED and X.shape[0] == T.shape[0] > 1000
    assert not T[:, 3:].any()                          # particles: no rotation part
    m = learned.train(X, T, steps=800, batch=4096, lr=1e-3, log_every=100)
    pred = learned.infer(m.params, m.norm, X)
    explained = 1.0 - ((pred[:, :3] - T[:, :3]) ** 2).mean(axis=0) / T[:, :3].var(axis=0)
    print("loss history", [round(h, 4) for h in m.history], "explained variance", np.round(explained, 3))
    assert explained[2] > 0.5 and np.mean(m.history[-3:]) < np.mean(m.history[:2])


def test_learned_warm_start_lowers_the_residual(cuda_lib):
    """The committed soft-cube model, on a held-out seed: at equal iteration
    counts the learned warm start leaves a smaller median AL residual."""
    import os
    path = os.path.join(os.path.dirname(learned.__file__), "models", "soft_cube_24_warm_start.npz")
    model = learned.WarmStartModel.load(path)
    make = lambda seed: demos.soft_cube_scene(seed=seed, n=24)   # noqa: E731
    p = learned.evaluate(make, 201, None, 50, 10)
    q = learned.evaluate(make, 201, model, 50, 10)
    print(f"10 iterations: r/r0 plain {p['rel_residual_final']:.4f} learned {q['rel_residual_final']:.4f}, "
          f"accepted {q['accepted']}/{q['frames']}")
    assert q["accepted"] > 0 and q["rel_residual_final"] < p["rel_residual_final"]
