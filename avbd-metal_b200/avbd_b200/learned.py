"""Learned warm start: data collection from the solver's own rollouts,
training with the library's BF16 tensor-core kernels, and evaluation in
iterations-to-tolerance against the plain gamma warm start.

The network (csrc/learned.cu) maps 32 per-body features to the correction
the solve applies to the plain warm start: outputs 0-2 move a particle or a
rigid body's centre, outputs 3-5 rotate a rigid body (arc length at its
bounding radius); a model with `rigid=True` is applied to the rigid bodies
too.  Training runs on the GPU through
avbd_mlp_train_step (forward, backward and Adam are the library's kernels;
torch only owns the device buffers).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from . import abi
from .solver import GPUSolver, load_library

DIN, HID, DOUT, USED = 32, 128, 16, 6
RING = slice(25, 28)            # 1-ring aggregates among the features
NNORM, XM, XI, YM, YS = 96, 0, 32, 64, 80
NPARAM = HID * DIN + HID + 2 * (HID * HID + HID) + DOUT * HID + DOUT


def init_params(seed: int = 0) -> np.ndarray:
    """He-initialised weights, zero biases, small output layer."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, np.float32)
    o = 0
    for fan_out, fan_in, scale in ((HID, DIN, 1.0), (HID, HID, 1.0), (HID, HID, 1.0), (DOUT, HID, 0.1)):
        w = rng.normal(0.0, scale * math.sqrt(2.0 / fan_in), size=(fan_out, fan_in))
        p[o:o + fan_out * fan_in] = w.ravel()
        o += fan_out * fan_in + fan_out
    return p


def fit_norm(features: np.ndarray, targets: np.ndarray) -> np.ndarray:
    """Per-feature mean and 1/std, per-target mean and std (96 floats)."""
    n = np.zeros(NNORM, np.float32)
    mu = features.mean(axis=0)
    sd = features.std(axis=0)
    const = sd <= 1e-6                                  # constant features pass through
    n[XM:XM + DIN] = np.where(const, 0.0, mu)
    n[XI:XI + DIN] = np.where(const, 1.0, 1.0 / np.maximum(sd, 1e-6))
    n[YM:YM + USED] = targets.mean(axis=0)
    n[YS:YS + USED] = np.maximum(targets.std(axis=0), 1e-6)
    n[YS + USED:NNORM] = 1.0
    return n


@dataclass
class WarmStartModel:
    params: np.ndarray
    norm: np.ndarray
    history: List[float] = field(default_factory=list)
    rigid: bool = False            # trained on rigid-body rows as well as particles

    def save(self, path: str) -> None:
        np.savez(path, params=self.params, norm=self.norm, history=np.array(self.history, np.float32),
                 rigid=np.array(self.rigid))

    @staticmethod
    def load(path: str) -> "WarmStartModel":
        z = np.load(path)
        return WarmStartModel(z["params"].astype(np.float32), z["norm"].astype(np.float32),
                              list(z["history"]) if "history" in z else [],
                              bool(z["rigid"]) if "rigid" in z else False)


def collect(make_scene: Callable[[int], object], seeds: Sequence[int], frames: int, skip: int = 2,
            every: int = 1, motor_targets: Optional[Callable] = None, fraction: float = 1.0,
            rigid: bool = False):
    """Roll out the plain solver on seeded scene variants and record, per
    frame, the features and the solve's correction of the plain warm start
    (of a seeded random `fraction` of the rows, for large scenes); with
    `rigid` the rigid bodies' rows are recorded after the particles'.
    `motor_targets(solver, frame)` (default: the scene's `motor_drive`, if
    it has one) drives the scene's motors."""
    feats, targs = [], []
    rng = np.random.default_rng(12345)
    for seed in seeds:
        scene = make_scene(seed)
        drive = motor_targets or getattr(scene, "motor_drive", None)
        g = GPUSolver(scene)
        if rigid:
            g.set_warm_start_rigid(True)
        g.set_learning_capture(True)
        for f in range(frames):
            if drive is not None:
                drive(g, f)
            g.step(1)
            if f >= skip and (f - skip) % every == 0:
                x, t = g.learning_sample()
                if fraction < 1.0:
                    keep = rng.random(len(x)) < fraction
                    x, t = x[keep], t[keep]
                feats.append(x.copy())
                targs.append(t.copy())
        g.close()
    return np.concatenate(feats), np.concatenate(targs)


def train(features: np.ndarray, targets: np.ndarray, steps: int = 2000, batch: int = 8192, lr: float = 1e-3,
          seed: int = 0, norm: Optional[np.ndarray] = None, device: int = 0,
          log_every: int = 100) -> WarmStartModel:
    """Adam on the mean-squared error, on the GPU with the library's kernels."""
    import torch
    lib = load_library()
    dev = torch.device("cuda", device)
    norm = fit_norm(features, targets) if norm is None else norm
    X = torch.from_numpy(np.ascontiguousarray(features, np.float32)).to(dev)
    T = torch.from_numpy(np.ascontiguousarray(targets, np.float32)).to(dev)
    prm = torch.from_numpy(init_params(seed)).to(dev)
    nrm = torch.from_numpy(norm).to(dev)
    m = torch.zeros_like(prm)
    v = torch.zeros_like(prm)
    ws = torch.empty(lib.avbd_mlp_workspace_bytes(batch), dtype=torch.uint8, device=dev)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    stream = torch.cuda.current_stream(dev).cuda_stream
    hist = []
    n = X.shape[0]
    for step in range(1, steps + 1):
        idx = torch.randint(0, n, (batch,), device=dev, generator=gen)
        xb = X[idx].contiguous()
        tb = T[idx].contiguous()
        rc = lib.avbd_mlp_train_step(prm.data_ptr(), nrm.data_ptr(), xb.data_ptr(), tb.data_ptr(), batch,
                                     m.data_ptr(), v.data_ptr(), step, C.c_float(lr), ws.data_ptr(),
                                     loss.data_ptr(), stream)
        if rc != 0:
            raise RuntimeError(f"avbd_mlp_train_step failed: {rc}")
        if step % log_every == 0 or step == steps:
            # the steps run asynchronously; a tensor-core wait that gave up
            # since step 1 is latched in the workspace
            if lib.avbd_mlp_workspace_status(ws.data_ptr(), batch, stream) != 0:
                raise RuntimeError("avbd_mlp_train_step: a tensor-core wait gave up")
            hist.append(float(loss.item()) / USED)           # per-component mean squared error
    return WarmStartModel(prm.cpu().numpy(), norm, hist)


def gradients(params, norm, features, targets, device: int = 0):
    """(loss, gradient) of one batch from the library's kernels."""
    import torch
    lib = load_library()
    dev = torch.device("cuda", device)
    B = features.shape[0]
    prm = torch.from_numpy(np.ascontiguousarray(params, np.float32)).to(dev)
    nrm = torch.from_numpy(np.ascontiguousarray(norm, np.float32)).to(dev)
    X = torch.from_numpy(np.ascontiguousarray(features, np.float32)).to(dev)
    T = torch.from_numpy(np.ascontiguousarray(targets, np.float32)).to(dev)
    ws = torch.empty(lib.avbd_mlp_workspace_bytes(B), dtype=torch.uint8, device=dev)
    g = torch.zeros(NPARAM, dtype=torch.float32, device=dev)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    rc = lib.avbd_mlp_gradients(prm.data_ptr(), nrm.data_ptr(), X.data_ptr(), T.data_ptr(), B, ws.data_ptr(),
                                g.data_ptr(), loss.data_ptr(), torch.cuda.current_stream(dev).cuda_stream)
    if rc != 0:
        raise RuntimeError(f"avbd_mlp_gradients failed: {rc}")
    torch.cuda.synchronize(dev)
    return float(loss.item()), g.cpu().numpy()


def infer(params, norm, features, device: int = 0) -> np.ndarray:
    """Predictions [n][6] from the fused inference kernel."""
    import torch
    lib = load_library()
    dev = torch.device("cuda", device)
    n = features.shape[0]
    prm = torch.from_numpy(np.ascontiguousarray(params, np.float32)).to(dev)
    nrm = torch.from_numpy(np.ascontiguousarray(norm, np.float32)).to(dev)
    X = torch.from_numpy(np.ascontiguousarray(features, np.float32)).to(dev)
    out = torch.zeros((n, USED), dtype=torch.float32, device=dev)
    ws = torch.empty(1 << 17, dtype=torch.uint8, device=dev)
    rc = lib.avbd_mlp_infer(prm.data_ptr(), nrm.data_ptr(), X.data_ptr(), n, out.data_ptr(), ws.data_ptr(),
                            torch.cuda.current_stream(dev).cuda_stream)
    if rc != 0:
        raise RuntimeError(f"avbd_mlp_infer failed: {rc}")
    torch.cuda.synchronize(dev)
    return out.cpu().numpy()


def iterations_to_tolerance(trace: np.ndarray, r0_plain: float, tol: float) -> int:
    """First iteration k (1-based) with r_k / r0_plain <= tol, or -1."""
    rel = trace[2:] / max(r0_plain, 1e-300)
    hit = np.nonzero(rel <= tol)[0]
    return int(hit[0]) + 1 if hit.size else -1


def evaluate(make_scene: Callable[[int], object], seed: int, model: Optional[WarmStartModel], frames: int,
             iterations: int, skip: int = 2, trial_sweeps: int = 1,
             tolerances: Sequence[float] = (1e-1, 1e-2, 1e-3, 1e-6)) -> Dict[str, object]:
    """Per-frame residual traces of one rollout with the plain (model=None)
    or the learned warm start, at `iterations` iterations per frame."""
    scene = make_scene(seed)
    scene.settings.iterations = iterations
    drive = getattr(scene, "motor_drive", None)
    g = GPUSolver(scene)
    if model is not None:
        g.set_warm_start_model(model.params, model.norm, trial_sweeps, rigid=model.rigid)
        g.set_warm_start_mode(abi.WARM_START_LEARNED)
    g.set_residual_trace(True)
    its = {t: [] for t in tolerances}
    rel_final, rel_first = [], []
    for f in range(frames):
        if drive is not None:
            drive(g, f)
        g.step(1)
        if f < skip:
            continue
        tr = g.residual_trace(2 + iterations)
        r0 = tr[0]
        rel_first.append(tr[2] / max(r0, 1e-300))
        rel_final.append(tr[-1] / max(r0, 1e-300))
        for t in tolerances:
            its[t].append(iterations_to_tolerance(tr, r0, t))
    c = g.counters()
    g.close()
    return {"iterations_to_tolerance": its, "rel_residual_after_1": float(np.median(rel_first)),
            "rel_residual_final": float(np.median(rel_final)), "accepted": int(c.learn_accepted),
            "frames": frames - skip}


def matched_residual_iterations(make_scene: Callable[[int], object], seed: int, model: WarmStartModel,
                                plain_iterations: int, frames: int = 60,
                                candidates: Sequence[int] = None,
                                trial_sweeps: int = 1):
    """Smallest learned iteration count whose median relative residual
    (r_final / r0 of the plain warm start) is no larger than the plain warm
    start's at `plain_iterations`.  Every count from 4 up is tried in turn
    (the residual need not fall monotonically with the count).  Returns
    (iterations, plain residual, learned residual, accepted fraction)."""
    plain = evaluate(make_scene, seed, None, frames, plain_iterations, trial_sweeps=trial_sweeps)
    target = plain["rel_residual_final"]
    if candidates is None:
        candidates = range(4, plain_iterations)
    for k in candidates:
        if k >= plain_iterations:
            break
        r = evaluate(make_scene, seed, model, frames, k, trial_sweeps=trial_sweeps)
        if r["rel_residual_final"] <= target:
            return k, target, r["rel_residual_final"], r["accepted"] / max(1, r["frames"])
    r = evaluate(make_scene, seed, model, frames, plain_iterations, trial_sweeps=trial_sweeps)
    return plain_iterations, target, r["rel_residual_final"], r["accepted"] / max(1, r["frames"])


class _Rollout:
    """One solver of a seeded scene, rewound to its first frame for every
    evaluation (no scene rebuild per iteration count)."""

    def __init__(self, make_scene, seed, model, trial_sweeps):
        scene = make_scene(seed)
        self.drive = getattr(scene, "motor_drive", None)
        self.g = GPUSolver(scene)
        if model is not None:
            self.g.set_warm_start_model(model.params, model.norm, trial_sweeps, rigid=model.rigid)
            self.g.set_warm_start_mode(abi.WARM_START_LEARNED)
        self.g.set_residual_trace(True)
        self.start = self.g.snapshot()

    def run(self, iterations, frames, skip=2, tolerances=()):
        g = self.g
        g.restore(self.start)
        st = g.settings
        st.iterations = iterations
        g.settings = st
        its = {t: [] for t in tolerances}
        rel_final = []
        for f in range(frames):
            if self.drive is not None:
                self.drive(g, f)
            g.step(1)
            if f < skip:
                continue
            tr = g.residual_trace(2 + iterations)
            rel_final.append(tr[-1] / max(tr[0], 1e-300))
            for t in tolerances:
                its[t].append(iterations_to_tolerance(tr, tr[0], t))
        return float(np.median(rel_final)), its

    def close(self):
        self.g.close()


def matched_comparison(make_scene: Callable[[int], object], seed: int, model: WarmStartModel,
                       plain_iterations: int, frames: int = 120, trial_sweeps: int = 1,
                       tolerances: Sequence[float] = (0.5, 0.3, 0.2, 0.1, 1e-2, 1e-3, 1e-6),
                       budget: int = 60) -> Dict[str, object]:
    """Plain vs learned warm start at a matched AL residual.

    The matched level is the plain warm start's median r_final / r0 over the
    rollout at `plain_iterations`.  For the plain form every count from 4 to
    `plain_iterations` is evaluated (the residual need not fall monotonically
    with the count) and the smallest that reaches the level is reported; for
    the learned form, the smallest count from 4 up that reaches it.  Both
    forms are also run at `budget` iterations to report, for each tolerance,
    the median number of iterations to reach it (frames that never reach a
    tolerance count as `budget + 1`; a tolerance neither form reaches in half
    the frames is reported as None)."""
    plain = _Rollout(make_scene, seed, None, trial_sweeps)
    curve = {k: plain.run(k, frames)[0] for k in range(4, plain_iterations + 1)}
    target = curve[plain_iterations]
    plain_min = min(k for k, r in curve.items() if r <= target)
    _, p_its = plain.run(budget, frames, tolerances=tolerances)
    plain.close()
    learned = _Rollout(make_scene, seed, model, trial_sweeps)
    learned_k, learned_r = plain_iterations, None
    for k in range(4, plain_iterations + 1):
        r = learned.run(k, frames)[0]
        if r <= target:
            learned_k, learned_r = k, r
            break
    if learned_r is None:
        learned_r = learned.run(plain_iterations, frames)[0]
    _, q_its = learned.run(budget, frames, tolerances=tolerances)
    learned.close()
    itt = {}
    for t in tolerances:
        a = np.array([x if x > 0 else budget + 1 for x in p_its[t]])
        b = np.array([x if x > 0 else budget + 1 for x in q_its[t]])
        reached = (a <= budget).mean() >= 0.5 or (b <= budget).mean() >= 0.5
        itt[f"{t:g}"] = ({"plain": float(np.median(a)), "learned": float(np.median(b))} if reached else None)
    return {"target": float(target), "plain_curve": {str(k): float(v) for k, v in curve.items()},
            "plain_min_iterations": int(plain_min), "learned_iterations": int(learned_k),
            "learned_residual": float(learned_r), "iterations_to_tolerance": itt, "budget": budget}


def _soft_cube(seed):
    from . import demos
    return demos.soft_cube_scene(seed=seed, n=24)


def _mixed(seed):
    from . import demos
    return demos.mixed_scene(seed=seed)


class MotorDrive:
    """Joint targets U(+-0.5 rad) for every motor, a fresh draw each frame;
    frame f's draw depends only on (seed, f), so a rewound rollout replays
    the same targets."""

    def __init__(self, motors, seed):
        self.ids = np.asarray(motors, np.uint32)
        self.seed = seed

    def __call__(self, solver, frame):
        rng = np.random.default_rng((self.seed, frame))
        solver.set_motor_targets(self.ids, rng.uniform(-0.5, 0.5, len(self.ids)).astype(np.float32))


def _batched_worlds(seed):
    from . import demos
    scene, motors, _ = demos.batched_worlds_scene(worlds=4096, seed=seed)
    scene.motor_drive = MotorDrive(motors, seed)
    return scene


def _rigid_stack(seed):
    from . import demos
    return demos.rigid_stack_scene(seed=seed)


# scene families of the learned warm start (trained models: avbd_b200/models)
SCENES = {"soft-cube": _soft_cube, "mixed": _mixed, "batched-worlds": _batched_worlds, "rigid-stack": _rigid_stack}


def _main(argv=None):
    """Train a warm-start model from the solver's own rollouts:

      PYTHONPATH=avbd-metal_b200 python -m avbd_b200.learned [--scene soft-cube|mixed] --out MODEL.npz
    """
    import argparse
    ap = argparse.ArgumentParser(description=_main.__doc__)
    ap.add_argument("--out", required=True)
    ap.add_argument("--scene", choices=sorted(SCENES), default="soft-cube")
    ap.add_argument("--seeds", type=int, nargs="+", default=[100, 101, 102, 103])
    ap.add_argument("--frames", type=int, default=200)
    ap.add_argument("--every", type=int, default=2)
    ap.add_argument("--fraction", type=float, default=1.0, help="share of the vertices sampled per frame")
    ap.add_argument("--target-iterations", type=int, default=80,
                    help="iterations of the rollouts that give the targets (a more converged solve than the "
                         "iteration counts the model is used at)")
    ap.add_argument("--drop-ring", action="store_true",
                    help="train without the 1-ring features (25-27): their inputs and first-layer weights are zero")
    ap.add_argument("--rigid", action="store_true",
                    help="learn the rigid bodies' corrections as well as the particles'")
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--eval-seed", type=int, default=200)
    a = ap.parse_args(argv)
    scene = SCENES[a.scene]

    def rollout_scene(s):
        sc = scene(s)
        sc.settings.iterations = a.target_iterations
        return sc

    X, T = collect(rollout_scene, a.seeds, a.frames, every=a.every, fraction=a.fraction, rigid=a.rigid)
    if a.drop_ring:
        X[:, RING] = 0.0
    model = train(X, T, steps=a.steps, batch=a.batch, lr=a.lr)
    model.rigid = a.rigid
    if a.drop_ring:
        model.params[:HID * DIN].reshape(HID, DIN)[:, RING] = 0.0
    model.save(a.out)
    print(f"samples {len(X)}, loss {model.history[0]:.4f} -> {model.history[-1]:.4f}")
    for iters in (10, 20):
        p = evaluate(scene, a.eval_seed, None, 120, iters)
        q = evaluate(scene, a.eval_seed, model, 120, iters)
        print(f"{iters} iterations: median r/r0 plain {p['rel_residual_final']:.4f}, learned "
              f"{q['rel_residual_final']:.4f}, accepted {q['accepted']}/{q['frames']}")


if __name__ == "__main__":
    _main()
