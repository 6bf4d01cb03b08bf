#!/usr/bin/env python
"""Benchmark of the AVBD solver step on B200.

Workload: the soft-body configuration — a 24x24x24-vertex lattice of a 1 m
cube (13,824 particles, 60,835 Stable Neo-Hookean tets, 5 tets per cell),
E = 1e5 Pa, nu = 0.4, density 1000, dropped from 0.5 m onto a static ground,
friction 0.4, dt = 1/60, 20 iterations, static topology palette; seeded
synthetic scene (SplitMix64).  One step = one solver frame of the whole scene.

Metric: vertex-steps/s (dynamic particles x frames / second), plain AVBD warm
start.  `value` is device-timed with CUDA events on the solver's stream,
inputs resident in HBM, L2 flushed between timed steps; `e2e` is the same
metric through the C ABI with host buffers (positions uploaded from pinned
memory and read back every step).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload soft-cube|cloth-sphere|mixed|batched-worlds]

`--workload cloth-sphere` measures the cloth configuration instead: a
256 x 256 sheet of 2 m (65,536 particles, 130,050 StVK membranes, Bergou
bends, hard structural rods), two pinned corners, draped over a static
sphere, Planar-DAT truncation, dt = 1/120, 30 iterations.
`--workload mixed` measures the mixed configuration: 64 soft cubes of 10^3
vertices, 256 rigid boxes and a 128 x 128 cloth falling together, with
isotropic-OGC vertex-triangle, edge-edge and rigid-triangle contacts.
`--workload batched-worlds` measures 4096 independent articulated worlds
per GPU (body-steps/s; new motor targets every step); under torchrun each
rank owns its own 4096 worlds (weak scaling, no data-path collective).

Under torchrun (N > 1) every rank runs an independent replica of the scene
("replicas only": the coupled scene has no natural partition); time is the
max over ranks and `value` counts the vertices of all ranks.
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "avbd-metal_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "vertex-steps/s at matched AL residual: plain vs learned warm-start, 1 B200"
WORKLOADS = {
    "soft-cube": ("soft-cube-24: 24^3-vertex lattice of a 1 m cube, 13,824 particles, 60,835 "
                  "Stable Neo-Hookean tets, E=1e5 Pa, nu=0.4, rho=1000, friction 0.4, dt=1/60, "
                  "20 iterations, static palette, plain warm start"),
    "cloth-sphere": ("cloth-sphere-256: 256^2-vertex sheet of 2 m (65,536 particles, 130,050 StVK "
                     "membranes mu=lambda=1e4, Bergou bending 1e-3, hard structural rods), contact "
                     "radius 2e-3 m, two pinned corners, static sphere r=0.5 m, Planar-DAT, dt=1/120, "
                     "30 iterations, plain warm start"),
    "mixed": ("mixed-64: 64 soft cubes of 10^3 vertices (Stable Neo-Hookean E=5e4 Pa, nu=0.45, side 0.3 m), "
              "256 rigid boxes with edges U(0.1, 0.4) m and a 128^2 cloth (mu=lambda=1e4, bending 1e-3) falling "
              "together onto the ground (80,384 particles + 256 boxes, 233,280 tets, 32,258 triangles), "
              "isotropic OGC element contacts, dt=1/60, 20 iterations, plain warm start"),
    "batched-worlds": ("batched-worlds-4096: 4096 worlds (one collision group each) of a planar 3-7 link "
                       "hinge chain with implicit PD motors (targets U(+-0.5 rad) every step) and a welded "
                       "T block on a plane, friction 0.5, dt=1/60, 8 iterations, dynamic coloring; "
                       "worlds sharded across ranks"),
}
MOTORS = []
WORKLOAD_KEY = "soft-cube"
WORKLOAD = WORKLOADS[WORKLOAD_KEY]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="bound on the CPU baseline sample")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="soft-cube")
    ap.add_argument("--frames-only", action="store_true",
                    help="profiling runs: warm-up and timed frames of the workload only (no e2e, stage "
                         "profile, learned comparison or CPU baseline); prints ms per frame")
    ap.add_argument("--warm-start", choices=["plain", "learned"], default="plain",
                    help="with --frames-only: the warm start of the frames")
    ap.add_argument("--iterations", type=int, default=0, help="with --frames-only: override the iterations")
    ap.add_argument("--pusht-obs", action="store_true",
                    help="time the Push-T pixel-observation kernel instead (--obs-envs x --obs-res^2 x 3 "
                         "bytes per launch) and print its own JSON line")
    ap.add_argument("--obs-envs", type=int, default=4096)
    ap.add_argument("--obs-res", type=int, default=64)
    args = ap.parse_args()
    global WORKLOAD_KEY, WORKLOAD
    WORKLOAD_KEY, WORKLOAD = args.workload, WORKLOADS[args.workload]
    return args


def make_scene(rank=0, worlds=4096):
    from avbd_b200 import demos
    if WORKLOAD_KEY == "cloth-sphere":
        return demos.cloth_sphere_scene(seed=3, n=256)
    if WORKLOAD_KEY == "mixed":
        return demos.mixed_scene(seed=5)
    if WORKLOAD_KEY == "batched-worlds":
        # rank r owns worlds [r * worlds, (r + 1) * worlds)
        scene, motors, _ = demos.batched_worlds_scene(worlds=worlds, seed=4, first_world=worlds * rank)
        MOTORS[:] = motors
        return scene
    return demos.soft_cube_scene(seed=2, n=24)


class MotorTargets:
    """Per-step joint targets U(+-0.5 rad) of the batched workload, drawn
    ahead of the timed region (host arrays; uploaded by set_motor_targets)."""

    def __init__(self, steps, seed=11):
        import numpy as np
        rng = np.random.default_rng(seed)
        self.ids = np.array(MOTORS, np.uint32)
        self.t = rng.uniform(-0.5, 0.5, size=(max(1, steps), len(MOTORS))).astype(np.float32) if MOTORS else None

    def apply(self, solver, i):
        if self.t is not None:
            solver.set_motor_targets(self.ids, self.t[i % len(self.t)])


def dynamic_vertices(scene):
    """Units of the metric: dynamic particles plus dynamic rigid bodies
    (vertex-steps; body-steps for a rigid-only scene)."""
    return sum(1 for b in scene.bodies if b.is_dynamic)


def unit():
    return "body-steps/s" if WORKLOAD_KEY == "batched-worlds" else "vertex-steps/s"


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(x, world, device=None):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (the reference algorithm restated in C++) on the
# host cores, bounded to about `seconds` of work.
# ---------------------------------------------------------------------------
def cpu_run(seconds, threads, warmup=1, max_frames=200):
    import oracle
    oracle.build()
    scene = make_scene()
    nv = dynamic_vertices(scene)
    o = oracle.OracleSolver(scene, threads=threads)
    targets = MotorTargets(max_frames + warmup)
    for i in range(warmup):
        targets.apply(o, i)
        o.step(1)
    frames, t0 = 0, time.perf_counter()
    while frames < max_frames:
        targets.apply(o, warmup + frames)
        o.step(1)
        frames += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    return nv * frames / dt, frames, dt, nv


# ---------------------------------------------------------------------------
# Clock sampling during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                       "-i", str(self.gpu), "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(", ") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = max(smax, float(r[2]))
                for i, n in enumerate(names):
                    if r[5 + i].strip().lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic_per_launch():
    """DRAM bytes per primal launch from the committed ncu summary, or None."""
    name = "k_primal_soft_cube_24.md" if WORKLOAD_KEY == "soft-cube" else "k_primal_cloth_sphere_256.md"
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(path).read())
    return float(m.group(1)) if m else None


def primal_bytes_per_iteration(solver, scene):
    """Algorithmic (unique-byte) traffic of the primal over one iteration:
    per body 16 B position read + 16 B write + 16 B inertial target + 4 B
    color-list entry + 16 B static adjacency segment + 8 B contact segment,
    4 B per adjacency entry, one 64 B tet record per tet, 64 B manifold
    header/basis + 80 B per active contact; cloth adds 48 B per membrane and
    bend, 64 B per spring, 112 B per element contact."""
    import numpy as np
    nb = dynamic_vertices(scene) + sum(1 for b in scene.bodies if not b.is_particle and b.is_dynamic)
    adj = int(solver.debug_read("ADJ_COUNT", np.uint32).sum())
    man = solver.debug_read("MANIFOLDS", np.uint32).reshape(-1, 176)
    contacts = int(man[:, 2].sum()) if man.size else 0
    active = int((man[:, 2] > 0).sum()) if man.size else 0
    cloth = 0
    if scene.tris:
        cloth = (48 * (solver.debug_read("MEMBRANES").size // 48 + solver.debug_read("BENDS").size // 48)
                 + 64 * len(scene.springs) + solver.debug_read("SOFT").size)
    rigid = sum(1 for b in scene.bodies if not b.is_particle and b.is_dynamic)
    joints = sum(1 for j in scene.joints if j.stiffness_lin != 0 or j.stiffness_ang != 0 or j.motor_torque != 0)
    return (nb * (16 + 16 + 16 + 4 + 16 + 8) + 48 * rigid + 4 * adj + 64 * len(scene.tets) + 64 * active
            + 80 * contacts + 224 * joints + cloth)


# ---------------------------------------------------------------------------
MODELS = {"soft-cube": "soft_cube_24_warm_start.npz", "mixed": "mixed_warm_start.npz"}


def model_path():
    name = MODELS.get(WORKLOAD_KEY)
    return os.path.join(ROOT, "avbd-metal_b200", "avbd_b200", "models", name) if name else None


def timed_steps(solver, targets, first, K, stream, flush):
    """K frames, one CUDA-event pair per frame on the solver stream, with an
    untimed L2 flush before each; returns the summed device milliseconds."""
    import torch
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    for i in range(K):
        flush.zero_()
        targets.apply(solver, first + i)
        starts[i].record(stream)
        solver.step(1)
        ends[i].record(stream)
    torch.cuda.synchronize()
    return sum(s.elapsed_time(e) for s, e in zip(starts, ends))


def learned_comparison(args, world, dev, stream, flush, plain_value):
    """The same workload with the learned warm start, at the iteration count
    whose median AL residual matches the plain warm start's."""
    from avbd_b200 import GPUSolver, abi, demos, learned
    model = learned.WarmStartModel.load(model_path())
    plain_iters = make_scene().settings.iterations
    make = learned.SCENES[WORKLOAD_KEY]
    k, r_plain, r_learned, acc = learned.matched_residual_iterations(make, 200, model, plain_iters, frames=120)
    scene = make_scene()
    scene.settings.iterations = k
    solver = GPUSolver(scene, device=dev.index)
    solver.set_stream(stream.cuda_stream)
    solver.set_warm_start_model(model.params, model.norm, 1)
    solver.set_warm_start_mode(abi.WARM_START_LEARNED)
    targets = MotorTargets(1)
    solver.step(args.warmup)
    solver.synchronize()
    ms = max_over_ranks(timed_steps(solver, targets, 0, args.steps, stream, flush), world, dev)
    nv = dynamic_vertices(scene)
    accepted = solver.counters().learn_accepted
    solver.close()
    value = world * nv * args.steps / (ms / 1e3)
    return {"warm_start": "learned: 32-128-128-128-3 MLP, BF16 tensor-core inference, kept only when its "
                          "residual after 1 trial sweep is no worse than the plain warm start's",
            "iterations": k, "plain_iterations": plain_iters,
            "matched_median_rel_residual": {"plain": r_plain, "learned": r_learned,
                                            "definition": "r_final / r0(plain warm start), r = ||AL gradient||_2 "
                                                          "over all dynamic DOFs, median over frames 3-120 of seed 200"},
            "value": value, "unit": unit(), "ms_per_step": ms / args.steps,
            "speedup_vs_plain": value / plain_value,
            "accepted_frames": accepted / float(args.warmup + args.steps),
            "model": f"avbd_b200/models/{MODELS[WORKLOAD_KEY]} (trained on the GPU by avbd_mlp_train_step "
                     "from plain rollouts of held-out seeds at a higher iteration count)"}


def run_frames(args, local):
    """Warm-up and timed frames only: the command the committed ncu launch
    lists were taken with."""
    import torch
    from avbd_b200 import GPUSolver, abi, learned
    torch.cuda.set_device(local)
    scene = make_scene()
    if args.iterations:
        scene.settings.iterations = args.iterations
    solver = GPUSolver(scene, device=local)
    if args.warm_start == "learned":
        model = learned.WarmStartModel.load(model_path())
        solver.set_warm_start_model(model.params, model.norm, 1)
        solver.set_warm_start_mode(abi.WARM_START_LEARNED)
    targets = MotorTargets(args.warmup + args.steps)
    for i in range(args.warmup):
        targets.apply(solver, i)
        solver.step(1)
    solver.synchronize()
    t0 = time.perf_counter()
    for i in range(args.steps):
        targets.apply(solver, args.warmup + i)
        solver.step(1)
    solver.synchronize()
    print(json.dumps({"workload": WORKLOAD_KEY, "frames": args.steps, "warm_start": args.warm_start,
                      "iterations": scene.settings.iterations,
                      "wall_ms_per_frame": (time.perf_counter() - t0) / max(1, args.steps) * 1e3,
                      "runtime_failure": solver.runtime_failure()}), flush=True)
    solver.close()


def run_pusht_obs(args, local):
    """The Push-T observation kernel alone: a batch of --obs-envs
    environments after a few frames, --steps back-to-back renders into one
    device buffer timed with CUDA events on the solver stream (the output is
    larger than nothing cached: each launch writes every byte once)."""
    import numpy as np
    import torch
    from avbd_b200 import GPUSolver, demos
    torch.cuda.set_device(local)
    scene, envs = demos.pusht_scene(args.obs_envs, seed=1)
    solver = GPUSolver(scene, device=local)
    stream = torch.cuda.Stream()
    solver.set_stream(stream.cuda_stream)
    solver.step(max(1, args.warmup))
    table = demos.pusht_env_table(envs)
    res = args.obs_res
    out = torch.empty((args.obs_envs, res, res, 3), dtype=torch.uint8, device="cuda")
    for _ in range(3):
        solver.render_pusht_obs(table, res, device_out=out.data_ptr())
    solver.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(args.steps):
        solver.render_pusht_obs(table, res, device_out=out.data_ptr())
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / args.steps
    nbytes = args.obs_envs * res * res * 3
    peak, kind = measured_peaks()
    host = solver.render_pusht_obs(table, res)
    assert np.array_equal(host, out.cpu().numpy())
    print(json.dumps({"workload": "pusht-obs", "envs": args.obs_envs, "res": res, "bytes_per_launch": nbytes,
                      "launches": args.steps, "ms_per_launch": ms, "achieved_gbs": nbytes / ms / 1e6,
                      "peak_gbs": peak, "peak_kind": kind, "frac": nbytes / ms / 1e6 / peak}), flush=True)
    solver.close()


def run_ours(args, world, rank, local):
    import numpy as np
    import torch
    from avbd_b200 import GPUSolver

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    scene = make_scene(rank)
    nv = dynamic_vertices(scene)
    solver = GPUSolver(scene, device=local)
    targets = MotorTargets(args.steps + args.warmup + 400)
    stream = torch.cuda.Stream(device=dev)
    solver.set_stream(stream.cuda_stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)   # > 126 MB L2

    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            targets.apply(solver, i)
            solver.step(1)
        solver.synchronize()
        K = args.steps
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
        clocks = ClockSampler(local)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()
        clocks.start()
        time.sleep(0.2)
        for i in range(K):
            flush.zero_()
            targets.apply(solver, args.warmup + i)    # input staging, before the timed step
            starts[i].record(stream)
            solver.step(1)
            ends[i].record(stream)
        torch.cuda.synchronize()
        clock = clocks.stop()
        solver.synchronize()
        dev_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
        dev_ms = max_over_ranks(dev_ms, world, dev)
        value = world * nv * K / (dev_ms / 1e3)

        # e2e through the C ABI with host buffers
        E = min(K, 300)
        pos4 = torch.empty((len(scene.bodies), 4), dtype=torch.float32, pin_memory=True).numpy()
        xyz = torch.empty((len(scene.bodies), 3), dtype=torch.float32, pin_memory=True).numpy()
        solver.read_positions_into(pos4)
        xyz[:] = pos4[:, :3]
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(E):
            solver.set_positions(xyz)            # H2D: n x 12 B from pinned memory
            targets.apply(solver, args.warmup + K + i)
            solver.step(1)
            solver.read_positions_into(pos4)     # D2H: n x 16 B, synchronising read
            xyz[:] = pos4[:, :3]
        e2e_s = max_over_ranks(time.perf_counter() - t0, world, dev)
        h2d = int(xyz.nbytes) + (targets.t.shape[1] * 8 if targets.t is not None else 0)
        e2e = {"value": world * nv * E / e2e_s, "unit": unit(),
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": int(pos4.nbytes),
               "steps": E}

        # roofline of the dominant kernel (the per-color primal), from a
        # profiled pass with CUDA events around every primal launch
        prof_frames = 20
        solver.set_profiling(True)
        for i in range(prof_frames):
            targets.apply(solver, i)
            solver.step(1)
        prof = solver.profile()
        solver.set_profiling(False)
        bytes_iter = primal_bytes_per_iteration(solver, scene)
        counters = solver.counters()
        launches_iter = max(1, prof["stage_launches"]["primal"] // (prof_frames * scene.settings.iterations))
        bytes_launch = bytes_iter / launches_iter
        avg_ms = prof["stage_ms"]["primal"] / max(1, prof["stage_launches"]["primal"])
        peak, peak_kind = measured_peaks()
        achieved = bytes_launch / (avg_ms / 1e3) / 1e9
        total_ms = sum(prof["stage_ms"].values())
        stage_share = {k: round(v / total_ms, 4) for k, v in prof["stage_ms"].items() if v > 0}
        kernels_per_frame = prof["kernels_per_frame"]

    learned_line = None
    if model_path() and os.path.exists(model_path()):
        with torch.cuda.stream(stream):
            learned_line = learned_comparison(args, world, dev, stream, flush, value)

    cpu = None
    if rank == 0 and world == 1:
        thr = host_threads()
        cv, frames, secs, _ = cpu_run(args.cpu_seconds, thr)
        cpu = {"value": cv, "unit": unit(), "cores": thr, "kind": "port",
               "sample": f"{WORKLOAD.split(':')[0]}, frames 2-{frames + 1} after a 1-frame warm-up, "
                         f"{frames} frames in {secs:.1f} s, oracle with {thr} OpenMP threads"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": unit(), "n_gpus": world,
            "steps": K, "warmup": args.warmup, "ms_per_step": dev_ms / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded SplitMix64 scene)",
            "config": {"workload": WORKLOAD, "vertices_per_step": nv, "tets": len(scene.tets),
                       "triangles": len(scene.tris),
                       "iterations": scene.settings.iterations,
                       "colors": int(counters.used_colors),
                       "lanes_per_body": prof["color_lanes"][:int(counters.used_colors)],
                       "lane_autotune": "fastest of 8/16/32 lanes per color, timed on the first 3 frames",
                       "warm_start": "plain gamma warm start (value); learned warm start in learned_warm_start",
                       "parallelism": (f"world shards x{world}" if WORKLOAD_KEY == "batched-worlds"
                                       else f"replicas x{world}"),
                       "l2": "flushed between timed steps (256 MiB device write, untimed)",
                       "timing": "CUDA events on the solver stream per step, max over ranks"},
            "clocks": clock, "e2e": e2e,
            "gpu_launches": int(kernels_per_frame * K),
            "roofline": {"bound": "hbm", "kernel": "k_primal_group (per-color block-descent primal, 8/16/32 lanes per body)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured"
                         else "fallback 6.65 TB/s",
                         "traffic": ncu_traffic_per_launch(),
                         "algorithmic_bytes_per_launch": bytes_launch,
                         "avg_launch_us": avg_ms * 1e3, "launches_per_iteration": launches_iter,
                         "measured": f"profiled pass of {prof_frames} frames, CUDA events around every launch"},
            "stage_share": stage_share,
            "learned_warm_start": learned_line,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    solver.close()


def run_reference(args, world, rank):
    if rank != 0:
        return
    thr = host_threads()
    budget = max(10.0, min(150.0, 8.0 * args.cpu_seconds))
    import oracle
    oracle.build()
    scene = make_scene()
    nv = dynamic_vertices(scene)
    o = oracle.OracleSolver(scene, threads=thr)
    targets = MotorTargets(args.steps + 3)
    for i in range(min(args.warmup, 3)):
        targets.apply(o, i)
        o.step(1)
    frames, t0 = 0, time.perf_counter()
    while frames < args.steps:
        targets.apply(o, 3 + frames)
        o.step(1)
        frames += 1
        if time.perf_counter() - t0 >= budget:
            break
    secs = time.perf_counter() - t0
    value = nv * frames / secs
    sample = (f"{WORKLOAD.split(':')[0]}, {frames} of {args.steps} requested frames after "
              f"{min(args.warmup, 3)} warm-up frames, bounded to {budget:.0f} s; the reference's "
              "solver restated in C++ (Swift/Metal cannot run here), OpenMP over bodies of a color")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": unit(),
        "n_gpus": world, "steps": frames, "warmup": min(args.warmup, 3),
        "ms_per_step": secs / frames * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded SplitMix64 scene)",
        "config": {"workload": WORKLOAD, "vertices_per_step": nv, "parallelism": "host cores"},
        "cpu_baseline": {"value": value, "unit": unit(), "cores": thr, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": unit(), "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.pusht_obs:
            run_pusht_obs(args, local)
        elif args.frames_only:
            run_frames(args, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            if dist.is_initialized():
                dist.destroy_process_group()


if __name__ == "__main__":
    main()
