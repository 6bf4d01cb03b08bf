"""The N > 1 path of bench.py on CPU: two `gloo` ranks, each owning its own
shard of batched worlds (weak scaling, no data-path collective), stepped by
the oracle; the max-over-ranks timing reduction and the shard ownership are
checked against single-process runs of the same shards."""
import hashlib
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WORLDS = 6
FRAMES = 15


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _shard_digest(rank, worlds=WORLDS, frames=FRAMES):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "avbd-metal_b200"))
    import bench
    import oracle
    bench.WORKLOAD_KEY = "batched-worlds"
    scene = bench.make_scene(rank, worlds=worlds)
    targets = bench.MotorTargets(frames)
    o = oracle.OracleSolver(scene, threads=1)
    for i in range(frames):
        targets.apply(o, i)
        assert o.step(1) == 0
    pos, rot = o.positions()
    h = hashlib.sha256(pos.tobytes() + rot.tobytes()).hexdigest()
    return h, len(scene.bodies), bench.dynamic_units(scene)


def _rank_main(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    digest, bodies, units = _shard_digest(rank)
    gathered = [None] * world
    dist.all_gather_object(gathered, (digest, bodies, units))
    slowest = bench.max_over_ranks(float(rank + 1) * 0.5, world)
    if rank == 0:
        out.put((gathered, slowest))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_worlds():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, slowest = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert slowest == 1.0                       # max over ranks of (0.5, 1.0)
    # each rank simulated exactly its own shard: digests equal single-process
    # runs of shards 0 and 1, and the shards differ from each other
    for r in range(2):
        assert gathered[r] == _shard_digest(r)
    assert gathered[0][0] != gathered[1][0]
    # whole-job units = sum over ranks (weak scaling)
    assert gathered[0][2] + gathered[1][2] == sum(g[2] for g in gathered)


def test_default_workload_under_torchrun_is_world_shards(monkeypatch):
    """bench.py --gpus N under torchrun (WORLD_SIZE > 1) measures the natural
    split — batched-world shards — unless a workload is named; one GPU
    defaults to the mixed scene."""
    import sys
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setattr(sys, "argv", ["bench.py", "--gpus", "2"])
    monkeypatch.setenv("WORLD_SIZE", "2")
    assert bench.parse().workload == "batched-worlds"
    monkeypatch.setenv("WORLD_SIZE", "1")
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    assert bench.parse().workload == "mixed"
