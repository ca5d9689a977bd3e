"""Multi-process (gloo, CPU) tests of the scene partition and the timing reduction."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from physica_b200 import distributed, scenes


def test_partition_covers_every_scene_once_and_balances():
    counts = scenes.batched_counts(4, 256, 2048, 65536, True)
    for world in (1, 2, 3, 8):
        parts = distributed.partition_scenes(counts, world)
        flat = sorted(s for p in parts for s in p)
        assert flat == list(range(len(counts)))
        loads = [sum(counts[s] for s in p) for p in parts]
        assert max(loads) - min(loads) <= max(counts)
    assert distributed.partition_scenes([5, 3], 4)[2:] == [[], []]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    counts = scenes.batched_counts(5, 32, 16384, 131072, False)
    mine = distributed.partition_scenes(counts, world)[rank]
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    t = distributed.max_over_ranks(float(rank + 1))
    out[rank] = (sorted(s for g in gathered for s in g), t)
    dist.destroy_process_group()


def test_two_rank_partition_and_max_reduction():
    world = 2
    manager = mp.Manager()
    out = manager.dict()
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        scenes_seen, tmax = out[r]
        assert scenes_seen == list(range(32))
        assert tmax == 2.0
