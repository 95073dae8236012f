"""Sharding of a batch across ranks (CPU): every system solved exactly once,
balanced sum(n^3), checked in-process and across two gloo ranks."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from linearalgebra_b200.batched import shard
from linearalgebra_b200.workloads import batch_sizes


def test_shard_partition_and_balance():
    sizes = batch_sizes(20000, seed=4)
    for world in (1, 2, 4, 8):
        parts = [shard(sizes, world, r) for r in range(world)]
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(len(sizes)))
        loads = [float((sizes[p].astype(float) ** 3).sum()) for p in parts]
        assert max(loads) / (sum(loads) / world) < 1.001


def _worker(rank, world, port, sizes, out):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = torch.from_numpy(shard(sizes, world, rank).astype(np.int64))
    counts = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(counts, torch.tensor([len(mine)]))
    mx = int(max(c.item() for c in counts))
    padded = torch.full((mx,), -1, dtype=torch.int64)
    padded[:len(mine)] = mine
    gathered = [torch.empty(mx, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(gathered, padded)
    if rank == 0:
        allidx = torch.cat([g[g >= 0] for g in gathered]).numpy()
        out.put(np.sort(allidx).tolist())
    dist.destroy_process_group()


def test_shard_across_two_gloo_ranks():
    sizes = batch_sizes(500, seed=9)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
    assert got == list(range(len(sizes)))
