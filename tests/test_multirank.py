"""The multi-GPU path on CPU: two gloo ranks split a batched workload with `balanced_shards`, each
computes its shard (with the oracle: this checks the host-side sharding and gathering, not the
device), and the gathered results cover every instance exactly once and equal a single-rank run."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    from datetime import timedelta

    from conftest import load_package

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    load_package()
    from oracle import oracle as O
    from theeggman_b200 import shard, workloads as W

    degrees = [8, 10, 12, 14, 8, 16, 10, 12, 14, 16, 8, 12]
    mats = [W.dense_complex(N, 900 + i, 0.5) for i, N in enumerate(degrees)]
    parts = shard.balanced_shards([shard.dp_cost(N) for N in degrees], world)
    mine = {i: complex(O.haf_dp(mats[i])) for i in parts[rank]}
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    if rank == 0:
        q.put((parts, gathered))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharding_covers_every_instance(orc, W):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    parts, gathered = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    seen = sorted(i for g in gathered for i in g)
    assert seen == list(range(12))
    degrees = [8, 10, 12, 14, 8, 16, 10, 12, 14, 16, 8, 12]
    merged = {k: v for g in gathered for k, v in g.items()}
    for i, N in enumerate(degrees):
        assert merged[i] == complex(orc.haf_dp(W.dense_complex(N, 900 + i, 0.5)))
    # balanced: neither rank carries more than the other plus the largest single instance
    from theeggman_b200 import shard

    loads = [sum(shard.dp_cost(degrees[i]) for i in p) for p in parts]
    assert max(loads) - min(loads) <= shard.dp_cost(16)


def test_shard_helpers(egg):
    from theeggman_b200 import shard

    for n, world in ((10, 3), (7, 8), (0, 2), (100, 4)):
        rs = [shard.shard_range(n, world, r) for r in range(world)]
        assert sorted(i for r in rs for i in r) == list(range(n))
    costs = [5, 1, 1, 1, 1, 1]
    assert shard.balanced_shards(costs, 2) == [[0], [1, 2, 3, 4, 5]]
