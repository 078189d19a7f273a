"""The host logic of the several-GPU path (gse_b200.multi) on the CPU: the
partition of a batch of independent systems across ranks, and the barrier and
max-over-ranks reduction of device times, run as two gloo ranks."""
import os
import socket

import numpy as np
import pytest


def test_partition_covers_every_system_once_and_balances():
    from gse_b200 import multi
    from gse_b200 import workloads as W
    syst = W.config_batch(256)
    costs = [multi.system_cost(y.n, y.grid) for y in syst]
    for world in (1, 2, 3, 4, 8):
        parts = multi.partition_systems(costs, world)
        assert len(parts) == world
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(256))
        loads = [sum(costs[i] for i in p) for p in parts]
        # longest-first greedy: within the largest single cost of the mean
        assert max(loads) - sum(loads) / world <= max(costs)
        assert parts == multi.partition_systems(costs, world)  # deterministic
    assert multi.partition_systems([], 2) == [[], []]
    with pytest.raises(ValueError):
        multi.partition_systems(costs, 0)


def test_max_over_ranks_without_a_group_is_the_value():
    from gse_b200 import multi
    assert multi.max_over_ranks(3.5) == 3.5
    multi.barrier()  # no process group: returns at once


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    from gse_b200 import multi
    from gse_b200 import workloads as W
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        syst = W.config_batch(256)
        parts = multi.partition_systems([multi.system_cost(y.n, y.grid) for y in syst], world)
        mine = parts[rank]
        multi.barrier()
        # each rank's "device time" differs; all must see the largest
        t = multi.max_over_ranks(1.0 + rank * 2.5)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        out.put((rank, t, gathered == parts, sorted(i for g in gathered for i in g) == list(range(256))))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_partition_and_max():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, same, cover in res:
        assert t == 3.5
        assert same and cover
