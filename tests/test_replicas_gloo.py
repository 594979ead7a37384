"""The replicas path across ranks: world-size-2 gloo process groups on the host.

Multi-GPU in this build is independent replicas (whole domains or requests per
rank, no data-path collective). What crosses ranks is the unit assignment and the
max-over-ranks job time; both are exercised here with two gloo ranks on CPU.
"""

from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

from rbsim import replicas


def _free_port() -> int:
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, costs, out):
    import torch.distributed as dist
    from datetime import timedelta

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        assert replicas.rank_world() == (rank, world)
        mine = replicas.shard_units(costs, world)[rank]
        units = float(sum(costs[i] for i in mine))
        seconds = 1.0 + rank  # rank 1 is the slow one
        rate, slowest = replicas.whole_job_rate(units, seconds)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        out.put((rank, mine, rate, slowest, gathered))
    finally:
        dist.destroy_process_group()


def _run(world: int, costs):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, costs, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return sorted(res)


def test_shard_units_lpt_is_deterministic_and_complete():
    costs = [5.0, 1.0, 4.0, 4.0, 2.0, 9.0, 0.0]
    a = replicas.shard_units(costs, 3)
    assert a == replicas.shard_units(costs, 3)
    assert sorted(i for units in a for i in units) == list(range(len(costs)))
    loads = [sum(costs[i] for i in units) for units in a]
    assert max(loads) - min(loads) <= max(costs)
    assert replicas.shard_units([], 2) == [[], []]
    with pytest.raises(ValueError):
        replicas.shard_units([1.0], 0)
    with pytest.raises(ValueError):
        replicas.shard_units([float("nan")], 2)


def test_single_process_fallbacks():
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.whole_job_rate(10.0, 2.0) == (5.0, 2.0)
    with pytest.raises(ValueError):
        replicas.whole_job_rate(1.0, 0.0)


def test_two_gloo_ranks_share_units_and_time_by_the_slowest():
    costs = [float(c) for c in (256, 2048, 512, 128, 1024, 768, 300, 40)]
    res = _run(2, costs)
    (_, mine0, rate0, slow0, gath0), (_, mine1, rate1, slow1, gath1) = res
    # every rank sees the same disjoint, complete assignment
    assert gath0 == gath1 == [mine0, mine1]
    assert not set(mine0) & set(mine1)
    assert sorted(mine0 + mine1) == list(range(len(costs)))
    # the job's time is the slowest rank's; the rate counts every rank's units
    assert slow0 == slow1 == 2.0
    assert rate0 == rate1 == pytest.approx(sum(costs) / 2.0)
