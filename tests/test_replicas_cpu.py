"""The N > 1 host logic on CPU: world-size-2 gloo ranks (the benchmark's max-over-ranks time and
whole-job rate, and the graph placement every rank must agree on)."""
import os
import socket

import pytest

from dyng_b200 import replicas as R


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # each replica timed its own steps; the job's time is the slowest rank's
        local_ms = 10.0 + 5.0 * rank
        mx = R.max_over_ranks(local_ms)
        rate = R.whole_job_rate(1_000_000, mx, world)
        sizes = [5e9, 1e9, 3e9, 3e9, 8e9, 2e9, 2e9, 1e9]
        placement = R.place_graphs(sizes, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, placement)
        dist.barrier()
        out.put((rank, mx, rate, gathered))
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas_agree():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, rate, gathered in results:
        assert mx == 15.0  # max over ranks, not the local time
        assert rate == pytest.approx(2 * 1_000_000 / 0.015)
        assert gathered[0] == gathered[1]  # every rank computes the same placement


def test_placement_balances_and_checks_capacity():
    sizes = [5e9, 1e9, 3e9, 3e9, 8e9, 2e9, 2e9, 1e9]
    ranks = R.place_graphs(sizes, 2)
    load = [sum(s for s, r in zip(sizes, ranks) if r == k) for k in range(2)]
    assert abs(load[0] - load[1]) <= max(sizes)
    assert R.place_graphs(sizes, 1) == [0] * len(sizes)
    with pytest.raises(MemoryError):
        R.place_graphs(sizes, 2, capacity_bytes=7e9)
    assert R.max_over_ranks(3.5) == 3.5  # no process group: the value itself
