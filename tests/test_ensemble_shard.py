"""Multi-rank ensembles on CPU (gloo): the size-balanced member partition and the result gather."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from discrete_adjoint_b200 import inputs
from discrete_adjoint_b200.ensemble import gather_results, shard_members


def test_partition_covers_every_member_once_and_balances():
    specs = inputs.ensemble_specs(64, seed=4)
    sizes = [s.side * s.side for s in specs]
    for world in (1, 2, 3, 8):
        parts = [shard_members(sizes, world, r) for r in range(world)]
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[k] for k in p) for p in parts]
        # greedy largest-first: no rank exceeds the mean by more than the largest member
        assert max(loads) - sum(loads) / world <= max(sizes)


def test_specs_are_seeded_and_in_range():
    a, b = inputs.ensemble_specs(16, seed=9), inputs.ensemble_specs(16, seed=9)
    assert a == b
    for s in a:
        assert 20.0 <= s.slope_deg <= 35.0 and 1e4 <= s.volume <= 1e6 and 12.0 <= s.bedfrict_deg <= 28.0
        assert 128 <= s.side <= 512 and s.side % 16 == 0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, sizes, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard_members(sizes, world, rank)
        # a stand-in result per member that only its owner can produce
        local = {k: (rank, sizes[k] * 2) for k in mine}
        allr = gather_results(local, world)
        q.put((rank, sorted(allr.items())))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_gather_returns_every_member_from_its_owner():
    sizes = [s.side * s.side for s in inputs.ensemble_specs(20, seed=5)]
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, sizes, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=100) for _ in range(world)]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    owners = {k: r for r in range(world) for k in shard_members(sizes, world, r)}
    for _, items in res:
        assert [k for k, _ in items] == list(range(len(sizes)))
        for k, (r, v) in items:
            assert r == owners[k] and v == 2 * sizes[k]
