"""The multi-rank paths of bench.py on the CPU: the ensemble's member sharding (host logic) and the
max / sum reductions over ranks, run as two gloo ranks on 127.0.0.1 (no GPU; the GPU runs use NCCL)."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402
import nsfsi  # noqa: E402


def ensemble_nodes():
    return [int(c.NI * c.NJ * c.NK) for c in nsfsi.ensemble_configs(n=64, steps=200)]


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_shards_cover_every_member_once_and_balance(world):
    nodes = ensemble_nodes()
    parts = bench.shard_members(nodes, world)
    assert len(parts) == world
    flat = sorted(m for p in parts for m in p)
    assert flat == list(range(len(nodes)))
    loads = [sum(nodes[m] for m in p) for p in parts]
    assert max(loads) - min(loads) <= max(nodes)  # LPT: within one member of each other
    assert bench.shard_members(nodes, world) == parts  # deterministic


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mx = bench.reduce_over_ranks(1.5 + rank, dist, "max")
        sm = bench.reduce_over_ranks(1.5 + rank, dist, "sum")
        mine = bench.shard_members(ensemble_nodes(), world)[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        out.put((rank, mx, sm, gathered))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_and_shard():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    nodes = ensemble_nodes()
    for rank, mx, sm, gathered in res:
        assert mx == 2.5 and sm == 1.5 + 2.5
        assert sorted(m for g in gathered for m in g) == list(range(len(nodes)))
        assert gathered == bench.shard_members(nodes, world)

