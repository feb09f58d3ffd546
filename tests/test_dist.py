"""Multi-rank host logic on CPU: two gloo ranks run the timing protocol of
bench.py (barrier, max over ranks) and shard the batched workload by channel;
the shards cover every channel once and balance the node counts."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, os.path.join(HERE, "..", "ek-pnp_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    import ekpnp
    from ekpnp.dist import Dist, shard_by_nodes
    d = Dist(backend="gloo", timeout_s=60)
    specs = ekpnp.batch_specs(512, seed=2)
    mine = shard_by_nodes(specs, d.world, d.rank)
    d.barrier()
    slowest = d.max(10.0 + rank)          # the timing protocol: the slowest rank's time
    shards = [None] * world
    dist.all_gather_object(shards, mine)
    d.close()
    out.put((rank, slowest, shards))


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_shard_and_time(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    import ekpnp
    specs = ekpnp.batch_specs(512, seed=2)
    for rank, slowest, shards in results:
        assert slowest == 10.0 + world - 1
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(512))
        loads = [sum(specs[i]["nx"] * specs[i]["ny"] for i in s) for s in shards]
        assert max(loads) - min(loads) <= max(s["nx"] * s["ny"] for s in specs)


def test_shard_single_rank_is_everything():
    import ekpnp
    from ekpnp.dist import shard_by_nodes
    specs = ekpnp.batch_specs(64, seed=5)
    assert shard_by_nodes(specs, 1, 0) == list(range(64))
