"""Multi-process host logic on the CPU: world-size-2 gloo groups exercise the rank sharding of
independent instances and the end-of-run reduction the benchmark uses for N GPUs."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, sizes, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    from awcm.dist import reduce_run, shard_instances

    mine = shard_instances(sizes, rank, world)
    points = float(sum(sizes[k] for k in mine))
    ms, total = reduce_run(10.0 + rank, points)
    q.put((rank, mine, ms, total))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_sharding_and_reduction_gloo(world):
    import numpy as np

    rng = np.random.default_rng(3)
    sizes = [int(16 * 2 ** (L - 1) + 1) for L in rng.integers(5, 10, size=37)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, sizes, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    owned = sorted(k for _, mine, _, _ in res for k in mine)
    assert owned == list(range(len(sizes)))  # a partition of the instances
    loads = [sum(sizes[k] for k in mine) for _, mine, _, _ in res]
    assert max(loads) - min(loads) <= max(sizes)  # balanced to within one instance
    for _, _, ms, total in res:
        assert ms == 10.0 + (world - 1)  # max over ranks
        assert total == float(sum(sizes))  # sum over ranks


def test_shard_single_rank():
    from awcm.dist import shard_instances

    assert shard_instances([5, 9, 3], 0, 1) == [0, 1, 2]
    with pytest.raises(ValueError):
        shard_instances([1], 2, 2)
