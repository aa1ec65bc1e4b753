"""Replica sharding over two CPU ranks (gloo): every mesh is owned by exactly
one rank, loads are balanced, and the max-over-ranks timing reduction works."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, sizes, q):
    import torch
    import torch.distributed as dist
    from gpu_cvt_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = replicas.partition(sizes, world, rank)
    load = float(sum(sizes[i] for i in mine))
    # gather every rank's shard
    t = torch.zeros(len(sizes), dtype=torch.int64)
    t[mine] = 1
    dist.all_reduce(t)
    tmax = replicas.max_over_ranks(10.0 + rank)
    tot = replicas.sum_over_ranks(load)
    q.put((rank, mine, load, t.tolist(), tmax, tot))
    dist.barrier()
    dist.destroy_process_group()


def test_partition_two_ranks_gloo():
    rng = np.random.default_rng(3)
    sizes = [int(x) for x in np.exp(rng.uniform(np.log(1e3), np.log(5e4), 256))]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    cover = out[0][3]
    assert cover == [1] * len(sizes)                    # each mesh on exactly one rank
    assert set(out[0][1]).isdisjoint(out[1][1])
    loads = [o[2] for o in out]
    assert abs(loads[0] - loads[1]) <= max(sizes)       # balanced to one item
    assert all(o[4] == 11.0 for o in out)               # max over ranks
    assert all(o[5] == sum(sizes) for o in out)


def test_partition_is_deterministic_and_total():
    from gpu_cvt_b200 import replicas
    sizes = [5, 3, 9, 1, 7, 7, 2]
    for w in (1, 2, 3, 8):
        parts = [replicas.partition(sizes, w, r) for r in range(w)]
        assert sorted(i for p in parts for i in p) == list(range(len(sizes)))
        assert parts == [replicas.partition(sizes, w, r) for r in range(w)]
