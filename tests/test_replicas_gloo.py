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


def _bench_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    meshes, cfg, _ = bench.batched_workload(12, world)
    mine = bench.rank_share(meshes, world, rank)
    sites = int(sum(meshes[i][3].shape[0] for i in mine))
    t = torch.zeros(len(meshes), dtype=torch.int64)
    t[mine] = 1
    dist.all_reduce(t)
    tot = torch.tensor([sites], dtype=torch.int64)
    dist.all_reduce(tot)
    q.put((rank, t.tolist(), int(tot.item()), cfg))
    dist.barrier()
    dist.destroy_process_group()


def test_bench_batched_workload_shards_over_two_ranks_gloo():
    """bench.py --gpus 2 on the batched workload: each rank remeshes its share
    of the meshes, every mesh exactly once, the shares add up to the whole
    job's sites, and both ranks report the same configuration."""
    import sys
    sys.path.insert(0, os.path.abspath(os.path.join(os.path.dirname(__file__), "..")))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_bench_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=300) for _ in procs), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][1] == [1] * 12
    assert out[0][2] == out[0][3]["sites_total"]
    assert out[0][3] == out[1][3] and "2 GPUs" in out[0][3]["parallelism"]
