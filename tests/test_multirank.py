"""Multi-GPU host logic on CPU: two gloo ranks, each with its own shard of the
batched workload (weak scaling), combine their counts and the max of their
step times the way bench.py does -- no collective touches the data path."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import sys
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(repo, "parallel-vertex-cover-algorithms-on-gpus_b200"))
    sys.path.insert(0, os.path.join(repo, "oracle"))
    from vcgpu import workloads as W
    import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    graphs = W.rank_batch(12, rank)
    solved, nodes = 0, 0
    for g in graphs:
        st, size, cover, nd = O.mvc(g, node_limit=20000)
        solved += st == O.OK
        nodes += nd
    step = torch.tensor([0.5 + rank], dtype=torch.float64)
    dist.all_reduce(step, op=dist.ReduceOp.MAX)
    cnt = torch.tensor([solved, nodes], dtype=torch.float64)
    dist.all_reduce(cnt)
    ids = torch.tensor([hash((g.n, g.m, int(g.col.sum()))) % (1 << 31) for g in graphs], dtype=torch.int64)
    gathered = [torch.zeros_like(ids) for _ in range(world)]
    dist.all_gather(gathered, ids)
    out[rank] = (float(step[0]), int(cnt[0]), int(cnt[1]), solved, nodes,
                 [int(x) for t in gathered for x in t.tolist()])
    dist.destroy_process_group()


def test_two_rank_weak_scaling_reduction():
    world, port = 2, _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
    r0, r1 = out[0], out[1]
    assert r0[0] == r1[0] == 1.5                      # max over ranks
    assert r0[1] == r1[1] == r0[3] + r1[3]            # graphs solved, summed
    assert r0[2] == r1[2] == r0[4] + r1[4]            # tree nodes, summed
    ids = r0[5]
    assert len(set(ids[:12]) & set(ids[12:])) == 0    # disjoint shards
