"""Multi-GPU host logic on CPU: two gloo ranks split the benchmark's graph set
with bench.py's own split_by_work and combine their step times and counts with
bench.py's own reduce_over_ranks (max of times, sum of counts) -- no collective
touches the data path."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _bench():
    if REPO not in sys.path:
        sys.path.insert(0, REPO)
    import bench
    return bench


def _rank(rank, world, port, out):
    sys.path.insert(0, os.path.join(REPO, "parallel-vertex-cover-algorithms-on-gpus_b200"))
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    bench = _bench()
    from vcgpu import workloads as W
    import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    idx = bench.pinned_indices()[:24]
    graphs = [W.batch_instance(i) for i in idx]
    parts = bench.split_by_work(idx, [g.n * g.m for g in graphs], world)
    mine = parts[rank]
    recs = bench.golden_batch()
    solved = nodes = wrong = 0
    for i in mine:
        st, size, cover, nd = O.mvc(W.batch_instance(i), node_limit=5_000_000)
        solved += st == O.OK
        wrong += st == O.OK and size != recs[i]["opt"]
        nodes += nd
    (step,), (s_all, n_all, w_all, g_all) = bench.reduce_over_ranks(dist, [0.5 + rank], [solved, nodes, wrong, len(mine)])
    out[rank] = (step, s_all, n_all, w_all, g_all, solved, nodes, list(mine), [list(p) for p in parts])
    dist.destroy_process_group()


def test_split_by_work_balances_and_partitions():
    bench = _bench()
    idx = list(range(100))
    work = [float((i * 37) % 101 + 1) for i in idx]
    for world in (1, 2, 3, 8):
        parts = bench.split_by_work(idx, work, world)
        assert sorted(x for p in parts for x in p) == idx       # a partition of the set
        loads = [sum(work[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(work)            # LPT: within one item of balanced


def test_two_rank_split_and_reduction():
    world, port = 2, _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
    r0, r1 = out[0], out[1]
    assert r0[0] == r1[0] == 1.5                        # max of the step times
    assert r0[1] == r1[1] == r0[5] + r1[5]              # graphs solved, summed
    assert r0[2] == r1[2] == r0[6] + r1[6]              # tree nodes, summed
    assert r0[3] == r1[3] == 0                          # every answer equals the pinned optimum
    assert r0[4] == r1[4] == 24                         # every graph on exactly one rank
    assert set(r0[7]).isdisjoint(r1[7]) and r0[8] == r1[8]
