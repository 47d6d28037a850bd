"""The continuous-batching server: results are identical alone and in the mix,
requests submitted while others run are admitted and overlap, and node
budgets are honoured per request."""
import json
import os
import time

import numpy as np
import pytest

import oracle as O
import vcgpu
from vcgpu import workloads as W

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _mix(count, seed=0):
    """Small-to-medium graphs of both families with their oracle optimum."""
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < count:
        i = int(rng.integers(0, 10**6))
        if rng.random() < 0.5:
            n = int(rng.integers(20, 90))
            g = W.gnp(n, float(rng.uniform(3, 8)) / (n - 1), i)
        else:
            n = int(rng.integers(10, 40)) * 2
            g = W.random_regular(n, 3, i)
        st, opt, _, nodes = O.mvc(g, node_limit=200_000)
        if st == O.OK:
            out.append((g, opt))
    return out


def _check(g, r, instance, k, opt):
    assert r.status == vcgpu.VC_OK, (g.name, r)
    if instance == "mvc":
        assert r.size == opt and r.cover is not None
        assert W.is_cover(g, r.cover) and int(r.cover.sum()) == opt
    else:
        assert r.decision == (1 if opt <= k else 0), (g.name, k, opt)
        if r.decision:
            assert W.is_cover(g, r.cover) and int(r.cover.sum()) <= k


@pytest.mark.parametrize("max_vertices", [255, 2048])
def test_server_same_alone_and_in_mix(max_vertices):
    items = _mix(40, seed=max_vertices)
    jobs = []
    for j, (g, opt) in enumerate(items):
        if j % 3 == 0:
            jobs.append((g, "pvc", opt - (j % 2), opt))
        else:
            jobs.append((g, "mvc", 0, opt))
    with vcgpu.Server(max_vertices=max_vertices) as srv:
        alone = []
        for g, inst, k, opt in jobs[:8]:  # one at a time
            t = srv.submit(g, inst, k=k)
            alone.append(srv.wait(t))
        tickets = [srv.submit(g, inst, k=k) for g, inst, k, opt in jobs]  # all at once
        mixed = [srv.wait(t) for t in tickets]
    for (g, inst, k, opt), r in zip(jobs, mixed):
        _check(g, r, inst, k, opt)
    for (g, inst, k, opt), a, m in zip(jobs[:8], alone, mixed[:8]):
        _check(g, a, inst, k, opt)
        assert (a.size, a.decision, a.status) == (m.size, m.decision, m.status)
        # and the same as the plain one-graph entry point
        p = vcgpu.solve(g, inst, k=k, time_limit=60.0)
        assert (p.size, p.decision) == (m.size, m.decision)


def test_server_admits_while_running():
    """A long request runs while short ones arrive; the short ones finish first."""
    recs = [json.loads(l) for l in open(os.path.join(GOLDEN, "batch_seed0.jsonl"))]
    hard = sorted([r for r in recs if r["status"] == "ok" and 3_000_000 < r["nodes"] < 40_000_000],
                  key=lambda r: r["i"])[0]
    g_hard = W.batch_instance(hard["i"])
    small = _mix(20, seed=5)
    with vcgpu.Server(max_vertices=255) as srv:
        th = srv.submit(g_hard, "mvc")
        time.sleep(0.002)
        ts = [srv.submit(g, "mvc") for g, _ in small]
        rs = [srv.wait(t) for t in ts]
        done_small = time.time()
        rh = srv.wait(th)
        done_hard = time.time()
    for (g, opt), r in zip(small, rs):
        _check(g, r, "mvc", 0, opt)
    assert rh.status == vcgpu.VC_OK and rh.size == hard["opt"]
    assert done_small <= done_hard
    assert max(r.total_ms for r in rs) < rh.total_ms


def test_server_node_budget_per_request():
    recs = [json.loads(l) for l in open(os.path.join(GOLDEN, "batch_seed0.jsonl"))]
    big = [r for r in recs if r["status"] == "ok" and r["nodes"] > 200_000][0]
    g = W.batch_instance(big["i"])
    small = _mix(5, seed=9)
    with vcgpu.Server(max_vertices=255) as srv:
        tb = srv.submit(g, "mvc", node_limit=5000)
        ts = [srv.submit(h, "mvc") for h, _ in small]
        rb = srv.wait(tb)
        rs = [srv.wait(t) for t in ts]
    assert rb.status == vcgpu.VC_BUDGET and rb.size >= big["opt"]
    for (h, opt), r in zip(small, rs):
        _check(h, r, "mvc", 0, opt)


def test_server_rejects_oversize():
    with vcgpu.Server(max_vertices=100) as srv:
        with pytest.raises(RuntimeError):
            srv.submit(W.gnp(150, 0.05, 1), "mvc")


def test_server_completed_reports_each_ticket_once():
    """vc_server_completed hands out every finished ticket exactly once and
    never one that vc_server_poll already collected."""
    mix = _mix(40, seed=11)
    with vcgpu.Server(max_vertices=255) as srv:
        first = srv.submit(mix[0][0], "mvc")
        r0 = srv.wait(first)  # collected by poll before completed() sees it
        _check(mix[0][0], r0, "mvc", 0, mix[0][1])
        want = {srv.submit(g, "mvc"): (g, opt) for g, opt in mix[1:]}
        seen = []
        t0 = time.time()
        while len(seen) < len(want) and time.time() - t0 < 60:
            seen += srv.completed(max_tickets=7)
            time.sleep(0.001)
        assert sorted(seen) == sorted(want) and first not in seen
        for t in seen:
            g, opt = want[t]
            _check(g, srv.poll(t), "mvc", 0, opt)
        assert srv.completed() == []


def test_server_lanes_small_and_large():
    """With max_vertices above 255 the server runs a dense lane for small
    requests, a wide dense lane for 256..640 vertices with byte degrees and a
    CSR lane for the rest, side by side; results match the oracle-pinned optima
    alone and in a mix, and each request runs in its lane."""
    recs = [json.loads(l) for l in open(os.path.join(GOLDEN, "stream_seed0.jsonl"))]
    pinned = sorted([r for r in recs if r["status"] == "ok" and r["nodes"] <= 300_000], key=lambda r: r["i"])
    large = [r for r in pinned if r["n"] > 255][:6] + [r for r in pinned if r["n"] > 640][:2]
    small = [r for r in pinned if r["n"] <= 255][:18]
    assert large and small
    items = [(W.stream_instance(r["i"]), r["opt"]) for r in large + small]
    max_n = max(g.n for g, _ in items)
    with vcgpu.Server(max_vertices=max_n) as srv:
        g0, o0 = items[0]
        _check(g0, srv.wait(srv.submit(g0, "mvc")), "mvc", 0, o0)  # a large one alone
        tickets = [srv.submit(g, "mvc") for g, _ in items]
        tickets += [srv.submit(g, "pvc", k=opt - 1) for g, opt in items[::3]]
        res = [srv.wait(t) for t in tickets]
    for t, (g, _) in zip(tickets, items):  # narrow dense, wide dense (byte degrees), CSR
        deg_ok = int(np.diff(g.row_ptr).max()) <= 254
        want = 0 if g.n <= 255 else (1 if g.n <= 640 and deg_ok else 2)
        assert vcgpu.Server.lane(t) == want, (g.n, vcgpu.Server.lane(t))
    for (g, opt), r in zip(items, res):
        _check(g, r, "mvc", 0, opt)
    for (g, opt), r in zip(items[::3], res[len(items):]):
        _check(g, r, "pvc", opt - 1, opt)


def test_server_reuses_arena_blocks_while_running():
    """An arena that holds only a handful of graphs at a time serves a stream of
    many more: finished requests' blocks are reused while the lane's kernel keeps
    running (no stop-and-drain), and every answer is still exact."""
    recs = sorted((json.loads(l) for l in open(os.path.join(GOLDEN, "batch_seed0.jsonl")) if l.strip()),
                  key=lambda r: r["i"])
    easy = [r for r in recs if r["status"] == "ok" and r["nodes"] <= 20_000][:240]
    graphs = [(W.batch_instance(r["i"]), r["opt"]) for r in easy]
    biggest = max(((g.n + 1) + 2 * g.m) * 4 for g, _ in graphs)
    # one lane (max_vertices <= 255); its arena is the whole budget
    with vcgpu.Server(max_vertices=255, max_requests=64, mem_budget=6 * ((biggest + 255) // 256 * 256)) as srv:
        tickets = []
        for g, opt in graphs:
            tickets.append((srv.submit(g, "mvc"), g, opt))
        for tk, g, opt in tickets:
            r = srv.wait(tk, timeout=120.0)
            _check(g, r, "mvc", 0, opt)
