"""GPU parity: the CUDA search (through the C ABI) against the CPU oracle.

The bar is bit-exact: the MVC size equals the oracle's optimum (the oracle is
the restatement of the reference's Sequential(), pinned to the reference's own
compiled solver by tests/test_oracle.py), every PVC decision equals the
oracle's, and every returned cover is checked edge by edge and has exactly the
reported size.
"""
import json
import os

import numpy as np
import pytest

import oracle as O
import vcgpu
from vcgpu import workloads as W

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TL = 60.0  # seconds: every solve here finishes far below this


def _check_mvc(g, r, opt):
    assert r.status == vcgpu.VC_OK, (g.name, r)
    assert r.size == opt, (g.name, r.size, opt)
    assert r.cover is not None, g.name
    assert int(r.cover.sum()) == opt, g.name
    assert W.is_cover(g, r.cover), g.name


def _check_pvc(g, r, k, expect):
    assert r.status == vcgpu.VC_OK, (g.name, k, r)
    assert r.decision == expect, (g.name, k, r.decision, expect)
    if expect:
        assert r.cover is not None and W.is_cover(g, r.cover) and int(r.cover.sum()) <= k
        assert r.size == int(r.cover.sum())


def test_config1_gnp60():
    g = W.config1_graph()
    small = json.load(open(os.path.join(GOLDEN, "small.json")))
    opt = small["config1"]["opt"]
    _check_mvc(g, vcgpu.solve(g, "mvc", time_limit=TL), opt)
    _check_pvc(g, vcgpu.solve(g, "pvc", k=opt, time_limit=TL), opt, 1)
    _check_pvc(g, vcgpu.solve(g, "pvc", k=opt - 1, time_limit=TL), opt - 1, 0)


def test_config2_planted_cover():
    g = W.config2_graph()
    small = json.load(open(os.path.join(GOLDEN, "small.json")))
    opt = small["config2"]["opt"]
    _check_mvc(g, vcgpu.solve(g, "mvc", time_limit=TL), opt)
    _check_pvc(g, vcgpu.solve(g, "pvc", k=opt, time_limit=TL), opt, 1)
    _check_pvc(g, vcgpu.solve(g, "pvc", k=opt - 1, time_limit=TL), opt - 1, 0)


def test_exhaustive_small_graphs_batched():
    """Every graph on <= 5 vertices plus a seeded sample on 6 and 7 vertices, all
    in one batched launch (empty graphs, isolated vertices, K2, triangles ...)."""
    import itertools
    small = json.load(open(os.path.join(GOLDEN, "small.json")))
    graphs, opts = [], []
    for n, mask, opt in small["exhaustive"]:
        pairs = list(itertools.combinations(range(n), 2))
        e = [pairs[j] for j in range(len(pairs)) if (mask >> j) & 1]
        graphs.append(W.from_edges(n, np.asarray(e, dtype=np.int64).reshape(-1, 2), f"n{n}_m{mask}"))
        opts.append(opt)
    st, sols = vcgpu.solve_batch(W.pack(graphs), "mvc", time_limit=TL)
    assert st == vcgpu.VC_OK
    for g, r, opt in zip(graphs, sols, opts):
        assert r.status == vcgpu.VC_OK and r.size == opt, (g.name, r, opt)
        assert r.cover is not None and W.is_cover(g, r.cover) and int(r.cover.sum()) == opt, g.name


@pytest.mark.parametrize("seed", range(12))
def test_random_gnp_vs_oracle(seed):
    rng = np.random.default_rng(1000 + seed)
    n = int(rng.integers(10, 90))
    d = float(rng.uniform(1.0, 8.0))
    g = W.gnp(n, min(1.0, d / max(n - 1, 1)), 5000 + seed)
    st, opt, _, _ = O.mvc(g)
    assert st == O.OK
    _check_mvc(g, vcgpu.solve(g, "mvc", time_limit=TL), opt)
    for k, expect in ((opt, 1), (opt - 1, 0), (opt + 3, 1), (max(opt - 5, 0), 0 if opt > 0 else 1)):
        if k < 0:
            continue
        _check_pvc(g, vcgpu.solve(g, "pvc", k=k, time_limit=TL), k, expect)


@pytest.mark.parametrize("seed", range(4))
def test_random_regular_vs_oracle(seed):
    g = W.random_regular(40 + 10 * seed, 3, 77 + seed)
    st, opt, _, _ = O.mvc(g)
    assert st == O.OK
    _check_mvc(g, vcgpu.solve(g, "mvc", time_limit=TL), opt)
    _check_pvc(g, vcgpu.solve(g, "pvc", k=opt - 1, time_limit=TL), opt - 1, 0)


def test_ub_semantics_match_reference():
    """`ub` is the reference's `minimum` argument: the answer is min(ub, OPT)."""
    g = W.gnp(50, 0.12, 42)
    st, opt, _, _ = O.mvc(g)
    for ub in (opt + 5, opt, opt - 1, opt - 3):
        r = vcgpu.solve(g, "mvc", ub=ub, time_limit=TL)
        assert r.status == vcgpu.VC_OK
        assert r.size == min(ub, opt), (ub, opt, r.size)
        if ub >= opt:
            assert r.cover is not None and W.is_cover(g, r.cover) and int(r.cover.sum()) == opt
        else:
            assert r.cover is None


def _golden_batch(max_nodes):
    path = os.path.join(GOLDEN, "batch_seed0.jsonl")
    recs = [json.loads(l) for l in open(path) if l.strip()]
    return sorted([r for r in recs if r["status"] == "ok" and r["nodes"] <= max_nodes], key=lambda r: r["i"])


def test_batch_instances_vs_golden():
    """A slice of the batched workload (G(n, p), n in [30, 200], average degree
    in [3, 12]) in one launch, against the oracle's pinned optima."""
    recs = _golden_batch(2_000_000)[:256]
    graphs = [W.batch_instance(r["i"]) for r in recs]
    st, sols = vcgpu.solve_batch(W.pack(graphs), "mvc", time_limit=TL)
    assert st == vcgpu.VC_OK
    for g, r, rec in zip(graphs, sols, recs):
        _check_mvc(g, r, rec["opt"])


def test_plain_equals_batched():
    recs = _golden_batch(200_000)[:16]
    graphs = [W.batch_instance(r["i"]) for r in recs]
    st, sols = vcgpu.solve_batch(W.pack(graphs), "mvc", time_limit=TL)
    for g, rb, rec in zip(graphs, sols, recs):
        rp = vcgpu.solve(g, "mvc", time_limit=TL)
        assert rp.size == rb.size == rec["opt"]


def test_node_limit_reports_budget():
    recs = [r for r in _golden_batch(10**9) if r["nodes"] > 100_000]
    g = W.batch_instance(recs[0]["i"])
    r = vcgpu.solve(g, "mvc", node_limit=2000, time_limit=TL)
    assert r.status == vcgpu.VC_BUDGET
    assert r.size >= recs[0]["opt"]
    if r.cover is not None:
        assert W.is_cover(g, r.cover) and int(r.cover.sum()) == r.size


def test_invalid_graphs_rejected():
    g = W.gnp(20, 0.2, 1)
    bad = W.Graph(g.n, g.row_ptr.copy(), g.col.copy())
    bad.col[0] = bad.n + 5  # id out of range
    assert vcgpu.solve(bad).status == vcgpu.VC_ERR_INVALID
    loop = W.Graph(3, np.array([0, 1, 2, 2], np.uint32), np.array([0, 0], np.uint32))  # self-loop
    assert vcgpu.solve(loop).status == vcgpu.VC_ERR_INVALID
    asym = W.Graph(3, np.array([0, 1, 1, 1], np.uint32), np.array([1], np.uint32))  # one direction only
    assert vcgpu.solve(asym).status == vcgpu.VC_ERR_INVALID


def test_empty_and_edgeless():
    assert vcgpu.solve(W.from_edges(0, np.zeros((0, 2)))).size == 0
    r = vcgpu.solve(W.from_edges(7, np.zeros((0, 2))), time_limit=TL)
    assert r.status == vcgpu.VC_OK and r.size == 0 and not r.cover.any()
    r = vcgpu.solve(W.from_edges(7, np.zeros((0, 2))), "pvc", k=0, time_limit=TL)
    assert r.decision == 1


def test_config5_chung_lu_plain_and_batched():
    """Chung-Lu n=100000 (gamma 2.1, average degree 8, max degree 2000, seed 7),
    plain, and batched alongside 512 G(100, 0.08) graphs."""
    small = json.load(open(os.path.join(GOLDEN, "small.json")))
    g = W.chung_lu()
    assert (g.n, g.m) == (small["config5"]["n"], small["config5"]["m"])
    opt = small["config5"]["opt"]
    _check_mvc(g, vcgpu.solve(g, "mvc", time_limit=TL), opt)
    side = [(W.gnp(100, 0.08, s), o) for s, o, _ in small["config5_side"]]
    graphs = [g] + [h for h, _ in side]
    st, sols = vcgpu.solve_batch(W.pack(graphs), "mvc", time_limit=TL)
    assert st == vcgpu.VC_OK
    _check_mvc(g, sols[0], opt)
    for (h, o), r in zip(side, sols[1:]):
        _check_mvc(h, r, o)


def test_mixed_size_classes_in_one_batch():
    """Graphs for all three kernel shapes (dense <= 255 vertices, warp CSR units
    up to 2048, CTA units above) in one batched call."""
    rng = np.random.default_rng(77)
    graphs, opts = [], []
    for n in (40, 180, 300, 700, 1500, 2500, 3000):
        g = W.gnp(n, 2.2 / (n - 1), int(rng.integers(1 << 30)))
        st, opt, _, _ = O.mvc(g, node_limit=2_000_000)
        assert st == O.OK
        graphs.append(g)
        opts.append(opt)
    st, sols = vcgpu.solve_batch(W.pack(graphs), "mvc", time_limit=TL)
    assert st == vcgpu.VC_OK
    for g, r, opt in zip(graphs, sols, opts):
        _check_mvc(g, r, opt)
    for g, opt in zip(graphs, opts):  # and the plain entry point on each
        _check_mvc(g, vcgpu.solve(g, "mvc", time_limit=TL), opt)


def test_csr_kernel_on_small_graphs():
    """The CSR search (forced for graphs the dense kernel would take) stays exact."""
    recs = _golden_batch(200_000)[:24]
    graphs = [W.batch_instance(r["i"]) for r in recs]
    vcgpu.debug_stats(2)  # force the CSR kernel
    try:
        st, sols = vcgpu.solve_batch(W.pack(graphs), "mvc", time_limit=TL)
        single = vcgpu.solve(graphs[0], "pvc", k=recs[0]["opt"] - 1, time_limit=TL)
    finally:
        vcgpu.debug_stats(0)
    assert st == vcgpu.VC_OK
    for g, r, rec in zip(graphs, sols, recs):
        _check_mvc(g, r, rec["opt"])
    assert single.status == vcgpu.VC_OK and single.decision == 0


def test_time_limit_returns_timeout_and_device_stays_usable():
    """A launch that reaches its time limit stops every search unit through its
    bounded waits and reports VC_TIMEOUT; the next solve on the device works."""
    recs = [r for r in _golden_batch(10**9) if r["nodes"] > 20_000_000]
    g = W.batch_instance(recs[0]["i"])
    r = vcgpu.solve(g, "mvc", time_limit=0.02)
    assert r.status == vcgpu.VC_TIMEOUT
    assert r.size >= recs[0]["opt"]
    if r.cover is not None:
        assert W.is_cover(g, r.cover) and int(r.cover.sum()) == r.size
    g1 = W.config1_graph()
    small = json.load(open(os.path.join(GOLDEN, "small.json")))
    _check_mvc(g1, vcgpu.solve(g1, "mvc", time_limit=TL), small["config1"]["opt"])


def _wide_graphs():
    """Graphs of 256..640 vertices with small degrees (the wide dense kernel's
    range) with their optima: G(n, p) at average degree 3.2 solved by the
    oracle, and the served stream's pinned pool graphs of that size."""
    rng = np.random.default_rng(4242)
    out = []
    for n in (260, 330, 400, 480, 560, 640):
        g = W.gnp(n, 3.2 / (n - 1), int(rng.integers(1 << 30)))
        st, opt, _, _ = O.mvc(g, node_limit=300_000)
        if st == O.OK:
            out.append((g, opt))
    recs = [json.loads(l) for l in open(os.path.join(GOLDEN, "stream_seed0.jsonl")) if l.strip()]
    for r in sorted(recs, key=lambda r: r["i"]):
        if r["status"] == "ok" and 255 < r["n"] <= 640 and r["nodes"] <= 300_000:
            out.append((W.stream_instance(r["i"]), r["opt"]))
    return out


def test_wide_dense_kernel_batched_and_plain():
    """256..640 vertices with byte degrees run on the 20-word dense kernel,
    batched and one at a time, with the oracle's optima and decisions."""
    items = _wide_graphs()
    assert len(items) >= 8
    graphs = [g for g, _ in items]
    st, sols = vcgpu.solve_batch(W.pack(graphs), "mvc", time_limit=TL)
    assert st == vcgpu.VC_OK
    _, shape = vcgpu.debug_stats()
    assert int(shape[4]) >> 31 == 1 and (int(shape[4]) & 0x7FFFFFFF) == 640, shape  # the wide dense plan ran
    for (g, opt), r in zip(items, sols):
        _check_mvc(g, r, opt)
    for g, opt in items[::3]:
        _check_mvc(g, vcgpu.solve(g, "mvc", time_limit=TL), opt)
        _check_pvc(g, vcgpu.solve(g, "pvc", k=opt - 1, time_limit=TL), opt - 1, 0)
        _check_pvc(g, vcgpu.solve(g, "pvc", k=opt, time_limit=TL), opt, 1)


def _hub_graphs():
    """Graphs of 256..1024 vertices with one to three hubs of degree above 254 on
    a sparse G(n, p) base: the range of the dense kernels with 16-bit degrees,
    with the oracle's optima."""
    rng = np.random.default_rng(2024)
    out = []
    for n, hubs in ((300, 1), (420, 2), (512, 1), (600, 2), (800, 3), (1000, 2), (1024, 1)):
        base = W.gnp(n, 3.0 / (n - 1), int(rng.integers(1 << 30)))
        e = [(u, int(v)) for u in range(n) for v in base.col[base.row_ptr[u]:base.row_ptr[u + 1]] if u < v]
        for h in range(hubs):
            k = min(n - hubs, max(260, int(n * rng.uniform(0.6, 0.9))))
            e += [(h, int(x)) for x in rng.choice(np.arange(hubs, n), k, replace=False)]
        e = list({(min(u, v), max(u, v)) for u, v in e})
        g = W.from_edges(n, np.asarray(e, dtype=np.int64), f"hub{n}x{hubs}")
        assert int(np.diff(g.row_ptr).max()) > 254
        st, opt, _, _ = O.mvc(g, node_limit=2_000_000)
        if st == O.OK:
            out.append((g, opt))
    return out


def test_half_dense_kernels_batched_and_plain():
    """Degrees above a byte (up to 1024 vertices) run on the dense kernels with
    16-bit degrees (16-word rows up to 512 vertices, 32-word rows above),
    batched and one at a time, with the oracle's optima and decisions."""
    items = _hub_graphs()
    assert len(items) >= 6
    graphs = [g for g, _ in items]
    st, sols = vcgpu.solve_batch(W.pack(graphs), "mvc", time_limit=TL)
    assert st == vcgpu.VC_OK
    _, shape = vcgpu.debug_stats()
    assert int(shape[4]) >> 31 == 1 and (int(shape[4]) & 0x7FFFFFFF) == 1024, shape  # the 32-word dense plan ran
    for (g, opt), r in zip(items, sols):
        _check_mvc(g, r, opt)
    for g, opt in items:
        r = vcgpu.solve(g, "mvc", time_limit=TL)
        _, shape = vcgpu.debug_stats()
        assert int(shape[4]) >> 31 == 1 and (int(shape[4]) & 0x7FFFFFFF) == (512 if g.n <= 512 else 1024), shape
        _check_mvc(g, r, opt)
        _check_pvc(g, vcgpu.solve(g, "pvc", k=opt - 1, time_limit=TL), opt - 1, 0)
        _check_pvc(g, vcgpu.solve(g, "pvc", k=opt, time_limit=TL), opt, 1)


def test_half_dense_range_on_the_csr_kernel():
    """The same graphs forced onto the CSR kernel (rows walked by teams of
    lanes where the average degree allows) stay exact."""
    items = _hub_graphs()[:4]
    vcgpu.debug_stats(2)  # force the CSR kernel
    try:
        st, sols = vcgpu.solve_batch(W.pack([g for g, _ in items]), "mvc", time_limit=TL)
        _, shape = vcgpu.debug_stats()
    finally:
        vcgpu.debug_stats(0)
    assert st == vcgpu.VC_OK and int(shape[4]) >> 31 == 0, shape
    for (g, opt), r in zip(items, sols):
        _check_mvc(g, r, opt)


def test_batch_pvc_vs_golden():
    """Batched PVC over 256 graphs of the batched workload, half at k = opt (yes,
    with a cover of at most k) and half at k = opt - 1 (no), in one launch."""
    recs = _golden_batch(2_000_000)[256:512]
    graphs = [W.batch_instance(r["i"]) for r in recs]
    ks = [r["opt"] - (j % 2) for j, r in enumerate(recs)]
    st, sols = vcgpu.solve_batch(W.pack(graphs), "pvc", ks=ks, time_limit=TL)
    assert st == vcgpu.VC_OK
    for g, r, rec, k in zip(graphs, sols, recs, ks):
        _check_pvc(g, r, k, 1 if rec["opt"] <= k else 0)


def test_every_golden_batch_graph_up_to_2m_oracle_nodes():
    """Every graph of the batched workload that the oracle solved within 2 M
    nodes (most of the 4096), in batches of 1024, without a node budget: the
    optimum and a verified cover of that size for each."""
    recs = _golden_batch(2_000_000)
    assert len(recs) > 3000
    for c in range(0, len(recs), 1024):
        chunk = recs[c:c + 1024]
        graphs = [W.batch_instance(r["i"]) for r in chunk]
        st, sols = vcgpu.solve_batch(W.pack(graphs), "mvc", time_limit=TL)
        assert st == vcgpu.VC_OK
        for g, r, rec in zip(graphs, sols, chunk):
            _check_mvc(g, r, rec["opt"])


def test_device_input_entry_points():
    """vc_solve with VC_FLAG_DEVICE_INPUT and vc_solve_batch_device (the CSR
    already in device memory): the same optima as the host entry points, on an
    arena that takes every kernel class (dense, wide dense, warp CSR, CTA CSR)."""
    torch = pytest.importorskip("torch")
    recs = _golden_batch(200_000)[:40]
    graphs = [W.batch_instance(r["i"]) for r in recs]
    opts = [r["opt"] for r in recs]
    wide = _wide_graphs()[:4]
    graphs += [g for g, _ in wide]
    opts += [o for _, o in wide]
    rng = np.random.default_rng(313)
    for n in (900, 1500):
        g = W.gnp(n, 2.2 / (n - 1), int(rng.integers(1 << 30)))
        st, opt, _, _ = O.mvc(g, node_limit=2_000_000)
        assert st == O.OK
        graphs.append(g)
        opts.append(opt)
    arena = W.pack(graphs)
    d_rp = torch.from_numpy(arena.row_ptr.astype(np.int32)).cuda()
    d_col = torch.from_numpy(arena.col.astype(np.int32)).cuda()
    torch.cuda.synchronize()
    st, sols = vcgpu.solve_batch(arena, "mvc", time_limit=TL, d_row_ptr=d_rp.data_ptr(), d_col=d_col.data_ptr())
    assert st == vcgpu.VC_OK
    for g, r, opt in zip(graphs, sols, opts):
        _check_mvc(g, r, opt)
    for j in (0, 40, len(graphs) - 1):  # one graph at a time, device-resident
        g = graphs[j]
        grp = torch.from_numpy(g.row_ptr.astype(np.int32)).cuda()
        gcol = torch.from_numpy(g.col.astype(np.int32)).cuda()
        torch.cuda.synchronize()
        r = vcgpu.solve_device(g.n, g.m, grp.data_ptr(), gcol.data_ptr(), "mvc", time_limit=TL)
        _check_mvc(g, r, opts[j])


def _device_csr(torch, g, mutate=None):
    rp = g.row_ptr.astype(np.int64).copy()
    col = g.col.astype(np.int64).copy()
    if mutate:
        mutate(rp, col)
    return (torch.from_numpy(rp.astype(np.int32)).cuda(), torch.from_numpy(col.astype(np.int32)).cuda())


def test_device_input_layout_checked_on_the_device():
    """Device-resident CSR cannot be validated on the host: a kernel checks the
    layout the search relies on.  A neighbour id out of range, a self loop, a
    decreasing row offset or a row_ptr[n] that disagrees with the stated m is
    reported VC_ERR_INVALID -- for the dense kernel, the CSR kernel and in a batch
    beside a good graph, which still gets its optimum -- and the device stays
    usable."""
    torch = pytest.importorskip("torch")
    g = W.config1_graph()
    opt = json.load(open(os.path.join(GOLDEN, "small.json")))["config1"]["opt"]

    def bad_id(rp, col):
        col[3] = g.n + 7

    def self_loop(rp, col):
        col[rp[5]] = 5

    def decreasing(rp, col):
        rp[10] = rp[12] + 1

    def overlong(rp, col):
        rp[-1] = rp[-1] + 4

    for mutate in (bad_id, self_loop, decreasing, overlong):
        d_rp, d_col = _device_csr(torch, g, mutate)
        torch.cuda.synchronize()
        r = vcgpu.solve_device(g.n, g.m, d_rp.data_ptr(), d_col.data_ptr(), "mvc", time_limit=TL)
        assert r.status == vcgpu.VC_ERR_INVALID, (mutate.__name__, r)
        vcgpu.debug_stats(2)  # the CSR kernel
        try:
            r = vcgpu.solve_device(g.n, g.m, d_rp.data_ptr(), d_col.data_ptr(), "mvc", time_limit=TL)
        finally:
            vcgpu.debug_stats(0)
        assert r.status == vcgpu.VC_ERR_INVALID, (mutate.__name__, r)
    # a batch on the device: graph 1 broken on the device only, graph 0 and 2 good
    graphs = [g, g, g]
    arena = W.pack(graphs)
    rp = arena.row_ptr.astype(np.int64).copy()
    col = arena.col.astype(np.int64).copy()
    col[int(arena.col_off[1]) + 2] = g.n + 1
    d_rp = torch.from_numpy(rp.astype(np.int32)).cuda()
    d_col = torch.from_numpy(col.astype(np.int32)).cuda()
    torch.cuda.synchronize()
    st, sols = vcgpu.solve_batch(arena, "mvc", time_limit=TL, d_row_ptr=d_rp.data_ptr(), d_col=d_col.data_ptr())
    assert sols[1].status == vcgpu.VC_ERR_INVALID
    _check_mvc(g, sols[0], opt)
    _check_mvc(g, sols[2], opt)
    _check_mvc(g, vcgpu.solve(g, "mvc", time_limit=TL), opt)


def test_lane_search_units_match_golden():
    """The opt-in lane kernel (one thread per search unit) returns the oracle's
    optimum with a verified cover on golden batch graphs, MVC and PVC, batched
    and plain."""
    recs = _golden_batch(300_000)[:160]
    graphs = [W.batch_instance(r["i"]) for r in recs]
    vcgpu.debug_stats(4)
    try:
        st, sols = vcgpu.solve_batch(W.pack(graphs), "mvc", time_limit=TL)
        ks = [r["opt"] - (i % 2) for i, r in enumerate(recs[:40])]
        stp, pv = vcgpu.solve_batch(W.pack(graphs[:40]), "pvc", ks=ks, time_limit=TL)
        single = [vcgpu.solve(graphs[j], "mvc", time_limit=TL) for j in (0, 1, 2)]
        shape = vcgpu.debug_stats()[1]
    finally:
        vcgpu.debug_stats(0)
    assert int(shape[1]) != 256  # the lane kernel's CTA shape, not the dense kernel's
    for g, r, rec in zip(graphs, sols, recs):
        _check_mvc(g, r, rec["opt"])
    for g, r, rec, k in zip(graphs, pv, recs, ks):
        _check_pvc(g, r, k, 1 if rec["opt"] <= k else 0)
    for j, r in zip((0, 1, 2), single):
        _check_mvc(graphs[j], r, recs[j]["opt"])
