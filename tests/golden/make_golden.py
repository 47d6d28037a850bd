"""Generates the golden fixtures under tests/golden/ with the CPU oracle.

Every graph is regenerated from its seed by vcgpu.workloads, so a fixture holds
only the answers: the optimum cover size (MVC) from the oracle's restatement of
the reference's Sequential(), the oracle's tree-node count, and a status
("ok", or "budget" when the oracle stopped at its node limit -- such instances
carry no answer and are left out of parity claims).

    python tests/golden/make_golden.py small      # config 1/2 + exhaustive n<=7
    python tests/golden/make_golden.py batch [--count 4096] [--limit 100000000] [--workers 6]
    python tests/golden/make_golden.py batch-hard [--workers 6]   # the "budget" ones, no limit
    python tests/golden/make_golden.py stream [--count 2000] [--limit 20000000]
    python tests/golden/make_golden.py files      # reference known-answer graph files
    python tests/golden/make_golden.py mcm        # the MCM mode's answers (needs networkx)

Output files are JSON (lines for the long runs, so partial runs are usable).
Workers are started with the `spawn` method.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "parallel-vertex-cover-algorithms-on-gpus_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))


def _batch_job(args):
    i, seed, limit = args
    from vcgpu import workloads as W
    import oracle as O
    g = W.batch_instance(i, seed)
    t = time.time()
    st, size, cover, nodes = O.mvc(g, node_limit=limit)
    return {"i": i, "n": g.n, "m": g.m, "opt": size if st == O.OK else None,
            "ub": size, "nodes": nodes, "status": "ok" if st == O.OK else "budget",
            "cpu_s": round(time.time() - t, 4)}


def _hard_job(args):
    """A batch graph the budgeted run left open, solved without a node limit.
    The search starts from the oracle's own best cover of that run (size `ub`):
    the restatement returns min(ub, OPT), and OPT <= ub because that cover
    exists, so the result is OPT and depends on nothing but the oracle."""
    i, seed, ub = args
    from vcgpu import workloads as W
    import oracle as O
    g = W.batch_instance(i, seed)
    t = time.time()
    st, size, cover, nodes = O.mvc(g, ub=ub, node_limit=0)
    return {"i": i, "n": g.n, "m": g.m, "opt": size if st == O.OK else None, "ub_start": ub,
            "nodes": nodes, "status": "ok" if st == O.OK else "error", "cpu_s": round(time.time() - t, 4)}


def _stream_job(args):
    i, seed, limit = args
    from vcgpu import workloads as W
    import oracle as O
    g = W.stream_instance(i, seed)
    t = time.time()
    st, size, cover, nodes = O.mvc(g, node_limit=limit)
    return {"i": i, "name": g.name, "n": g.n, "m": g.m, "opt": size if st == O.OK else None,
            "nodes": nodes, "status": "ok" if st == O.OK else "budget", "cpu_s": round(time.time() - t, 4)}


def _run_pool(job, items, out_path, workers):
    done = set()
    if os.path.exists(out_path):
        with open(out_path) as f:
            for line in f:
                if line.strip():
                    done.add(json.loads(line)["i"])
    todo = [it for it in items if it[0] not in done]
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool, open(out_path, "a") as f:
        for rec in pool.imap_unordered(job, todo, chunksize=1):
            f.write(json.dumps(rec) + "\n")
            f.flush()


def small():
    from vcgpu import workloads as W
    import oracle as O
    import itertools
    import numpy as np
    out = {}
    g1 = W.config1_graph()
    st, opt1, _, nodes1 = O.mvc(g1)
    out["config1"] = {"n": g1.n, "m": g1.m, "opt": opt1, "nodes": nodes1}
    g2 = W.config2_graph()
    st, opt2, _, nodes2 = O.mvc(g2)
    out["config2"] = {"n": g2.n, "m": g2.m, "opt": opt2, "nodes": nodes2,
                      "pvc_k_opt": O.pvc(g2, opt2)[1], "pvc_k_opt_minus_1": O.pvc(g2, opt2 - 1)[1]}
    g5 = W.chung_lu()
    ub5, _ = O.greedy_ub(g5)
    st, opt5, _, nodes5 = O.mvc(g5, ub=ub5 + 1)
    out["config5"] = {"n": g5.n, "m": g5.m, "opt": opt5, "nodes": nodes5}
    side = []
    for i in range(512):
        gs = W.gnp(100, 0.08, 10_000 + i)
        st, o, _, nd = O.mvc(gs, node_limit=5_000_000)
        side.append([10_000 + i, o if st == O.OK else None, nd])
    out["config5_side"] = side
    # every graph on up to 6 vertices is enumerable; keep a seeded sample of 7-vertex ones
    rng = np.random.default_rng(0)
    small_cases = []
    for n in range(1, 8):
        pairs = list(itertools.combinations(range(n), 2))
        masks = range(1 << len(pairs)) if n <= 5 else rng.integers(0, 1 << len(pairs), size=300).tolist()
        for mask in masks:
            e = [pairs[j] for j in range(len(pairs)) if (mask >> j) & 1]
            g = W.from_edges(n, np.asarray(e, dtype=np.int64).reshape(-1, 2))
            st, opt, _, _ = O.mvc(g)
            small_cases.append([n, int(mask), opt])
    out["exhaustive"] = small_cases
    with open(os.path.join(HERE, "small.json"), "w") as f:
        json.dump(out, f)
    print("config1", out["config1"], "config2", out["config2"], "config5", out["config5"],
          "side solved", sum(1 for x in side if x[1] is not None), "exhaustive", len(small_cases))


def files():
    """Known answers from the reference's own test/runGraphs.py:8-30, checked by
    running the reference's Sequential on each tractable 1-based file."""
    import oracle as O
    import re
    ref_root = O.REFERENCE_ROOT
    src = open(os.path.join(ref_root, "test", "runGraphs.py")).read()
    body = src[src.index("MVCS = {"):src.index("}", src.index("MVCS = {"))]
    golden = {k: int(v) for k, v in re.findall(r'"([^"]+)"\s*:\s*(\d+)', body)}
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump({"source": "test/runGraphs.py:8-30", "mvc": golden}, f, indent=1)
    print(golden)


def _mcm_graph(spec):
    from vcgpu import workloads as W
    if spec["family"] == "gnp":
        return W.gnp(spec["n"], spec["d"] / (spec["n"] - 1), spec["seed"])
    return W.planted_matching(spec["n"], spec["d"], spec["seed"])


def mcm():
    """Answers of the MCM mode (the search of the reference's default build):
    2 * maximum matching + isolated vertices, from networkx's maximum-cardinality
    matching.  The search is exhaustive (exponential in the edges), so the
    graphs are the ones it can finish: G(n, p) graphs on which the oracle's
    restatement (no cut at all) finishes within 3e7 tree nodes and agrees, and
    planted-matching graphs of up to 1024 vertices whose maximum matching is the
    first one the in-order search meets (odd n: one vertex unmatched, which the
    search's bound then proves at once)."""
    import networkx as nx
    import oracle as O
    specs = [{"family": "gnp", "n": n, "d": d, "seed": 700 + i}
             for i, (n, d) in enumerate([(6, 2.0), (8, 1.5), (9, 3.0), (10, 2.5), (11, 4.0), (12, 1.2), (13, 3.0),
                                          (14, 2.0), (15, 5.0), (16, 2.5), (17, 3.5), (18, 1.8), (18, 4.0),
                                          (22, 2.5), (26, 3.0), (30, 2.0), (34, 3.5), (40, 2.5), (48, 3.0)])]
    specs += [{"family": "planted", "n": n, "d": 6.0, "seed": 800 + i}
              for i, n in enumerate([64, 101, 256, 511, 640, 1023, 1024])]
    out = []
    for sp in specs:
        g = _mcm_graph(sp)
        G = nx.Graph()
        G.add_nodes_from(range(g.n))
        for u in range(g.n):
            for v in g.col[g.row_ptr[u]:g.row_ptr[u + 1]]:
                if u < v:
                    G.add_edge(u, int(v))
        nu = len(nx.max_weight_matching(G, maxcardinality=True))
        iso = sum(1 for v in range(g.n) if G.degree(v) == 0)
        rec = dict(sp, m=g.m, matching=nu, isolated=iso, expect=2 * nu + iso)
        if sp["family"] == "gnp":
            st, best, nodes = O.mcm(g, node_limit=30_000_000)
            if st != O.OK:
                continue
            assert best == rec["expect"], (sp, best, rec["expect"])
            rec["oracle_nodes"] = nodes
        out.append(rec)
    with open(os.path.join(HERE, "mcm.json"), "w") as f:
        json.dump(out, f, indent=0)
    print(len(out), [(r["family"], r["n"], r["expect"], r.get("oracle_nodes")) for r in out])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["small", "batch", "batch-hard", "stream", "files", "mcm"])
    ap.add_argument("--count", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--limit", type=int, default=100_000_000)
    ap.add_argument("--workers", type=int, default=max(1, (os.cpu_count() or 2) - 2))
    a = ap.parse_args()
    if a.what == "small":
        small()
    elif a.what == "files":
        files()
    elif a.what == "mcm":
        mcm()
    elif a.what == "batch":
        _run_pool(_batch_job, [(i, a.seed, a.limit) for i in range(a.count)],
                  os.path.join(HERE, f"batch_seed{a.seed}.jsonl"), a.workers)
    elif a.what == "batch-hard":
        recs = [json.loads(l) for l in open(os.path.join(HERE, f"batch_seed{a.seed}.jsonl")) if l.strip()]
        open_recs = sorted((r for r in recs if r["status"] != "ok"), key=lambda r: -r["n"] * r["m"])
        _run_pool(_hard_job, [(r["i"], a.seed, r["ub"]) for r in open_recs],
                  os.path.join(HERE, f"batch_seed{a.seed}_hard.jsonl"), a.workers)
    else:
        _run_pool(_stream_job, [(i, a.seed, a.limit) for i in range(a.count)],
                  os.path.join(HERE, f"stream_seed{a.seed}.jsonl"), a.workers)


if __name__ == "__main__":
    main()
