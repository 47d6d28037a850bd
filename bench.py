#!/usr/bin/env python
"""Benchmark: batched exact MVC on one B200 (or N, one process per GPU).

Workload (one "step"): the batched configuration -- 4096 independent G(n, p)
graphs, n ~ U{30..200}, average degree ~ U[3, 12], each with its own seed --
solved in ONE persistent launch of the library's batched entry point, with a
per-graph search-tree node budget (default 2^22 nodes).  The metric counts the
graphs solved to a proven optimum per second; graphs that reach the budget are
reported separately and not counted.  Also reported: tree-nodes/s, the p50/p99
completion latency of graphs inside the batch, and the same graphs solved one
graph per launch ("plain") on a sample, for the batched-vs-plain ratio.

  value : graphs solved / s with the arena resident in HBM (device pointers),
          timed with CUDA events on the launching stream, L2 flushed between steps
  e2e   : the same through vc_solve_batch with pinned host buffers (H2D of the
          arena and D2H of results inside the timed region), wall clock
  roofline: the search kernel's algorithmic bytes (4*(3n+2m+1) per tree node)
          per launch / its event-timed duration, against the measured HBM copy
          bandwidth
  cpu_baseline: the reference's own CPU solver (oracle/_ref/ref_bench) on a
          bounded sample of the same graphs, all host cores

`--impl reference` runs only the reference's CPU solver over bounded samples of
the same workload (rank 0 only under torchrun).

`--workload stream` measures the served configuration instead: Poisson arrivals
(default 2000 requests/s for 60 s), 70% MVC / 30% PVC with k = opt or opt-1,
graphs drawn from the oracle-pinned pool of the stream family (G(n, p) and
random 3-regular, n log-uniform in [50, 5000]; tests/golden/stream_seed0.jsonl),
submitted to a vc_server as they arrive; it reports completed requests/s,
p50/p99 latency from submission to completion, and checks every answer.  Multi-GPU: every rank solves
its own batch (seed = rank): weak scaling, no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "parallel-vertex-cover-algorithms-on-gpus_b200")
sys.path.insert(0, PKG)

from vcgpu import workloads as W  # noqa: E402

METRIC = "instances/s and tree-nodes/s at exact optimum; p50/p99 latency, batched vs plain"
REF_BENCH = os.path.join(REPO, "oracle", "_ref", "ref_bench")
REF_NODE_RATE = 350e3  # the reference CPU solver's tree nodes/s on these graphs (one core)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--count", type=int, default=4096)
    ap.add_argument("--node-limit", type=int, default=1 << 22)
    ap.add_argument("--plain-sample", type=int, default=128)
    ap.add_argument("--cpu-sample-s", type=float, default=20.0)
    ap.add_argument("--ref-step-s", type=float, default=30.0)
    ap.add_argument("--workload", default="batch", choices=["batch", "stream", "ub"])
    ap.add_argument("--rate", type=float, default=2000.0)
    ap.add_argument("--stream-seconds", type=float, default=60.0)
    ap.add_argument("--stream-max-vertices", type=int, default=0)
    ap.add_argument("--stream-min-vertices", type=int, default=0)
    return ap.parse_args()


def algorithmic_bytes_per_node(n: int, m: int) -> int:
    """Read the parent degree array, write one child degree array, read the
    CSR offsets and adjacency once: 4 * (3n + 2m + 1) bytes."""
    return 4 * (3 * n + 2 * m + 1)


def write_graph_file(graphs, path, mode=0, ks=None):
    with open(path, "wb") as f:
        np.asarray([len(graphs)], np.uint32).tofile(f)
        for i, g in enumerate(graphs):
            np.asarray([g.n, g.col.shape[0], mode, 0 if ks is None else ks[i]], np.uint32).tofile(f)
            g.row_ptr.astype(np.uint32).tofile(f)
            g.col.astype(np.uint32).tofile(f)


def run_ref_bench(graphs, threads, per_graph_s, total_s):
    """The reference's CPU solver over `graphs` (fork per graph, all cores)."""
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "graphs.bin")
        write_graph_file(graphs, path)
        t0 = time.perf_counter()
        out = subprocess.run([REF_BENCH, path, str(threads), str(per_graph_s), str(total_s)],
                             capture_output=True, text=True, check=True).stdout
        wall = time.perf_counter() - t0
    rows = [l.split() for l in out.splitlines() if l.strip()]
    solved = sum(1 for r in rows if r[1] == "ok")
    return solved, len(rows), wall


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = max(mx, float(parts[1]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[3:7]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def search_kernel_traffic():
    """DRAM bytes per launch of the search kernel from the committed ncu summary."""
    path = os.path.join(REPO, "profiles", "search_kernel_traffic.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return d.get("dram_bytes_per_launch")
    return None


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1 and args.impl == "ours":
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def reference_arm(args, world, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    if not os.path.exists(REF_BENCH):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_bench was not built (no reference tree)"}))
        return
    graphs = W.batch_graphs(min(args.count, 512), seed=0)
    per_graph_s = args.node_limit / REF_NODE_RATE
    times, solved_l, tried_l = [], [], []
    for step in range(args.warmup + args.steps):
        solved, tried, wall = run_ref_bench(graphs, threads, per_graph_s, args.ref_step_s)
        if step >= args.warmup:
            times.append(wall)
            solved_l.append(solved)
            tried_l.append(tried)
    value = sum(solved_l) / sum(times)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "instances/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": "batched MVC, G(n,p) n~U{30..200} avg deg~U[3,12] (bounded sample, graphs in index order)",
                       "per_graph_limit_s": per_graph_s, "step_limit_s": args.ref_step_s,
                       "graphs_started_per_step": float(np.mean(tried_l)), "graphs_solved_per_step": float(np.mean(solved_l))},
            "cpu_baseline": {"value": value, "unit": "instances/s", "cores": threads, "kind": "reference",
                             "sample": f"graphs 0.. of the batch, {args.ref_step_s:.0f} s per step, per-graph limit {per_graph_s:.1f} s"},
            "e2e": {"value": value, "unit": "instances/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def our_arm(args, world, rank, local, pg):
    import torch
    import vcgpu
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    graphs = W.rank_batch(args.count, rank)
    arena = W.pack(graphs)
    n_arr = np.asarray([g.n for g in graphs], np.int64)
    m_arr = np.asarray([g.m for g in graphs], np.int64)
    bnode = 4 * (3 * n_arr + 2 * m_arr + 1)
    d_rp = torch.from_numpy(arena.row_ptr.astype(np.int32)).to(dev)
    d_col = torch.from_numpy(arena.col.astype(np.int32)).to(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def device_step():
        return vcgpu.solve_batch(arena, "mvc", node_limit=args.node_limit, want_cover=True, device=local,
                                 d_row_ptr=d_rp.data_ptr(), d_col=d_col.data_ptr(), validate=False,
                                 stream=stream.cuda_stream)

    def barrier():
        if pg is not None:
            pg.barrier()

    for _ in range(args.warmup):
        device_step()
    times, sols_last = [], None
    launches0 = vcgpu.kernel_launches()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1)  # L2 flush: the arena (~22 MB) is smaller than L2
            torch.cuda.synchronize()
            barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st, sols = device_step()
            e1.record(stream)
            torch.cuda.synchronize()
            barrier()
            times.append(e0.elapsed_time(e1) / 1e3)
            sols_last = sols
    launches = (vcgpu.kernel_launches() - launches0) // max(args.steps, 1)
    _, shape = vcgpu.debug_stats()
    launch_shape = {"grid": int(shape[0]), "block": int(shape[1]), "smem_bytes": int(shape[2]),
                    "search_units": int(shape[3]), "dense": bool(int(shape[4]) >> 31)}
    step_s = float(np.mean(times))
    solved = sum(1 for s in sols_last if s.status == vcgpu.VC_OK)
    budget = sum(1 for s in sols_last if s.status == vcgpu.VC_BUDGET)
    nodes = sum(s.tree_nodes for s in sols_last)
    kernel_s = sols_last[0].kernel_ms / 1e3
    done = np.asarray([s.done_ms for s in sols_last if s.status == vcgpu.VC_OK])
    alg_bytes = float(sum(int(s.tree_nodes) * int(b) for s, b in zip(sols_last, bnode)))

    # e2e: host buffers (pinned) through the public batched entry point
    pinned = {}
    for name in ("n", "row_off", "col_off", "row_ptr", "col"):
        a = getattr(arena, name)
        t = torch.empty(a.shape, dtype={np.uint32: torch.int32, np.uint64: torch.int64}[a.dtype.type]).pin_memory()
        t.numpy().view(a.dtype)[:] = a
        pinned[name] = t
    host_arena = W.Arena(*(pinned[k].numpy().view(getattr(arena, k).dtype)
                           for k in ("n", "row_off", "col_off", "row_ptr", "col")))
    h2d = int(arena.row_ptr.nbytes + arena.col.nbytes + 48 * arena.count)
    d2h = int(40 * arena.count + 4 * sum((g.n + 31) // 32 for g in graphs))
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    st_e, sols_e = vcgpu.solve_batch(host_arena, "mvc", node_limit=args.node_limit, want_cover=True, device=local,
                                     validate=True)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    barrier()
    solved_e = sum(1 for s in sols_e if s.status == vcgpu.VC_OK)

    # max over ranks of the step time, sum of solved graphs
    if pg is not None:
        tt = torch.tensor([step_s, e2e_s], device=dev)
        pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        cc = torch.tensor([solved, solved_e, nodes, budget], device=dev, dtype=torch.float64)
        pg.all_reduce(cc)
        step_s, e2e_s = float(tt[0]), float(tt[1])
        solved_all, solved_e_all, nodes_all, budget_all = (float(x) for x in cc)
    else:
        solved_all, solved_e_all, nodes_all, budget_all = solved, solved_e, nodes, budget
    if rank != 0:
        return

    # plain: one graph per launch on a sample of the same graphs
    sample = graphs[:args.plain_sample]
    t0 = time.perf_counter()
    plain_solved = 0
    for g in sample:
        r = vcgpu.solve(g, "mvc", node_limit=args.node_limit, device=local, validate=False)
        plain_solved += r.status == vcgpu.VC_OK
    plain_s = time.perf_counter() - t0
    batch_sample_s = max((s.done_ms for s in sols_last[:args.plain_sample]), default=0.0) / 1e3

    # CPU baseline: the reference's own solver on a bounded sample, all cores
    cpu = None
    if os.path.exists(REF_BENCH):
        threads = os.cpu_count() or 1
        per_graph_s = args.node_limit / REF_NODE_RATE
        c_solved, c_tried, c_wall = run_ref_bench(graphs[:256], threads, per_graph_s, args.cpu_sample_s)
        cpu = {"value": c_solved / c_wall, "unit": "instances/s", "cores": threads, "kind": "reference",
               "sample": f"graphs 0..{c_tried - 1} of the batch in {c_wall:.1f} s, per-graph limit {per_graph_s:.1f} s "
                         f"(the node budget at the reference's node rate); {c_solved} solved"}

    hbm, src = measured_peaks()
    achieved = alg_bytes / kernel_s / 1e9
    line = {
        "metric": METRIC, "value": solved_all / step_s, "unit": "instances/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * step_s, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {
            "workload": f"batched MVC: {args.count} G(n,p) graphs per GPU, n~U{{30..200}}, avg degree~U[3,12], "
                        f"seed per graph; node budget {args.node_limit} per graph",
            "graphs_per_gpu": args.count, "node_limit": args.node_limit, "solved": int(solved_all),
            "budget_exceeded": int(budget_all), "tree_nodes_per_s": nodes_all / step_s,
            "p50_latency_ms": float(np.percentile(done, 50)) if done.size else None,
            "p99_latency_ms": float(np.percentile(done, 99)) if done.size else None,
            "plain_instances_per_s": plain_solved / plain_s if plain_s > 0 else None,
            "plain_sample": len(sample), "plain_sample_s": plain_s, "batched_sample_done_s": batch_sample_s,
            "batched_over_plain": (solved / step_s) / (plain_solved / plain_s) if plain_solved else None,
            "l2": "flushed before every timed step (256 MB write); arena ~%.0f MB" % ((arena.row_ptr.nbytes + arena.col.nbytes) / 1e6),
            "parallelism": f"{world} GPU(s), graphs sharded by rank, no collective on the data path",
            "launch": launch_shape,
        },
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": search_kernel_traffic(), "peak_source": src,
                     "note": "algorithmic bytes 4*(3n+2m+1) per tree node over the search kernel's event-timed duration"},
        "cpu_baseline": cpu,
        "e2e": {"value": solved_e_all / e2e_s, "unit": "instances/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    print(json.dumps(line))


def stream_arm(args, world, rank):
    """The served stream through vc_server (rank 0; other ranks have no work)."""
    if rank != 0:
        return
    import vcgpu
    recs = [json.loads(l) for l in open(os.path.join(REPO, "tests", "golden", "stream_seed0.jsonl")) if l.strip()]
    pinned = sorted([r for r in recs if r["status"] == "ok" and r["n"] >= args.stream_min_vertices and
                     (not args.stream_max_vertices or r["n"] <= args.stream_max_vertices)], key=lambda r: r["i"])
    pool = [(W.stream_instance(r["i"]), r["opt"]) for r in pinned]
    rng = np.random.default_rng(1)
    arrivals, t = [], 0.0
    while True:
        t += float(rng.exponential(1.0 / args.rate))
        if t > args.stream_seconds:
            break
        arrivals.append(t)
    reqs = []
    for a in arrivals:
        g, opt = pool[int(rng.integers(len(pool)))]
        if rng.random() < 0.7:
            reqs.append((a, g, "mvc", 0, opt))
        else:
            reqs.append((a, g, "pvc", opt - int(rng.integers(0, 2)), opt))
    max_n = max(g.n for g, _ in pool)
    lat, bad, budget, done = [], 0, 0, 0
    lane_lat = {}
    with vcgpu.Server(max_vertices=max_n, max_requests=4096, mem_budget=2 << 30) as srv:
        lanes = srv.shape()
        for g, opt in pool[:32]:  # warm-up: kernel launch, first-touch of buffers
            srv.wait(srv.submit(g, "mvc", node_limit=args.node_limit))
        outstanding = {}
        t0 = time.perf_counter()
        i = 0
        while i < len(reqs) or outstanding:
            now = time.perf_counter() - t0
            while i < len(reqs) and reqs[i][0] <= now:
                a, g, kind, k, opt = reqs[i]
                outstanding[srv.submit(g, kind, k=k, node_limit=args.node_limit, validate=False)] = (g, kind, k, opt)
                i += 1
            for tk in srv.completed():
                r = srv.poll(tk, want_cover=False)
                g, kind, k, opt = outstanding.pop(tk)
                done += 1
                lat.append(r.total_ms)
                lane_lat.setdefault(vcgpu.Server.lane(tk), []).append(r.total_ms)
                if r.status == vcgpu.VC_BUDGET:
                    budget += 1
                elif r.status != vcgpu.VC_OK:
                    bad += 1
                elif kind == "mvc" and r.size != opt:
                    bad += 1
                elif kind == "pvc" and r.decision != (1 if opt <= k else 0):
                    bad += 1
            nxt = reqs[i][0] - (time.perf_counter() - t0) if i < len(reqs) else 0.0005
            time.sleep(max(0.0, min(nxt, 0.0005)))
        wall = time.perf_counter() - t0
    lat = np.asarray(lat)
    for li, x in sorted(lane_lat.items()):
        if li < len(lanes):
            lanes[li].update({"requests": len(x), "p50_latency_ms": float(np.percentile(x, 50)),
                              "p99_latency_ms": float(np.percentile(x, 99))})
    line = {"metric": METRIC, "value": done / wall, "unit": "requests/s", "n_gpus": 1, "steps": 1, "warmup": 1,
            "ms_per_step": 1e3 * wall, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int32", "data": "synthetic",
            "config": {"workload": f"served stream: Poisson {args.rate:.0f} req/s for {args.stream_seconds:.0f} s, "
                                   "70% MVC / 30% PVC (k = opt or opt-1), G(n,p) and random 3-regular, "
                                   "n log-uniform [50,5000], drawn from the oracle-pinned pool",
                       "requests": len(reqs), "completed": done, "wrong": bad, "budget_exceeded": budget,
                       "node_limit": args.node_limit, "pool": len(pool), "pool_coverage": len(pinned) / max(len(recs), 1),
                       "p50_latency_ms": float(np.percentile(lat, 50)), "p99_latency_ms": float(np.percentile(lat, 99)),
                       "mean_latency_ms": float(lat.mean()), "max_vertices": max_n, "lanes": lanes}}
    print(json.dumps(line))


def ub_arm(args, world, rank):
    """The reference's upper-bound heuristics on the GPU (vc_remove_max_ub /
    vc_remove_edge_ub): Chung-Lu n=100000 (one graph) and the 4096 batched
    graphs, beside the reference's own CPU functions on the Chung-Lu graph
    (forked child, one core).  rand() value 12345 for RemoveEdge."""
    if rank != 0:
        return
    import vcgpu
    g5 = W.chung_lu()
    arena = W.pack(W.batch_graphs(args.count, seed=0))
    r = 12345
    out = {}
    for name, fn in (("remove_max", lambda a: vcgpu.remove_max_ub(a)), ("remove_edge", lambda a: vcgpu.remove_edge_ub(a, r))):
        fn(g5)  # warm-up
        t0 = time.perf_counter()
        ubs, _, kms = fn(g5)
        call_ms = 1e3 * (time.perf_counter() - t0)
        _, _, bms = fn(arena)
        out[name] = {"config5_bound": ubs[0], "config5_kernel_ms": kms, "config5_call_ms": call_ms,
                     "batch_kernel_ms": bms}
    cpu = {}
    if os.path.exists(os.path.join(REPO, "oracle", "_ref", "libvcref.so")):
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import oracle as O
        for name, fn in (("remove_max", O.ref_remove_max_ub_forked), ("remove_edge", O.ref_remove_edge_ub_forked)):
            t0 = time.perf_counter()
            fn(g5)
            cpu[name + "_config5_s"] = time.perf_counter() - t0
    line = {"metric": "upper-bound heuristics time (config 5, Chung-Lu n=100000)",
            "value": out["remove_edge"]["config5_call_ms"], "unit": "ms", "n_gpus": 1, "steps": 1, "warmup": 1,
            "ms_per_step": out["remove_edge"]["config5_call_ms"], "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": "RemoveMax / RemoveEdge upper bounds: Chung-Lu n=100000 (gamma 2.1, avg degree 8, "
                                   f"max degree 2000, seed 7) and {args.count} batched G(n,p) graphs", **out,
                       "reference_cpu": cpu}}
    print(json.dumps(line))


def main():
    args = parse()
    world, rank, local, pg = dist_setup(args)
    try:
        if args.impl == "reference":
            reference_arm(args, world, rank)
        elif args.workload == "stream":
            stream_arm(args, world, rank)
        elif args.workload == "ub":
            ub_arm(args, world, rank)
        else:
            our_arm(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
