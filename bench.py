#!/usr/bin/env python
"""Benchmark: batched exact MVC on one B200 (or N, one process per GPU).

Workload (one "step"): the batched configuration -- G(n, p) graphs, n ~ U{30..200},
average degree ~ U[3, 12], seed per graph -- restricted to the 3958 of its 4096
graphs whose optimum the CPU oracle pinned within 10^8 tree nodes
(tests/golden/batch_seed0.jsonl, status "ok"), solved to a PROVEN OPTIMUM with
no node budget in ONE persistent launch of the library's batched entry point.
Every answer of every step is checked against the pinned optimum.  The other
138 graphs need 0.4-1.1 G tree nodes each (37 G together, 3x the whole pinned
set); `--set full` runs all 4096.

  value : graphs solved / s with the arena resident in HBM (device pointers),
          device time of the launch (CUDA events on the launching stream), L2
          flushed before each step; max over ranks for N > 1
  e2e   : the same through vc_solve_batch with pinned host buffers (H2D of the
          arena and D2H of results inside the timed region), wall clock
  roofline: the search kernel's algorithmic bytes (4*(3n+2m+1) per tree node) per
          launch / its event-timed duration against the measured HBM copy
          bandwidth, and the issue roofline that binds it: measured warp
          instructions per tree node x node rate / (SMs x 4 schedulers x clock)
  cpu_baseline: the reference's own CPU solver (oracle/_ref/ref_bench, all host
          cores) on a like-for-like sample, with the GPU's figure on the same
          sample beside it
  config.plain_vs_batched: the same sample of the pinned set solved one graph per
          call and in one batched call
  config.reference_cuda: the reference's own CUDA program (oracle/_ref/cuda/output,
          built for sm_100a by oracle/Makefile), one process per graph
  config.reference_files: the same program and vc_solve on six of the
          reference's own graph files (--ref-files), answers checked against
          its known optima
  config.served: a short served stream through vc_server

`--impl reference` runs only the reference's CPU solver over the CPU sample
(rank 0 only under torchrun).  `--workload stream` runs the served configuration
alone for longer; `--workload ub` the upper-bound heuristics; `--workload files`
the reference's own graph files (staged by `make -C oracle graphs`) through
vc_solve beside the reference's own CUDA program on the same files; `--workload
mcm` the MCM mode (vc_mcm) beside the reference's default `VC 0` build on the
graphs of tests/golden/mcm.json; `--workload
profile` is the torch-free case for profiler captures: the first --count graphs
of the step's set in one vc_solve_batch call, --reps times.

Multi-GPU: `--gpus N` starts N ranks under torch.distributed.run when it is not
already running under it.  The pinned set is split across the ranks by
estimated work (n * m, longest first onto the least-loaded rank); there is no
collective on the data path, only the timing and count reductions.  Scaling is
strong (the set is fixed).
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
GOLDEN = os.path.join(REPO, "tests", "golden")
REF_BENCH = os.path.join(REPO, "oracle", "_ref", "ref_bench")
REF_CUDA = os.path.join(REPO, "oracle", "_ref", "cuda", "output")
ISSUE_PROFILE = os.path.join(REPO, "profiles", "k_dense_issue.json")
TRAFFIC_PROFILE = os.path.join(REPO, "profiles", "search_kernel_traffic.json")
CPU_EASY_S = 0.5  # CPU sample: pinned graphs the oracle solved within this many CPU seconds


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batch", choices=["batch", "stream", "ub", "profile", "files", "mcm"])
    ap.add_argument("--files", default="",
                    help="--workload files: comma-separated reference graph files (default: the 1-based ones)")
    ap.add_argument("--file-time-limit", type=float, default=30.0,
                    help="--workload files: seconds per solve, for this library and the reference's program alike")
    ap.add_argument("--count", type=int, default=128)
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--case", default="batch", choices=["batch", "csr-batch", "powergrid", "file"])
    ap.add_argument("--file", default="Power-Grid.txt",
                    help="--case file: one of the reference's graph files staged by `make -C oracle graphs`")
    ap.add_argument("--set", default="pinned", choices=["pinned", "full"])
    ap.add_argument("--time-limit", type=float, default=600.0)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--plain-every", type=int, default=16)
    ap.add_argument("--cpu-sample-s", type=float, default=20.0)
    ap.add_argument("--ref-step-s", type=float, default=15.0)
    ap.add_argument("--refcuda-graphs", type=int, default=16)
    ap.add_argument("--ref-files", default="cop_hat300-1.txt,cop_hat500-1.txt,cop_hat500-2.txt,cop_hat700-1.txt,"
                                           "cop_hat1000-1.txt,Power-Grid.txt",
                    help="reference graph files compared with the reference's CUDA program in the default run "
                         "('' to skip)")
    ap.add_argument("--served-seconds", type=float, default=10.0)
    ap.add_argument("--rate", type=float, default=2000.0)
    ap.add_argument("--stream-seconds", type=float, default=60.0)
    ap.add_argument("--stream-max-vertices", type=int, default=0)
    ap.add_argument("--stream-min-vertices", type=int, default=0)
    ap.add_argument("--node-limit", type=int, default=0)
    return ap.parse_args(argv)


# ---------------------------------------------------------------- workload

def golden_batch():
    """The oracle's records of the batched workload, by graph index."""
    recs = {}
    for name in ("batch_seed0.jsonl", "batch_seed0_hard.jsonl"):
        path = os.path.join(GOLDEN, name)
        if not os.path.exists(path):
            continue
        for line in open(path):
            if line.strip():
                r = json.loads(line)
                if name.endswith("_hard.jsonl") and r.get("status") != "ok":
                    continue
                recs[r["i"]] = r if r["i"] not in recs or r.get("status") == "ok" else recs[r["i"]]
    return recs


def pinned_indices(which: str = "pinned"):
    """The step's graphs: 'pinned' = solved by the oracle within 10^8 nodes in the
    budgeted run (a fixed list of 3958), 'full' = all 4096."""
    path = os.path.join(GOLDEN, "batch_seed0.jsonl")
    recs = [json.loads(l) for l in open(path) if l.strip()]
    if which == "full":
        return sorted(r["i"] for r in recs)
    return sorted(r["i"] for r in recs if r["status"] == "ok")


def split_by_work(indices, work, world):
    """Longest-processing-time split of graphs over `world` ranks: heaviest
    estimated work first, each onto the least-loaded rank.  Returns one sorted
    index list per rank."""
    order = sorted(range(len(indices)), key=lambda j: (-work[j], indices[j]))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for j in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(indices[j])
        load[r] += work[j]
    return [sorted(p) for p in parts]


def reduce_over_ranks(dist, values_max, values_sum, device=None):
    """Max of `values_max` and sum of `values_sum` over the ranks (a no-op
    without a process group)."""
    if dist is None:
        return list(values_max), list(values_sum)
    import torch
    tm = torch.tensor(values_max, dtype=torch.float64, device=device)
    ts = torch.tensor(values_sum, dtype=torch.float64, device=device)
    dist.all_reduce(tm, op=dist.ReduceOp.MAX)
    dist.all_reduce(ts)
    return [float(x) for x in tm.cpu()], [float(x) for x in ts.cpu()]


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


def cpu_sample(recs, idx_set, cores, seconds):
    """Like-for-like CPU sample: pinned graphs the oracle solved within CPU_EASY_S
    CPU seconds, every 4th by index, as many as fit `seconds` on `cores` cores by
    the oracle's recorded CPU time."""
    easy = [i for i in sorted(idx_set) if recs[i]["status"] == "ok" and recs[i]["cpu_s"] <= CPU_EASY_S][::4]
    out, acc = [], 0.0
    for i in easy:
        acc += recs[i]["cpu_s"]
        if acc > 0.5 * cores * seconds:
            break
        out.append(i)
    return out


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
    sizes = {int(r[0]): int(r[2]) for r in rows if r[1] == "ok"}
    return solved, len(rows), wall, sizes


def run_ref_cuda(graphs, opts, timeout_s=60.0):
    """The reference's own CUDA program, one process per graph (its CLI and its
    Results.csv row; hybrid MVC kernel, default sizing).  Returns per-graph
    (status, size, process wall s, kernel ms)."""
    out = []
    for g, opt in zip(graphs, opts):
        with tempfile.TemporaryDirectory() as td:
            os.makedirs(os.path.join(td, "Results"))  # the reference appends Results/Results.csv
            path = os.path.join(td, "g.txt")
            W.write_reference_file(g, path)
            t0 = time.perf_counter()
            try:
                p = subprocess.run([REF_CUDA, "-f", path, "-o", "bench"], cwd=td, capture_output=True, text=True,
                                   timeout=timeout_s)
            except subprocess.TimeoutExpired:
                out.append(("timeout", None, timeout_s, None))
                break
            wall = time.perf_counter() - t0
            try:
                row = open(os.path.join(td, "Results", "Results.csv")).read().strip().splitlines()[-1].split(",")
                size = int(row[18])
                kms = float(row[21])
            except (OSError, IndexError, ValueError):
                out.append(("error", None, wall, None))
                break
            out.append(("ok" if p.returncode == 0 and size == opt else "wrong", size, wall, kms))
    return out


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


def _profile(path, key):
    if os.path.exists(path):
        return json.load(open(path)).get(key)
    return None


# ---------------------------------------------------------------- ranks

def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1 and args.impl == "ours":
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=900))
        pg = dist
    return world, rank, local, pg


def maybe_relaunch(args):
    """`bench.py --gpus N` outside torchrun: start N ranks under
    torch.distributed.run (127.0.0.1 rendezvous) and exit with their status."""
    if args.gpus <= 1 or "WORLD_SIZE" in os.environ:
        return
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    sys.exit(subprocess.run(cmd).returncode)


# ---------------------------------------------------------------- arms

def reference_arm(args, world, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    if not os.path.exists(REF_BENCH):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_bench was not built (no reference tree)"}))
        return
    recs = golden_batch()
    idx = cpu_sample(recs, set(pinned_indices(args.set)), threads, args.ref_step_s)
    graphs = [W.batch_instance(i) for i in idx]
    times, solved_l, wrong = [], [], 0
    for step in range(args.warmup + args.steps):
        solved, tried, wall, sizes = run_ref_bench(graphs, threads, 120.0, 1e9)
        wrong += sum(1 for j, s in sizes.items() if s != recs[idx[j]]["opt"])
        if step >= args.warmup:
            times.append(wall)
            solved_l.append(solved)
    value = sum(solved_l) / sum(times)
    sample = (f"{len(idx)} pinned graphs of the batched workload (every 4th by index among those the oracle "
              f"solved within {CPU_EASY_S} CPU s), all run to their optimum, {threads} processes")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "instances/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)),
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": "batched MVC, G(n,p) n~U{30..200} avg deg~U[3,12]: bounded CPU sample", "graphs": len(idx),
                       "solved_per_step": float(np.mean(solved_l)), "wrong": wrong},
            "cpu_baseline": {"value": value, "unit": "instances/s", "cores": threads, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": "instances/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def _check(sols, opts):
    """(solved, wrong): a solution counts when its status is OK and its size is
    the pinned optimum (a None optimum is not checked)."""
    solved = wrong = 0
    for s, o in zip(sols, opts):
        if s.status != 0:
            wrong += 1
        elif o is not None and s.size != o:
            wrong += 1
        else:
            solved += 1
    return solved, wrong


def served_leg(seconds, rate, node_limit=0):
    """A short served stream (vc_server, Poisson arrivals, 70% MVC / 30% PVC)
    over the oracle-pinned stream pool; returns its figures."""
    import vcgpu
    recs = [json.loads(l) for l in open(os.path.join(GOLDEN, "stream_seed0.jsonl")) if l.strip()]
    pinned = sorted([r for r in recs if r["status"] == "ok"], key=lambda r: r["i"])
    pool = [(W.stream_instance(r["i"]), r["opt"]) for r in pinned]
    rng = np.random.default_rng(1)
    arrivals, t = [], 0.0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t > seconds:
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
    per_req = []  # (latency ms, tree nodes, lane, n)
    with vcgpu.Server(max_vertices=max_n, max_requests=4096, mem_budget=2 << 30) as srv:
        lanes = srv.shape()
        for g, opt in pool[:32]:  # warm-up: kernel launch, first-touch of buffers
            srv.wait(srv.submit(g, "mvc", node_limit=node_limit))
        outstanding = {}
        t0 = time.perf_counter()
        i = 0
        while i < len(reqs) or outstanding:
            now = time.perf_counter() - t0
            while i < len(reqs) and reqs[i][0] <= now:
                a, g, kind, k, opt = reqs[i]
                outstanding[srv.submit(g, kind, k=k, node_limit=node_limit, validate=False)] = (g, kind, k, opt)
                i += 1
            for tk in srv.completed():
                r = srv.poll(tk, want_cover=False)
                g, kind, k, opt = outstanding.pop(tk)
                done += 1
                lat.append(r.total_ms)
                lane_lat.setdefault(vcgpu.Server.lane(tk), []).append(r.total_ms)
                per_req.append((r.total_ms, r.tree_nodes, vcgpu.Server.lane(tk), g.n))
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
    # the tail: are the slowest 1% the requests with the most search work, or
    # requests that waited behind others?
    p99 = float(np.percentile(lat, 99))
    tail = [x for x in per_req if x[0] >= p99]
    nodes_all = np.asarray([x[1] for x in per_req], dtype=np.float64)
    tail_info = {"requests": len(tail), "median_tree_nodes": float(np.median([x[1] for x in tail])) if tail else None,
                 "median_tree_nodes_all": float(np.median(nodes_all)),
                 "tail_share_of_top1pct_work": (sum(1 for x in tail if x[1] >= np.percentile(nodes_all, 99)) / len(tail))
                 if tail else None,
                 "median_n": float(np.median([x[3] for x in tail])) if tail else None}
    return {"requests": len(reqs), "completed": done, "completed_per_s": done / wall, "wrong": bad, "tail": tail_info,
            "budget_exceeded": budget, "offered_per_s": rate, "seconds": seconds,
            "p50_latency_ms": float(np.percentile(lat, 50)), "p99_latency_ms": float(np.percentile(lat, 99)),
            "mean_latency_ms": float(lat.mean()), "pool": len(pool), "pool_coverage": len(pinned) / max(len(recs), 1),
            "max_vertices": max_n, "lanes": lanes}


def our_arm(args, world, rank, local, pg):
    import torch
    import vcgpu
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    recs = golden_batch()
    all_idx = pinned_indices(args.set)
    base = [W.batch_instance(i) for i in all_idx] if world > 1 else None
    work = [g.n * g.m for g in base] if base is not None else None
    mine = split_by_work(all_idx, work, world)[rank] if world > 1 else all_idx
    graphs = [W.batch_instance(i) for i in mine]
    opts = [recs[i]["opt"] if i in recs else None for i in mine]
    arena = W.pack(graphs)
    n_arr = np.asarray([g.n for g in graphs], np.int64)
    m_arr = np.asarray([g.m for g in graphs], np.int64)
    bnode = 4 * (3 * n_arr + 2 * m_arr + 1)
    d_rp = torch.from_numpy(arena.row_ptr.astype(np.int32)).to(dev)
    d_col = torch.from_numpy(arena.col.astype(np.int32)).to(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def device_step():
        return vcgpu.solve_batch(arena, "mvc", node_limit=args.node_limit, time_limit=args.time_limit, want_cover=True,
                                 device=local, d_row_ptr=d_rp.data_ptr(), d_col=d_col.data_ptr(), validate=False,
                                 stream=stream.cuda_stream)

    def barrier():
        if pg is not None:
            pg.barrier()

    wrong_total = 0
    for _ in range(args.warmup):
        _, sols = device_step()
        wrong_total += _check(sols, opts)[1]
    times, sols_last = [], None
    launches0 = vcgpu.kernel_launches()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1)  # L2 flush: the arena (~20 MB) is smaller than L2
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
            wrong_total += _check(sols, opts)[1]
    clocks = clk.summary()
    launches = (vcgpu.kernel_launches() - launches0) // max(args.steps, 1)
    _, shape = vcgpu.debug_stats()
    launch_shape = {"grid": int(shape[0]), "block": int(shape[1]), "smem_bytes": int(shape[2]),
                    "search_units": int(shape[3]), "dense": bool(int(shape[4]) >> 31)}
    step_s = float(np.mean(times))
    solved, _ = _check(sols_last, opts)
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
    e2e_times, solved_e = [], 0
    for _ in range(max(1, min(args.e2e_steps, args.steps))):
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        st_e, sols_e = vcgpu.solve_batch(host_arena, "mvc", node_limit=args.node_limit, time_limit=args.time_limit,
                                         want_cover=True, device=local, validate=True)
        torch.cuda.synchronize()
        e2e_times.append(time.perf_counter() - t0)
        barrier()
        s_e, w_e = _check(sols_e, opts)
        solved_e += s_e
        wrong_total += w_e
    e2e_s = float(np.mean(e2e_times))
    solved_e /= len(e2e_times)

    (step_s, e2e_s), (solved_all, solved_e_all, nodes_all, wrong_all, graphs_all) = reduce_over_ranks(
        pg, [step_s, e2e_s], [solved, solved_e, nodes, wrong_total, len(graphs)], device=dev)
    if rank != 0:
        return

    extras = {}
    if world == 1:
        extras = rank0_samples(args, recs, all_idx, local)
    if args.served_seconds > 0:
        extras["served"] = served_leg(args.served_seconds, args.rate)

    hbm, src = measured_peaks()
    achieved = alg_bytes / kernel_s / 1e9
    ipn = _profile(ISSUE_PROFILE, "warp_inst_per_node")
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    issue = None
    if ipn:
        issue_rate = ipn * (nodes / kernel_s)
        issue = {"achieved_warp_inst_per_s": issue_rate, "peak_warp_inst_per_s": sms * 4 * sm_mhz * 1e6,
                 "frac": issue_rate / (sms * 4 * sm_mhz * 1e6), "warp_inst_per_node": ipn,
                 "source": "warp instructions per tree node from ncu smsp__inst_executed.sum on the search kernel "
                           "(profiles/k_dense_issue.json); SMs x 4 schedulers x median sampled SM clock"}
    workload = ("batched MVC, config 3: the 3958 of 4096 G(n,p) graphs (n~U{30..200}, avg degree~U[3,12], seed "
                "per graph) whose optimum the CPU oracle pinned within 1e8 tree nodes, each solved to its proven "
                "optimum, no node budget, one persistent launch") if args.set == "pinned" else \
               "batched MVC, config 3: all 4096 G(n,p) graphs, each solved to its proven optimum, no node budget"
    line = {
        "metric": METRIC, "value": solved_all / step_s, "unit": "instances/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * step_s, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {
            "workload": workload, "graphs": int(graphs_all), "solved": int(solved_all), "wrong": int(wrong_all),
            "node_limit": args.node_limit, "tree_nodes_per_s": nodes_all / step_s, "tree_nodes_per_step": nodes_all,
            "p50_latency_ms": float(np.percentile(done, 50)) if done.size else None,
            "p99_latency_ms": float(np.percentile(done, 99)) if done.size else None,
            "l2": "flushed before every timed step (256 MB write); arena ~%.0f MB" % ((arena.row_ptr.nbytes + arena.col.nbytes) / 1e6),
            "parallelism": f"{world} GPU(s), the set split across ranks by estimated work (n*m), no collective on the data path",
            "launch": launch_shape, "e2e_steps": len(e2e_times),
            **{k: v for k, v in extras.items() if k != "cpu_baseline"},
        },
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": _profile(TRAFFIC_PROFILE, "dram_bytes_per_launch"), "peak_source": src,
                     "note": "algorithmic bytes 4*(3n+2m+1) per tree node over the search kernel's event-timed "
                             "duration; the search state is SM-resident, so the binding roof is instruction issue",
                     "issue": issue},
        "cpu_baseline": extras.get("cpu_baseline"),
        "e2e": {"value": solved_e_all / e2e_s, "unit": "instances/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    print(json.dumps(line))


def rank0_samples(args, recs, all_idx, local):
    """Like-for-like samples measured on rank 0 at N = 1: plain vs batched, the
    reference's CPU solver and its CUDA program against this library on the same
    graphs."""
    import vcgpu
    out = {}
    # plain (one call per graph) vs batched (one call), same graphs, host API
    samp = all_idx[::args.plain_every]
    g_s = [W.batch_instance(i) for i in samp]
    o_s = [recs[i]["opt"] for i in samp]
    t0 = time.perf_counter()
    _, sb = vcgpu.solve_batch(W.pack(g_s), "mvc", time_limit=args.time_limit, device=local)
    tb = time.perf_counter() - t0
    t0 = time.perf_counter()
    sp = [vcgpu.solve(g, "mvc", time_limit=args.time_limit, device=local) for g in g_s]
    tp = time.perf_counter() - t0
    sb_ok, sb_bad = _check(sb, o_s)
    sp_ok, sp_bad = _check(sp, o_s)
    out["plain_vs_batched"] = {
        "sample": f"every {args.plain_every}th graph of the step's set ({len(samp)} graphs)",
        "batched_instances_per_s": sb_ok / tb, "plain_instances_per_s": sp_ok / tp,
        "batched_over_plain": (sb_ok / tb) / (sp_ok / tp) if sp_ok else None, "wrong": sb_bad + sp_bad,
        "batched_s": tb, "plain_s": tp, "tree_nodes": sum(s.tree_nodes for s in sb)}
    # the reference's CPU solver on the CPU sample, and this library on the same graphs
    threads = os.cpu_count() or 1
    idx_c = cpu_sample(recs, set(all_idx), threads, args.cpu_sample_s)
    g_c = [W.batch_instance(i) for i in idx_c]
    o_c = [recs[i]["opt"] for i in idx_c]
    t0 = time.perf_counter()
    _, sc = vcgpu.solve_batch(W.pack(g_c), "mvc", time_limit=args.time_limit, device=local)
    tg = time.perf_counter() - t0
    gpu_ok, gpu_bad = _check(sc, o_c)
    if os.path.exists(REF_BENCH):
        c_solved, c_tried, c_wall, sizes = run_ref_bench(g_c, threads, 120.0, 1e9)
        c_bad = sum(1 for j, s in sizes.items() if s != o_c[j])
        out["cpu_baseline"] = {
            "value": c_solved / c_wall, "unit": "instances/s", "cores": threads, "kind": "reference",
            "sample": f"{len(idx_c)} pinned graphs of the batched workload (every 4th by index among those the oracle "
                      f"solved within {CPU_EASY_S} CPU s), each run to its optimum by the reference's Sequential, "
                      f"{threads} processes; {c_solved} solved in {c_wall:.1f} s, {c_bad} wrong",
            "gpu_same_sample_instances_per_s": gpu_ok / tg, "gpu_same_sample_wrong": gpu_bad,
            "gpu_over_cpu_same_sample": (gpu_ok / tg) / (c_solved / c_wall) if c_solved else None}
    # the reference's own CUDA program (one process per graph) vs vc_solve on the same graphs
    if os.path.exists(REF_CUDA) and args.refcuda_graphs > 0:
        gq, oq = g_c[:args.refcuda_graphs], o_c[:args.refcuda_graphs]
        rows = run_ref_cuda(gq, oq)
        ok = [r for r in rows if r[0] == "ok"]
        t0 = time.perf_counter()
        mine = [vcgpu.solve(g, "mvc", time_limit=args.time_limit, device=local) for g in gq]
        tm = time.perf_counter() - t0
        m_ok, m_bad = _check(mine, oq)
        status = "ok" if len(ok) == len(gq) else f"stopped: {rows[-1][0]} on graph {len(rows) - 1} of the sample"
        out["reference_cuda"] = {
            "program": "the reference's own CUDA build (VC 1 hybrid MVC kernel, default launch sizing), sm_100a, "
                       "one process per graph (its ./output CLI and Results.csv row)",
            "graphs": len(gq), "status": status, "correct": len(ok),
            "instances_per_s_process": len(ok) / sum(r[2] for r in rows) if ok else None,
            "kernel_ms_sum": sum(r[3] for r in ok) if ok else None,
            "ours_plain_instances_per_s": m_ok / tm, "ours_plain_wrong": m_bad,
            "ours_plain_kernel_ms_sum": sum(s.kernel_ms for s in mine)}
    # the same comparison on the reference's own graph files (those both sides
    # answer within seconds; `--workload files` runs all of them)
    if args.ref_files:
        rows = compare_files([f for f in args.ref_files.split(",") if f], 30.0, device=local)
        both = [r for r in rows if r.get("ours", {}).get("correct") and r.get("reference_cuda", {}).get("correct")]
        out["reference_files"] = {
            "files": rows,
            "ours_correct": sum(1 for r in rows if r.get("ours", {}).get("correct")),
            "reference_correct": sum(1 for r in rows if r.get("reference_cuda", {}).get("correct")),
            "kernel_ms_sum_where_both_correct": {"ours": round(sum(r["ours"]["kernel_ms"] for r in both), 2),
                                                 "reference_cuda": round(sum(r["reference_cuda"]["kernel_ms"]
                                                                             for r in both), 2)}}
    return out


def stream_arm(args, world, rank):
    """The served stream through vc_server alone (rank 0; other ranks have no work)."""
    if rank != 0:
        return
    s = served_leg(args.stream_seconds, args.rate, args.node_limit)
    line = {"metric": METRIC, "value": s["completed_per_s"], "unit": "requests/s", "n_gpus": 1, "steps": 1,
            "warmup": 1, "ms_per_step": 1e3 * args.stream_seconds, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": f"served stream: Poisson {args.rate:.0f} req/s for {args.stream_seconds:.0f} s, "
                                   "70% MVC / 30% PVC (k = opt or opt-1), G(n,p) and random 3-regular, "
                                   "n log-uniform [50,5000], drawn from the oracle-pinned pool", **s}}
    print(json.dumps(line))


# The reference's graph files its loader reads as they are (1-based ids;
# auxFunctions.cpp:150-154 shifts every id down by one, so the 0-based
# formated_* and lastfm files are not valid input to it).
REF_FILES_1BASED = ["cop_hat300-1.txt", "cop_hat300-2.txt", "cop_hat300-3.txt", "cop_hat500-1.txt", "cop_hat500-2.txt",
                    "cop_hat500-3.txt", "cop_hat700-1.txt", "cop_hat700-2.txt", "cop_hat1000-1.txt",
                    "cop_hat1000-2.txt", "Power-Grid.txt", "Sister-Cities.txt", "vc-exact_009.txt", "vc-exact_023.txt"]
# Files the reference's program is not run on: its stacks take (UB + 1) * n * 4
# bytes per block (stack.cuh:39, unchecked cudaMalloc), about 1.8 GB per block
# and hundreds of GB in all for these, so its kernel would run on a failed
# allocation.
REF_CUDA_NOT_RUN = {"vc-exact_009.txt": "stack allocation of (UB+1)*n*4 bytes per block (~3.3 GB) fails unchecked",
                    "vc-exact_023.txt": "stack allocation of (UB+1)*n*4 bytes per block (~1.8 GB) fails unchecked"}


def compare_files(names, tl, device=-1):
    """The reference's graph files (test/test_graphs, known optima from
    test/runGraphs.py:8-30): this library's plain vc_solve (host buffers, no
    upper bound given; the second of two calls is reported when the first
    solved it) and the reference's own CUDA program (oracle/_ref/cuda/output:
    hybrid MVC kernel, default sizing, its CPU upper bounds first), each with
    `tl` seconds per file.  Per file: kernel time, call time, and whether the
    answer equals the known optimum."""
    import gzip
    import shutil
    import vcgpu
    known = json.load(open(os.path.join(REPO, "tests", "golden", "known_answers.json")))["mvc"]
    rows = []
    for name in names:
        src = os.path.join(REPO, "oracle", "_ref", "graphs", name + ".gz")
        if not os.path.exists(src):
            rows.append({"file": name, "missing": "stage with `make -C oracle graphs`"})
            continue
        zero = name.startswith("formated_") or name.startswith("lastfm")
        g = W.read_reference_file(src, one_based=not zero)
        r = vcgpu.solve(g, "mvc", time_limit=tl, device=device)
        r = vcgpu.solve(g, "mvc", time_limit=tl, device=device) if r.status == vcgpu.VC_OK else r
        ok = r.status == vcgpu.VC_OK and r.size == known[name] and W.is_cover(g, r.cover)
        ours = {"status": vcgpu.STATUS_NAMES.get(r.status, r.status), "size": r.size, "correct": bool(ok),
                "kernel_ms": round(r.kernel_ms, 2), "call_ms": round(r.total_ms, 2), "tree_nodes": int(r.tree_nodes)}
        ref = {"unavailable": "oracle/_ref/cuda/output not built"}
        if name in REF_CUDA_NOT_RUN:
            ref = {"not_run": REF_CUDA_NOT_RUN[name]}
        elif zero:
            ref = {"not_run": "0-based file (the reference's loader shifts every id down by one)"}
        elif os.path.exists(REF_CUDA):
            with tempfile.TemporaryDirectory() as td:
                os.makedirs(os.path.join(td, "Results"))
                path = os.path.join(td, name)
                with gzip.open(src, "rb") as fi, open(path, "wb") as fo:
                    shutil.copyfileobj(fi, fo)
                t0 = time.perf_counter()
                try:
                    p = subprocess.run([REF_CUDA, "-f", path, "-o", "files"], cwd=td, capture_output=True, text=True,
                                       timeout=tl + 30)
                    wall = time.perf_counter() - t0
                    row = open(os.path.join(td, "Results", "Results.csv")).read().strip().splitlines()[-1].split(",")
                    size = int(row[18])
                    ref = {"status": "ok" if p.returncode == 0 else f"exit {p.returncode}", "size": size,
                           "correct": p.returncode == 0 and size == known[name], "kernel_ms": float(row[21]),
                           "process_s": round(wall, 2), "cpu_upper_bounds": [int(row[14]), int(row[16])]}
                except subprocess.TimeoutExpired:
                    ref = {"status": "timeout", "process_s": tl + 30}
                except (OSError, IndexError, ValueError) as e:
                    ref = {"status": "error", "error": repr(e)[:120]}
        rows.append({"file": name, "n": g.n, "m": g.m, "known_opt": known[name], "ours": ours, "reference_cuda": ref})
    return rows


def files_arm(args, world, rank):
    """`--workload files`: compare_files over --files (default: every 1-based
    file), --file-time-limit seconds per file; one JSON line."""
    if rank != 0:
        return
    names = [f for f in args.files.split(",") if f] or REF_FILES_1BASED
    tl = args.file_time_limit
    line = {"metric": "reference graph files: kernel ms per file, this library vs the reference's CUDA program",
            "unit": "ms", "higher_is_better": False, "n_gpus": 1, "data": "the reference's test/test_graphs files",
            "time_limit_s": tl, "files": compare_files(names, tl)}
    print(json.dumps(line))


REF_CUDA_MCM = os.path.join(REPO, "oracle", "_ref", "cuda_mcm", "output")


def mcm_arm(args, world, rank):
    """The MCM mode: vc_mcm against the reference's own default build
    (oracle/_ref/cuda_mcm/output, `#define VC 0`, one process per graph) on the
    graphs of tests/golden/mcm.json, whose answers (2 * maximum matching +
    isolated vertices) come from maximum-cardinality matchings.  The reference
    runs --file-time-limit seconds per graph."""
    if rank != 0:
        return
    import vcgpu
    recs = json.load(open(os.path.join(REPO, "tests", "golden", "mcm.json")))
    rows = []
    for r in recs:
        g = (W.gnp(r["n"], r["d"] / (r["n"] - 1), r["seed"]) if r["family"] == "gnp"
             else W.planted_matching(r["n"], r["d"], r["seed"]))
        s = vcgpu.mcm(g, time_limit=60.0)
        s = vcgpu.mcm(g, time_limit=60.0) if s.status == vcgpu.VC_OK else s
        row = {"graph": f"{r['family']} n={r['n']} d={r['d']} seed={r['seed']}", "expect": r["expect"],
               "ours": {"status": vcgpu.STATUS_NAMES.get(s.status, s.status), "maximum": s.size,
                        "correct": s.status == vcgpu.VC_OK and s.size == r["expect"],
                        "kernel_ms": round(s.kernel_ms, 3), "tree_nodes": s.tree_nodes}}
        if os.path.exists(REF_CUDA_MCM):
            with tempfile.TemporaryDirectory() as td:
                os.makedirs(os.path.join(td, "Results"))
                path = os.path.join(td, "g.txt")
                W.write_reference_file(g, path)
                t0 = time.perf_counter()
                try:
                    p = subprocess.run([REF_CUDA_MCM, "-f", path, "-o", "mcm"], cwd=td, capture_output=True,
                                       text=True, timeout=args.file_time_limit)
                    f = open(os.path.join(td, "Results", "Results.csv")).read().strip().splitlines()[-1].split(",")
                    row["reference_cuda"] = {"status": "ok" if p.returncode == 0 else f"exit {p.returncode}",
                                             "maximum": int(f[18]), "correct": int(f[18]) == r["expect"],
                                             "kernel_ms": float(f[21]),
                                             "process_s": round(time.perf_counter() - t0, 2)}
                except subprocess.TimeoutExpired:
                    row["reference_cuda"] = {"status": "timeout", "process_s": args.file_time_limit}
                except (OSError, IndexError, ValueError) as e:
                    row["reference_cuda"] = {"status": "error", "error": repr(e)[:120]}
        rows.append(row)
    print(json.dumps({"metric": "MCM mode: kernel ms per graph, this library vs the reference's default build",
                      "unit": "ms", "higher_is_better": False, "n_gpus": 1, "data": "synthetic (tests/golden/mcm.json)",
                      "graphs": rows}))


def ub_arm(args, world, rank):
    """The reference's upper-bound heuristics on the GPU (vc_remove_max_ub /
    vc_remove_edge_ub): Chung-Lu n=100000 (one graph) and the 4096 batched
    graphs, beside the reference's own CPU functions on the Chung-Lu graph
    (forked child, one core).  rand() value 12345 for RemoveEdge."""
    if rank != 0:
        return
    import vcgpu
    g5 = W.chung_lu()
    arena = W.pack(W.batch_graphs(4096, seed=0))
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
                                   "max degree 2000, seed 7) and 4096 batched G(n,p) graphs", **out,
                       "reference_cpu": cpu}}
    print(json.dumps(line))


def profile_arm(args):
    """Small torch-free launches for ncu.  --case batch: the first --count graphs
    of the step's set in one vc_solve_batch call (the dense kernel); csr-batch:
    the same graphs with the CSR kernel forced; file: one of the reference's
    graph files (--file, staged by `make -C oracle graphs`; the formated_* and
    lastfm files are 0-based), one vc_solve; powergrid: --case file on
    Power-Grid (n = 4942, the CSR kernel with CTA search units).  --reps times
    each."""
    import vcgpu
    if args.case in ("powergrid", "file"):
        name = "Power-Grid.txt" if args.case == "powergrid" else args.file
        path = os.path.join(REPO, "oracle", "_ref", "graphs", name + ".gz")
        g = W.read_reference_file(path, one_based=not (name.startswith("formated_") or name.startswith("lastfm")))
        for it in range(args.reps):
            r = vcgpu.solve(g, "mvc", time_limit=args.time_limit)
            print(f"rep {it}: status {r.status} size {r.size} tree nodes {r.tree_nodes} kernel {r.kernel_ms:.1f} ms "
                  f"{r.tree_nodes / max(r.kernel_ms, 1e-9) / 1e3:.1f} Mnodes/s", flush=True)
        return
    idx = pinned_indices(args.set)[:args.count]
    arena = W.pack([W.batch_instance(i) for i in idx])
    if args.case == "csr-batch":
        vcgpu.debug_stats(2)
    for it in range(args.reps):
        st, sols = vcgpu.solve_batch(arena, "mvc", node_limit=args.node_limit, time_limit=args.time_limit)
        nodes = sum(s.tree_nodes for s in sols)
        solved = sum(1 for s in sols if s.status == vcgpu.VC_OK)
        print(f"rep {it}: status {st} solved {solved}/{len(idx)} tree nodes {nodes} kernel {sols[0].kernel_ms:.1f} ms "
              f"{nodes / max(sols[0].kernel_ms, 1e-9) / 1e3:.1f} Mnodes/s", flush=True)


def main():
    args = parse()
    if args.workload == "profile":
        profile_arm(args)
        return
    if args.impl == "ours":
        maybe_relaunch(args)
    world, rank, local, pg = dist_setup(args)
    try:
        if args.impl == "reference":
            reference_arm(args, world, rank)
        elif args.workload == "stream":
            stream_arm(args, world, rank)
        elif args.workload == "ub":
            ub_arm(args, world, rank)
        elif args.workload == "files":
            files_arm(args, world, rank)
        elif args.workload == "mcm":
            mcm_arm(args, world, rank)
        else:
            our_arm(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
