"""A small, torch-free driver of the batched entry point for profiler captures.

Solves the first --count graphs of the batched workload (G(n, p), n in
[30, 200], average degree in [3, 12], seed 0) in one launch, --reps times, with
the same per-graph node budget as bench.py, and prints nodes and kernel time.

    python parallel-vertex-cover-algorithms-on-gpus_b200/vcgpu/profile_case.py --count 512
"""
import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import vcgpu  # noqa: E402
from vcgpu import workloads as W  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=512)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--node-limit", type=int, default=1 << 22)
    a = ap.parse_args()
    arena = W.pack(W.batch_graphs(a.count, seed=0))
    for it in range(a.reps):
        st, sols = vcgpu.solve_batch(arena, "mvc", node_limit=a.node_limit, time_limit=120.0)
        nodes = sum(s.tree_nodes for s in sols)
        solved = sum(1 for s in sols if s.status == vcgpu.VC_OK)
        print(f"rep {it}: status {st} solved {solved}/{a.count} tree nodes {nodes} kernel {sols[0].kernel_ms:.1f} ms "
              f"{nodes / max(sols[0].kernel_ms, 1e-9) / 1e3:.1f} Mnodes/s", flush=True)


if __name__ == "__main__":
    main()
