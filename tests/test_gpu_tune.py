"""The autotuner (vc_autotune / vc_set_tuning): it measures launch shapes per
size class and installs the fastest; answers stay exact under any tuned shape,
and a table of zeros returns to the built-in rules."""
import json
import os

import numpy as np
import pytest

import vcgpu
from vcgpu import workloads as W

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _golden(max_nodes, count):
    recs = [json.loads(l) for l in open(os.path.join(GOLDEN, "batch_seed0.jsonl")) if l.strip()]
    return sorted([r for r in recs if r["status"] == "ok" and r["nodes"] <= max_nodes], key=lambda r: r["i"])[:count]


def test_autotune_installs_valid_shapes_and_answers_stay_exact():
    try:
        st, words, table = vcgpu.autotune(slice_s=0.08)
        assert st == vcgpu.VC_OK
        for row in table:
            assert row["set"] == 1 and row["warps"] in (2, 4, 8) and row["pool_per_warp"] in (1, 2, 4)
            assert row["nodes_per_s"] > 0 and row["ring_bias"] in (-64, -16, 0, 4, 32) and row["ring_first"] in (0, 1)
        recs = _golden(500_000, 120)
        graphs = [W.batch_instance(r["i"]) for r in recs]
        rng = np.random.default_rng(5)
        for n in (700, 1500):  # the 16-bit dense class and the CSR class
            graphs.append(W.gnp(n, 2.5 / (n - 1), int(rng.integers(1 << 30))))
        opts = [r["opt"] for r in recs] + [vcgpu.solve(g, "mvc", time_limit=60).size for g in graphs[len(recs):]]
        _, sols = vcgpu.solve_batch(W.pack(graphs), "mvc", time_limit=60.0)
        for g, s, o in zip(graphs, sols, opts):
            assert s.status == vcgpu.VC_OK and s.size == o and W.is_cover(g, s.cover) and int(s.cover.sum()) == o
        # the same table installed again is accepted; a malformed one is not
        assert vcgpu.set_tuning(words) == vcgpu.VC_OK
        bad = words.copy()
        bad[2] = 3  # warps must be 2, 4 or 8
        assert vcgpu.set_tuning(bad) == vcgpu.VC_ERR_INVALID
    finally:
        assert vcgpu.set_tuning(np.zeros(vcgpu.TUNE_WORDS * len(vcgpu.TUNE_CLASSES), dtype=np.uint32)) == vcgpu.VC_OK
