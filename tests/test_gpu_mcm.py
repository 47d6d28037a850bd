"""GPU parity of the MCM mode (vc_mcm): the search of the reference's default
build (`#define VC 0`, GlobalWorkList_MCM.cuh:13-190), whose finished answer is
2 * maximum matching + isolated vertices.  Small graphs are checked against the
oracle's exhaustive restatement of that search (run here); every graph of
tests/golden/mcm.json against its answer from a maximum-cardinality matching
(made by tests/golden/make_golden.py mcm, where the oracle agrees on the G(n,p)
ones; the search is exhaustive, so the larger graphs are planted matchings it
meets first).  The command line's -M mode prints the reference's line and row."""
import json
import os
import subprocess

import numpy as np
import pytest

import oracle as O
import vcgpu
from vcgpu import workloads as W

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CLI = os.path.join(REPO, "parallel-vertex-cover-algorithms-on-gpus_b200", "output")
RECS = json.load(open(os.path.join(HERE, "golden", "mcm.json")))


def _graph(r):
    if r["family"] == "gnp":
        return W.gnp(r["n"], r["d"] / (r["n"] - 1), r["seed"])
    return W.planted_matching(r["n"], r["d"], r["seed"])


def test_mcm_small_graphs_vs_oracle():
    rng = np.random.default_rng(31)
    for _ in range(40):
        n = int(rng.integers(1, 15))
        g = W.gnp(n, float(rng.uniform(0.05, 0.5)), int(rng.integers(1 << 30)))
        st, best, _ = O.mcm(g)
        assert st == O.OK
        r = vcgpu.mcm(g, time_limit=30.0)
        assert r.status == vcgpu.VC_OK and r.size == best, (n, r, best)


@pytest.mark.parametrize("rec", RECS, ids=[f"{r['family']}{r['n']}" for r in RECS])
def test_mcm_golden(rec):
    g = _graph(rec)
    assert g.m == rec["m"]
    r = vcgpu.mcm(g, time_limit=60.0)
    assert r.status == vcgpu.VC_OK and r.size == rec["expect"], (rec, r)


def test_mcm_limits_and_errors():
    g = W.gnp(300, 2.0 / 299, 951)  # many unmatched vertices: a large tree
    r = vcgpu.mcm(g, node_limit=20000, time_limit=30.0)
    assert r.status == vcgpu.VC_BUDGET and r.size > 0
    big = W.planted_matching(1026, 3.0, 1)
    assert vcgpu.mcm(big).status == vcgpu.VC_ERR_TOO_LARGE
    empty = W.from_edges(5, np.zeros((0, 2), dtype=np.int64))
    r = vcgpu.mcm(empty)
    assert r.status == vcgpu.VC_OK and r.size == 5  # every vertex isolated


@pytest.mark.skipif(not os.path.exists(CLI), reason="output not built")
def test_mcm_command_line(tmp_path):
    rec = next(r for r in RECS if r["family"] == "planted" and r["n"] == 256)
    g = _graph(rec)
    path = tmp_path / "g.txt"
    W.write_reference_file(g, str(path))
    p = subprocess.run([CLI, "-M", "-f", str(path), "-o", "mcm"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=120)
    assert p.returncode == 0, p.stderr
    assert f"Size of maximum matching: {rec['expect'] // 2}" in p.stdout
    row = (tmp_path / "Results" / "Results.csv").read_text().strip().splitlines()[-1].split(",")
    assert len(row) == 22 and row[18] == str(rec["expect"]) and row[20] == "0"
    p = subprocess.run([CLI, "-M", "-i", "pvc", "-k", "3", "-f", str(path)], cwd=tmp_path, capture_output=True,
                       text=True, timeout=60)
    assert p.returncode == 1 and "unsupported version 1 instance 1" in p.stdout
