"""The reference's upper-bound heuristics on the GPU (vc_remove_max_ub,
vc_remove_edge_ub) against their exact CPU restatements in the oracle, which
tests/test_oracle.py pins to the reference's own compiled functions: the same
bound on every graph, and a valid cover of that size."""
import json
import os

import numpy as np
import pytest

import oracle as O
import vcgpu
from vcgpu import workloads as W

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _graphs():
    out = []
    for i in range(160):
        rng = np.random.default_rng(9000 + i)
        n = int(rng.integers(2, 400))
        d = float(rng.uniform(1.2, 9.0))
        if i % 4 == 3:
            out.append(W.random_regular(n + (n % 2), 3, i))
        else:
            out.append(W.gnp(n, min(1.0, d / max(n - 1, 1)), 9000 + i))
    out.append(W.from_edges(5, np.zeros((0, 2))))          # no edges
    out.append(W.from_edges(2, np.array([[0, 1]])))         # one edge
    return out


def _check(graphs, ubs, covers, want):
    for g, u, c, w in zip(graphs, ubs, covers, want):
        assert u == w, (g.name, u, w)
        assert W.is_cover(g, c) and int(c.sum()) == u, g.name


def test_remove_max_matches_oracle_batched():
    graphs = _graphs()
    ubs, covers, _ = vcgpu.remove_max_ub(W.pack(graphs))
    _check(graphs, ubs, covers, [O.remove_max_ub(g)[0] for g in graphs])


@pytest.mark.parametrize("r", [0, 7, 1804289383])
def test_remove_edge_matches_oracle_batched(r):
    graphs = _graphs()
    ubs, covers, _ = vcgpu.remove_edge_ub(W.pack(graphs), r)
    _check(graphs, ubs, covers, [O.remove_edge_ub(g, r)[0] for g in graphs])


def test_configs_one_two_five():
    """Configs 1 and 2 for both heuristics; config 5 (Chung-Lu n = 100000) for
    RemoveMax, whose reference value is pinned here (31217, equal to the optimum)."""
    small = json.load(open(os.path.join(GOLDEN, "small.json")))
    for g in (W.config1_graph(), W.config2_graph()):
        ubs, covers, _ = vcgpu.remove_max_ub(g)
        _check([g], ubs, covers, [O.remove_max_ub(g)[0]])
        ubs, covers, _ = vcgpu.remove_edge_ub(g, 12345)
        _check([g], ubs, covers, [O.remove_edge_ub(g, 12345)[0]])
    g5 = W.chung_lu()
    ubs, covers, _ = vcgpu.remove_max_ub(g5)
    assert ubs[0] == 31217 == small["config5"]["opt"]
    assert W.is_cover(g5, covers[0])
