"""Seeded generators and the CSR / arena layout (host side)."""
import numpy as np

from vcgpu import workloads as W


def _simple(g):
    rp, col = g.row_ptr.astype(np.int64), g.col.astype(np.int64)
    assert rp[0] == 0 and rp[-1] == col.size and np.all(np.diff(rp) >= 0)
    for v in range(g.n):
        row = col[rp[v]:rp[v + 1]]
        assert np.all(np.diff(row) > 0) and not np.any(row == v) and np.all(row < g.n)
    e = g.edges()
    back = {(int(b), int(a)) for a, b in e}
    assert len(back) == g.m


def test_generators_deterministic_and_simple():
    for make in (W.config1_graph, W.config2_graph, lambda: W.random_regular(100, 3, 1),
                 lambda: W.batch_instance(7), lambda: W.stream_instance(3)):
        a, b = make(), make()
        assert a.n == b.n and np.array_equal(a.row_ptr, b.row_ptr) and np.array_equal(a.col, b.col)
        _simple(a)


def test_config_shapes():
    g1 = W.config1_graph()
    assert g1.n == 60
    g2 = W.config2_graph()
    assert 2000 < g2.n <= 2400 and g2.m >= 6000
    r = W.random_regular(50, 3, 2)
    assert np.all(r.degrees() == 3)
    for i in range(50):
        g = W.batch_instance(i)
        assert 30 <= g.n <= 200


def test_planted_cover_is_a_cover():
    g = W.planted_cover(300, 50, 800, 10, 4, 9)
    # the planted set plus every second path vertex covers the graph; check the
    # weaker fact that any edge among base vertices touches the planted set size
    assert g.m >= 800 and g.n > 300


def test_pack_offsets():
    graphs = [W.batch_instance(i) for i in range(10)]
    a = W.pack(graphs)
    for i, g in enumerate(graphs):
        ro, co = int(a.row_off[i]), int(a.col_off[i])
        assert np.array_equal(a.row_ptr[ro:ro + g.n + 1], g.row_ptr)
        assert np.array_equal(a.col[co:co + g.col.size], g.col)


def test_reference_file_roundtrip(tmp_path):
    g = W.gnp(40, 0.1, 3)
    p = str(tmp_path / "g.txt")
    W.write_reference_file(g, p)
    h = W.read_reference_file(p)
    assert np.array_equal(g.row_ptr, h.row_ptr) and np.array_equal(g.col, h.col)


def test_chung_lu_small():
    g = W.chung_lu(n=3000, gamma=2.1, avg_deg=8, max_deg=200, seed=7)
    _simple(g)
    assert g.degrees().max() <= 400


def test_planted_matching_holds_its_pairs():
    """The MCM mode's large test graphs: every pair (2i, 2i+1) is an edge, so the
    maximum matching has n // 2 pairs, and the extra edges bring the average
    degree near d."""
    for n, d, seed in ((64, 6.0, 1), (101, 4.0, 2), (1024, 6.0, 3)):
        g = W.planted_matching(n, d, seed)
        assert g.n == n
        for i in range(0, n - 1, 2):
            row = g.col[g.row_ptr[i]:g.row_ptr[i + 1]]
            assert i + 1 in row
        assert abs(2 * g.m / n - d) < 1.0
        assert W.planted_matching(n, d, seed).m == g.m  # seeded
