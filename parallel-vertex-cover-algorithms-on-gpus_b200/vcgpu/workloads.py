"""Seeded synthetic graph workloads and the CSR layout they share.

Graphs are undirected and simple.  The layout is the reference's CSRGraph
(src/CSRGraphRep.h:4-18): ``row_ptr`` has n+1 uint32 offsets, ``col`` holds the
2m neighbour ids (both directions of every edge) with each row sorted ascending
(the loader sorts rows at src/auxFunctions.cpp:203-206), and the degree of v is
``row_ptr[v+1] - row_ptr[v]``.

Every generator takes an explicit seed and draws only from
``numpy.random.default_rng(seed)`` (PCG64), so the same seed gives the same graph
on every machine.  The families follow the five workloads the solver is measured
on: G(n, p); a planted-cover graph with pendant paths; a batch of 4096 G(n, p)
instances of uneven size; a served stream of G(n, p) and random 3-regular
graphs; and a Chung-Lu power-law graph.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Iterable, List, Sequence, Tuple

import numpy as np


@dataclasses.dataclass
class Graph:
    n: int
    row_ptr: np.ndarray  # uint32[n+1]
    col: np.ndarray      # uint32[2m]
    name: str = ""

    @property
    def m(self) -> int:
        return int(self.col.shape[0]) // 2

    def degrees(self) -> np.ndarray:
        return np.diff(self.row_ptr.astype(np.int64)).astype(np.int32)

    def edges(self) -> np.ndarray:
        """(m, 2) array of edges u < v."""
        src = np.repeat(np.arange(self.n, dtype=np.uint32), np.diff(self.row_ptr.astype(np.int64)))
        keep = src < self.col
        return np.stack([src[keep], self.col[keep]], axis=1)


def from_edges(n: int, edges: np.ndarray, name: str = "") -> Graph:
    """CSR from an (m, 2) edge array; drops self-loops and duplicate edges."""
    e = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
    if e.size:
        if e.min() < 0 or e.max() >= n:
            raise ValueError("vertex id out of range")
        e = e[e[:, 0] != e[:, 1]]
        e = np.sort(e, axis=1)
        e = np.unique(e, axis=0)
    src = np.concatenate([e[:, 0], e[:, 1]])
    dst = np.concatenate([e[:, 1], e[:, 0]])
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    counts = np.bincount(src, minlength=n) if n else np.zeros(0, dtype=np.int64)
    row_ptr = np.zeros(n + 1, dtype=np.uint32)
    np.cumsum(counts, out=row_ptr[1:])
    return Graph(n, row_ptr, dst.astype(np.uint32), name)


def _distinct_pairs(rng: np.random.Generator, n: int, count: int) -> np.ndarray:
    """`count` distinct unordered pairs {i, j}, i != j, uniform over all pairs."""
    total = n * (n - 1) // 2
    if count > total:
        raise ValueError("more edges than pairs")
    if count == 0:
        return np.zeros((0, 2), dtype=np.int64)
    if count * 4 > total:  # dense: permute all pairs
        iu = np.triu_indices(n, 1)
        pick = rng.permutation(total)[:count]
        return np.stack([iu[0][pick], iu[1][pick]], axis=1).astype(np.int64)
    seen: dict = {}
    out: List[Tuple[int, int]] = []
    while len(out) < count:
        need = count - len(out)
        a = rng.integers(0, n, size=2 * need + 16)
        b = rng.integers(0, n, size=2 * need + 16)
        for x, y in zip(a.tolist(), b.tolist()):
            if x == y:
                continue
            key = (x, y) if x < y else (y, x)
            if key in seen:
                continue
            seen[key] = True
            out.append(key)
            if len(out) == count:
                break
    return np.asarray(out, dtype=np.int64)


def gnp(n: int, p: float, seed: int, name: str = "") -> Graph:
    """Erdos-Renyi G(n, p): the edge count is Binomial(n(n-1)/2, p), the edges a
    uniform set of that many distinct pairs (the same law as independent coins)."""
    rng = np.random.default_rng(seed)
    total = n * (n - 1) // 2
    m = int(rng.binomial(total, min(max(p, 0.0), 1.0))) if total else 0
    return from_edges(n, _distinct_pairs(rng, n, m), name or f"gnp_n{n}_p{p:.4f}_s{seed}")


def planted_matching(n: int, d: float, seed: int, name: str = "") -> Graph:
    """The pairs (2i, 2i+1) plus uniform random edges up to average degree d:
    a graph whose maximum matching is known (n // 2 pairs) and is the first one
    an in-order greedy matching finds (the MCM mode's large test graphs)."""
    rng = np.random.default_rng(seed)
    pairs = np.stack([np.arange(0, n - 1, 2), np.arange(1, n, 2)], axis=1)
    extra = _distinct_pairs(rng, n, max(0, int(n * d / 2) - len(pairs)))
    return from_edges(n, np.concatenate([pairs, extra]) if len(extra) else pairs,
                      name or f"planted_matching_n{n}_d{d}_s{seed}")


def random_regular(n: int, d: int, seed: int, name: str = "") -> Graph:
    """Uniform random d-regular simple graph by the pairing model with rejection."""
    if (n * d) % 2 or d >= n:
        raise ValueError("no d-regular graph with these sizes")
    rng = np.random.default_rng(seed)
    stubs = np.repeat(np.arange(n, dtype=np.int64), d)
    for _ in range(10000):
        perm = rng.permutation(stubs)
        e = perm.reshape(-1, 2)
        if np.any(e[:, 0] == e[:, 1]):
            continue
        s = np.sort(e, axis=1)
        if np.unique(s, axis=0).shape[0] != s.shape[0]:
            continue
        return from_edges(n, s, name or f"reg{d}_n{n}_s{seed}")
    raise RuntimeError("pairing model did not produce a simple graph")


def planted_cover(n: int = 2000, cover: int = 300, m: int = 6000, paths: int = 100,
                  max_path: int = 4, seed: int = 0) -> Graph:
    """A planted vertex cover C (|C| = cover, uniform) and m distinct uniform edges
    with at least one endpoint in C, plus `paths` pendant paths of U{1..max_path}
    new vertices each, hung from uniform vertices of the base graph (they feed the
    degree-1 and degree-2 rules)."""
    rng = np.random.default_rng(seed)
    in_c = np.zeros(n, dtype=bool)
    in_c[rng.choice(n, size=cover, replace=False)] = True
    c_ids = np.flatnonzero(in_c)
    seen = set()
    edges: List[Tuple[int, int]] = []
    while len(edges) < m:
        a = c_ids[rng.integers(0, cover, size=2 * (m - len(edges)) + 16)]
        b = rng.integers(0, n, size=a.shape[0])
        for x, y in zip(a.tolist(), b.tolist()):
            if x == y:
                continue
            key = (x, y) if x < y else (y, x)
            if key in seen:
                continue
            seen.add(key)
            edges.append(key)
            if len(edges) == m:
                break
    nxt = n
    lengths = rng.integers(1, max_path + 1, size=paths)
    anchors = rng.integers(0, n, size=paths)
    for length, anchor in zip(lengths.tolist(), anchors.tolist()):
        prev = anchor
        for _ in range(length):
            edges.append((prev, nxt))
            prev = nxt
            nxt += 1
    return from_edges(nxt, np.asarray(edges, dtype=np.int64), f"planted_n{n}_c{cover}_m{m}_s{seed}")


def chung_lu(n: int = 100000, gamma: float = 2.1, avg_deg: float = 8.0, max_deg: float = 2000.0,
             seed: int = 7) -> Graph:
    """Chung-Lu power-law graph: expected degrees w_i proportional to
    (i + i0)^(-1/(gamma-1)), scaled to mean `avg_deg` and capped at `max_deg`;
    Poisson(sum(w)/2) endpoint pairs are drawn with P(v) proportional to w_v, and
    self-loops and repeated pairs are dropped (the fast edge-sampling form)."""
    rng = np.random.default_rng(seed)
    i = np.arange(n, dtype=np.float64)
    w = (i + 1.0) ** (-1.0 / (gamma - 1.0))
    for _ in range(50):  # rescale until the capped mean matches avg_deg
        w = w * (avg_deg / np.minimum(w, max_deg).mean())
    w = np.minimum(w, max_deg)
    total = w.sum()
    pairs = int(rng.poisson(total / 2.0))
    prob = w / total
    a = rng.choice(n, size=pairs, p=prob)
    b = rng.choice(n, size=pairs, p=prob)
    perm = rng.permutation(n)  # spread hubs over ids
    e = np.stack([perm[a], perm[b]], axis=1)
    return from_edges(n, e, f"chunglu_n{n}_g{gamma}_d{avg_deg}_s{seed}")


def config1_graph() -> Graph:
    """G(n=60, p=0.1), seed 0."""
    return gnp(60, 0.1, 0, "config1_gnp_n60_p0.1_s0")


def config2_graph() -> Graph:
    """Planted cover: n=2000, |C|=300, 6000 edges touching C, 100 pendant paths."""
    return planted_cover(2000, 300, 6000, 100, 4, 0)


def batch_instance(i: int, seed: int = 0, n_lo: int = 30, n_hi: int = 200,
                   d_lo: float = 3.0, d_hi: float = 12.0) -> Graph:
    """Instance i of the batched workload: n ~ U{n_lo..n_hi}, average degree
    d ~ U[d_lo, d_hi], G(n, d/(n-1)); its own seed is derived from (seed, i)."""
    rng = np.random.default_rng([seed, i])
    n = int(rng.integers(n_lo, n_hi + 1))
    d = float(rng.uniform(d_lo, d_hi))
    return gnp(n, d / (n - 1), int(rng.integers(0, 2**63 - 1)), f"batch{seed}_{i}_n{n}_d{d:.2f}")


def batch_graphs(count: int = 4096, seed: int = 0, **kw) -> List[Graph]:
    return [batch_instance(i, seed, **kw) for i in range(count)]


def rank_batch(count: int, rank: int) -> List[Graph]:
    """The batch a rank of a multi-GPU run solves: the batched workload with the
    rank as its seed (weak scaling: every rank has its own, disjoint graphs)."""
    return batch_graphs(count, seed=rank)


def stream_instance(i: int, seed: int = 0, n_lo: int = 50, n_hi: int = 5000) -> Graph:
    """Request i of the served stream: G(n, p) with average degree U[3, 12] or a
    random 3-regular graph (equal odds), n log-uniform in [n_lo, n_hi]."""
    rng = np.random.default_rng([seed, 7919, i])
    n = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
    if rng.random() < 0.5:
        d = float(rng.uniform(3.0, 12.0))
        return gnp(n, d / (n - 1), int(rng.integers(0, 2**63 - 1)), f"stream{seed}_{i}_gnp_n{n}_d{d:.2f}")
    n += n % 2
    return random_regular(n, 3, int(rng.integers(0, 2**63 - 1)), f"stream{seed}_{i}_reg3_n{n}")


@dataclasses.dataclass
class Arena:
    """Many graphs packed for one batched call: instance i's n_i+1 local row
    offsets start at row_ptr[row_off[i]] and its neighbour ids at col[col_off[i]]."""
    n: np.ndarray        # uint32[count]
    row_off: np.ndarray  # uint64[count]
    col_off: np.ndarray  # uint64[count]
    row_ptr: np.ndarray  # uint32[sum(n_i + 1)]
    col: np.ndarray      # uint32[sum(2 m_i)]

    @property
    def count(self) -> int:
        return int(self.n.shape[0])


def pack(graphs: Sequence[Graph]) -> Arena:
    n = np.asarray([g.n for g in graphs], dtype=np.uint32)
    rows = np.asarray([g.n + 1 for g in graphs], dtype=np.uint64)
    cols = np.asarray([g.col.shape[0] for g in graphs], dtype=np.uint64)
    row_off = np.zeros(len(graphs), dtype=np.uint64)
    col_off = np.zeros(len(graphs), dtype=np.uint64)
    if len(graphs) > 1:
        np.cumsum(rows[:-1], out=row_off[1:])
        np.cumsum(cols[:-1], out=col_off[1:])
    row_ptr = np.concatenate([g.row_ptr for g in graphs]).astype(np.uint32) if graphs else np.zeros(0, np.uint32)
    col = np.concatenate([g.col for g in graphs]).astype(np.uint32) if graphs else np.zeros(0, np.uint32)
    return Arena(n, row_off, col_off, row_ptr, col)


def read_reference_file(path: str, one_based: bool = True) -> Graph:
    """Reads the reference's text format: a header "n m", then m lines "u v"
    (1-based ids, shifted down by one as src/auxFunctions.cpp:150-154 does; with
    one_based=False the ids are taken as they are, the CLI's -z).  A path ending
    in .gz is read through gzip."""
    import gzip
    with (gzip.open(path, "rt") if path.endswith(".gz") else open(path, "r")) as f:
        data = np.array(f.read().split(), dtype=np.int64)
    n, m = int(data[0]), int(data[1])
    e = data[2:2 + 2 * m].reshape(m, 2)
    if one_based:
        e = e - 1
    return from_edges(n, e, path.rsplit("/", 1)[-1])


def write_reference_file(g: Graph, path: str) -> None:
    e = g.edges().astype(np.int64) + 1
    with open(path, "w") as f:
        f.write(f"{g.n} {g.m}\n")
        if e.size:
            np.savetxt(f, e, fmt="%d")


def is_cover(g: Graph, mask: Iterable) -> bool:
    """Edge-by-edge check that `mask` (n booleans) covers every edge."""
    mk = np.asarray(mask, dtype=bool)
    e = g.edges()
    return bool(np.all(mk[e[:, 0]] | mk[e[:, 1]])) if e.size else True
