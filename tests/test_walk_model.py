"""CPU model of the index kernel's counting rules (no GPU): the lockstep walk of
`clique.cuh` (`WalkR`, `lockstep_items`) and the item space of batched small roots
(`clique_cached.cuh` `BatchItems`), restated in Python over per-root local bitmaps and
checked against the oracle's clique counts.

The walk: stack entry j holds the candidates for clique vertex 4 + j of an item (the root, c1
and c2 being vertices 1..3); one step pops the lowest member x of the top set and forms
T = rest & row[x]. Fused counts add |T| to the count of size 5 + j; one size K adds |T| at
the last entry only and keeps a set only while it can still complete a K-clique. Lanes take
items together once REFILL_MIN of them are idle, and an item with 24 or more candidates (k >= 6)
is deferred to the whole warp, which spreads the candidates over the lanes."""
from __future__ import annotations

import bisect

import numpy as np
import pytest

from conftest import GOLDEN

HEAVY_BITS, HEAVY_SLOTS, REFILL_MIN, LANES = 24, 32, 8, 32


def pc(x: int) -> int:
    return bin(x).count("1")


class Walk:
    def __init__(self, K, multi, lev0, acc):
        self.K, self.multi, self.lev0, self.acc = K, multi, lev0, acc
        self.cur, self.stack, self.cnt = 0, [], 0   # stack: entries below the top (j, set)
        self.top = -1

    def start(self, S):
        p = pc(S)
        K, L = self.K, self.lev0
        if self.multi:
            self.acc[L] += p
            go = L < K and p >= 2
        else:
            if L == K:
                self.cnt += p
            go = L < K and p >= K - L + 1
        if go:
            self.cur, self.top, self.stack = S, 0, []

    def step(self, rows):
        K, L, j = self.K, self.lev0, self.top
        low = self.cur & -self.cur
        x = low.bit_length() - 1
        rest = self.cur ^ low
        T = rest & rows[x]
        p = pc(T)
        if self.multi:
            self.acc[L + j + 1] += p
            push = L + j + 1 < K and p >= 2
        else:
            if L + j + 1 == K:
                self.cnt += p
            push = L + j + 1 < K and p >= K - L - j
            if pc(rest) <= K - L - j:
                rest = 0
        if push:
            if rest:
                self.stack.append((j, rest))
            self.cur, self.top = T, j + 1
        elif rest:
            self.cur = rest
        elif self.stack:
            self.top, self.cur = self.stack.pop()
        else:
            self.top = -1


def lockstep(walks, start_item, n_items, rows_of):
    nxt = 0
    while True:
        idle = [w.top < 0 for w in walks]
        if nxt < n_items and any(idle) and (all(idle) or sum(idle) >= REFILL_MIN):
            for i, w in enumerate(walks):
                if idle[i] and nxt < n_items:
                    start_item(i, nxt)
                    nxt += 1
        if all(w.top < 0 for w in walks):
            if nxt >= n_items:
                return
            continue
        for w in walks:
            if w.top >= 0:
                w.step(rows_of(w))


def dag_roots(u, v, n):
    """Local bitmap rows of every root of the (degree, id)-ordered DAG with >= 2 out-neighbours."""
    deg = np.bincount(np.concatenate([u, v]), minlength=n)
    rank = np.empty(n, np.int64)
    rank[np.lexsort((np.arange(n), deg))] = np.arange(n)
    out = [[] for _ in range(n)]
    for x, y in zip(u, v):
        a, b = (x, y) if rank[x] < rank[y] else (y, x)
        out[a].append(b)
    outs = [sorted(o, key=lambda z: rank[z]) for o in out]
    for r in range(n):
        nb = outs[r]
        if len(nb) < 2:
            continue
        pos = {x: i for i, x in enumerate(nb)}
        yield [sum(1 << pos[y] for y in outs[x] if y in pos) for x in nb]


def count_root(rows, K, multi):
    """One root's counts: the item loop, then the deferred heavy items' positions."""
    d = len(rows)
    acc = [0] * (K + 1)
    items = [(c1, b) for c1 in range(d) for b in range(d) if rows[c1] >> b & 1]
    heavy = []
    walks = [Walk(K, multi, 4, acc) for _ in range(LANES)]

    def start_item(lane, i):
        c1, c2 = items[i]
        if multi:
            acc[3] += 1
        S = rows[c1] & rows[c2]
        if K >= 6 and pc(S) >= HEAVY_BITS and len(heavy) < HEAVY_SLOTS:
            heavy.append(S)
            if multi:
                acc[4] += pc(S)
            return
        walks[lane].start(S)

    lockstep(walks, start_item, len(items), lambda w: rows)
    total = sum(w.cnt for w in walks)
    for S in heavy:
        members = [b for b in range(d) if S >> b & 1]
        hw = [Walk(K, multi, 5, acc) for _ in range(LANES)]

        def start_pos(lane, j, S=S, members=members, hw=hw):
            c3 = members[j]
            hw[lane].start((S >> (c3 + 1) << (c3 + 1)) & rows[c3])

        lockstep(hw, start_pos, len(members), lambda w: rows)
        total += sum(w.cnt for w in hw)
    return acc, total


def model_counts(u, v, n, K):
    fused = [0] * (K + 1)
    single = 0
    for rows in dag_roots(u, v, n):
        acc, _ = count_root(rows, K, True)
        fused = [a + b for a, b in zip(fused, acc)]
        single += count_root(rows, K, False)[1]
    return {k: fused[k] for k in range(3, K + 1)}, single


def dense_core(seed=3, core=60, n=800, extra=3000, p=0.8):
    rng = np.random.default_rng(seed)
    ids = rng.choice(n, core, replace=False)
    iu = np.triu_indices(core, 1)
    keep = rng.random(iu[0].size) < p
    s = np.concatenate([ids[iu[0][keep]], rng.integers(0, n, extra)])
    t = np.concatenate([ids[iu[1][keep]], rng.integers(0, n, extra)])
    m = s != t
    a, b = np.minimum(s[m], t[m]), np.maximum(s[m], t[m])
    pairs = np.unique(np.stack([a, b], 1), axis=0)
    return pairs[:, 0], pairs[:, 1], n


@pytest.mark.parametrize("K", [4, 5, 6, 7, 8])
def test_walk_model_citeseer(dm, orc, K):
    g = dm.Graph.load_edgelist(GOLDEN / "citeseer.edgelist")  # host-side reader, no GPU
    u, v = g.edges()
    og = orc.OracleGraph.from_pairs(u, v)
    want = {k: orc.clique_dag_bytes(og, k)[0] for k in range(3, K + 1)}
    fused, single = model_counts(np.asarray(u), np.asarray(v), g.info().n_vertices, K)
    assert fused == want and single == want[K]


@pytest.mark.parametrize("K", [6, 7, 8])
def test_walk_model_dense_core_heavy_items(orc, K):
    """A 60-vertex core of density 0.8: items with 24+ candidates take the deferred path."""
    u, v, n = dense_core()
    og = orc.OracleGraph.from_pairs(u, v)
    want = {k: orc.clique_dag_bytes(og, k)[0] for k in range(3, K + 1)}
    fused, single = model_counts(u, v, n, K)
    assert fused == want and single == want[K]


def test_batch_item_space_maps_every_edge_once():
    """BatchItems: item g -> (entry, row c1, bit c2) through the entries' item offsets and
    the exclusive popcount prefix E of every staged word (rows of one word, blocks padded to
    two words, entries that are not batched holding no items)."""
    rng = np.random.default_rng(5)
    for _ in range(200):
        ne = int(rng.integers(2, 17))
        ds = [int(rng.choice([2, 3, 5, 9, 17, 33, 64])) for _ in range(ne)]
        batched = [bool(rng.random() < 0.8) for _ in range(ne)]
        words, base = [], []
        for d in ds:
            base.append(len(words))
            rows = [sum(1 << j for j in range(i + 1, d) if rng.random() < 0.3) for i in range(d)]
            words += rows + [0] * (d % 2)
        E = [0]
        for w in words:
            E.append(E[-1] + pc(w))
        n_items = [E[base[i] + ds[i]] - E[base[i]] if batched[i] else 0 for i in range(ne)]
        O = [0]
        for m in n_items:
            O.append(O[-1] + m)
        got = []
        for g in range(O[-1]):
            j = bisect.bisect_right(O, g) - 1
            e = g - O[j]
            target = E[base[j]] + e
            r = bisect.bisect_right(E, target, base[j], base[j] + ds[j] + 1) - 1
            bits = [b for b in range(64) if words[r] >> b & 1]
            got.append((j, r - base[j], bits[target - E[r]]))
        want = [(i, c1, b) for i in range(ne) if batched[i] for c1 in range(ds[i])
                for b in range(64) if words[base[i] + c1] >> b & 1]
        assert got == want
