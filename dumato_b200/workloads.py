"""Seeded synthetic workloads standing in for the benchmark datasets (sizes from the
five benchmark configurations). Generator parameters are fixed here so tests, bench and
fixtures agree on the exact graphs."""
from __future__ import annotations

CONFIGS = {
    # Erdos-Renyi G(n, m): 2,000 vertices, 10,000 undirected edges
    "er2k": dict(kind=0, n=2000, m=10_000),
    # Chung-Lu power law: ~18,700 vertices, ~198,000 edges, exponent 2.1, max degree ~500
    "chunglu18k": dict(kind=1, n=18_700, m=198_000, gamma=2.1, dmax=500.0),
    # R-MAT (.57,.19,.19,.05): ids < 170,000 -> ~98.6k touched vertices, 1.08M edges
    "rmat100k": dict(kind=2, n=170_000, m=1_080_000, a=0.57, b=0.19, c=0.19),
    # R-MAT (.57,.19,.19,.05): ids < 1,400,000 -> ~321k touched vertices, 1.05M edges
    "rmat317k": dict(kind=2, n=1_400_000, m=1_050_000, a=0.57, b=0.19, c=0.19),
}


def make(name: str, seed: int = 1):
    """Generates the named workload graph (deterministic for a given seed)."""
    from . import Graph

    p = dict(CONFIGS[name])
    kind = p.pop("kind")
    return Graph.generate(kind, p.pop("n"), p.pop("m"), seed=seed, **p)


# Batched-mining workload: graphs of uneven size, one query each.
BATCH_QUERIES = [("clique", 3), ("clique", 4), ("clique", 5), ("clique", 6), ("motif", 3), ("motif", 4), ("motif", 5)]


def batch_specs(seed: int = 1, n_graphs: int = 256) -> list[dict]:
    """Parameters of the batched workload: per graph a Chung-Lu generator setting with
    V ~ U[50, 5000], average degree ~ U[4, 40] (clipped to (V-1)/4 so small graphs stay
    sparse enough to draw), exponent ~ U[2.0, 2.5], weight cap min(V-1, 10 x average degree),
    a seed per graph, and a query drawn uniformly from k-cliques k = 3..6 and motifs k = 3..5."""
    import numpy as np

    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_graphs):
        n = int(rng.integers(50, 5001))
        avg = float(min(rng.uniform(4.0, 40.0), (n - 1) / 4.0))
        gamma = float(rng.uniform(2.0, 2.5))
        kind, k = BATCH_QUERIES[int(rng.integers(0, len(BATCH_QUERIES)))]
        out.append(dict(n=n, m=int(round(n * avg / 2)), gamma=gamma, dmax=float(min(n - 1, 10.0 * avg)),
                        seed=seed * 100_003 + i, query=kind, k=k))
    return out


def make_batch(seed: int = 1, n_graphs: int = 256):
    """The batched workload as (queries, graphs, dictionaries): Query objects ready for Batch."""
    from . import GEN_CHUNG_LU, QUERY_CLIQUE, QUERY_MOTIF, Dictionary, Graph, Query

    dicts = {}
    queries, graphs = [], []
    for s in batch_specs(seed, n_graphs):
        g = Graph.generate(GEN_CHUNG_LU, s["n"], s["m"], seed=s["seed"], gamma=s["gamma"], dmax=s["dmax"])
        graphs.append(g)
        if s["query"] == "clique":
            queries.append(Query(QUERY_CLIQUE, s["k"], g))
        else:
            if s["k"] not in dicts:
                dicts[s["k"]] = Dictionary.generate(s["k"])
            queries.append(Query(QUERY_MOTIF, s["k"], g, dicts[s["k"]]))
    return queries, graphs, dicts


def main(argv=None) -> int:
    """Runs one query on a named workload `reps` times and prints the last run's count and
    kernel time (the command line the kernel profiles are taken with); `upto` counts every
    clique size 3..k in one launch; `batch` runs the batched workload instead."""
    import argparse

    from . import Batch, Dictionary, count_cliques, count_cliques_upto, count_motifs

    ap = argparse.ArgumentParser(prog="python -m dumato_b200.workloads")
    ap.add_argument("query", choices=("clique", "upto", "motif", "batch"))
    ap.add_argument("workload", nargs="?", default="chunglu18k", choices=sorted(CONFIGS))
    ap.add_argument("k", type=int, nargs="?", default=4)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--graphs", type=int, default=256, help="batch: number of graphs")
    args = ap.parse_args(argv)
    if args.query == "batch":
        queries, _graphs, _dicts = make_batch(args.seed, args.graphs)
        b = Batch(queries)
        for _ in range(max(1, args.reps)):
            res, st = b.run()
        total = sum(int(r) if isinstance(r, int) else int(r.sum()) for r in res)
        print(f"batch of {len(queries)} queries: {total} subgraphs in {st.kernel_ms:.3f} ms "
              f"(tasks {st.tasks}, donations {st.donations})")
        return 0
    g = make(args.workload, args.seed)
    if args.query == "upto":
        for _ in range(max(1, args.reps)):
            counts, st = count_cliques_upto(g, args.k)
        print(f"cliques of sizes 3..{args.k} on {args.workload}: {counts} in {st.kernel_ms:.3f} ms "
              f"(one launch; tasks {st.tasks}, donations {st.donations})")
        return 0
    d = Dictionary.generate(args.k) if args.query == "motif" else None
    for _ in range(max(1, args.reps)):
        if d is None:
            total, st = count_cliques(g, args.k)
        else:
            hist, st = count_motifs(g, args.k, d)
            total = int(hist.sum())
    print(f"{args.query} {args.workload} k={args.k}: {total} in {st.kernel_ms:.3f} ms "
          f"(tasks {st.tasks}, donations {st.donations}, prefix donations {st.prefix_donations})")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
