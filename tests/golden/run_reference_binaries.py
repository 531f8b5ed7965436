"""Runs the reference's own GPU binaries (built by `make -C oracle ref` into oracle/_ref)
and writes their counts and `Time (GPU)` figures as a golden fixture.

    python tests/golden/run_reference_binaries.py [OUT.json] [--only name,name]

OUT defaults to tests/golden/ref_counts.json; entries already in OUT are kept and the
selected graphs (default: all) are run again and replaced. Edgelists of the generated
graphs are written to a temporary directory.

Graphs: the reference's toy graph and citeseer, the 2,000-vertex ER workload (seed 1), a
small R-MAT graph (ids < 2,000, 8,000 edges, seed 3; motifs up to k = 4 there, since its
5-vertex count is in the billions), the benchmark's Chung-Lu graph (18,700 vertices,
198,000 edges; cliques k = 4..7, motifs k = 3, 4) and the large skewed R-MAT graph
(~321k vertices, 1.05M edges; 7-cliques). Runs use the reference's recommended launch shape
(102400 threads, 256 per block, 16 donations) with threshold 100 (no balancing), plus
threshold-30 runs (host-mediated balancing on) on citeseer (k = 4) and on the Chung-Lu
graph (k = 4..7), and the pattern-aware queries q4..q13 (`q<n>_PA` run with k = n) on the
small graphs.

A run is only made where the reference's per-warp extension buffers provably hold every
write. Motifs: each level's buffer is nextpow2(l * max(32, dmax)) ints and a level's writes
reach index <= (l-1)*dmax + roundup32(dmax) - 1 (DuMatoCPU.cu:70-87, DuMatoGPU.cu:317-343).
Cliques and the q_n queries (pattern-aware buffers of nextpow2(max(32, dmax)) ints per
level): extend_clique, extend_single, intersect, intersect_unique and copy_extensions write at
most roundup32(size of the list they filter) <= that many entries (DuMatoGPU.cu:1028-1075,
353-434, 1194-1445), on any graph.
"""
from __future__ import annotations

import argparse
import json
import re
import subprocess
import sys
import tempfile
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

EXEC = ROOT / "oracle" / "_ref" / "exec"
ARGS = ["102400", "256", "16"]


def nextpow2(x: int) -> int:
    p = 1
    while p < x:
        p <<= 1
    return p


def motif_buffers_hold(dmax: int, k: int) -> bool:
    dr = max(32, dmax)
    r32 = (dmax + 31) // 32 * 32
    for lvl in range(0, k - 1):  # levels 0..k-2 hold (lvl+1) unions
        if lvl * dmax + r32 - 1 >= nextpow2((lvl + 1) * dr):
            return False
    return True


def run(binary: str, graph: Path, k: int, threshold: int, timeout: int = 300) -> str:
    cmd = [str(EXEC / binary), str(graph), str(k), *ARGS, str(threshold)]
    res = subprocess.run(cmd, cwd=EXEC, capture_output=True, text=True, timeout=timeout)
    if res.returncode != 0:
        raise RuntimeError(f"{cmd} failed ({res.returncode}): {res.stdout[-500:]} {res.stderr[-500:]}")
    return res.stdout


def _clique(path: Path, k: int, threshold: int) -> tuple[int, float]:
    txt = run("clique_PA", path, k, threshold, timeout=600)
    return (int(re.search(r"Result: (\d+)\.", txt).group(1)),
            float(re.search(r"Time \(GPU\): ([0-9.]+)", txt).group(1)))


def main(out_path: str, only: set | None) -> None:
    import dumato_b200 as dm
    from dumato_b200 import workloads

    work = Path(tempfile.mkdtemp(prefix="ref_graphs"))
    gen = {"er2k_s1": lambda: workloads.make("er2k", 1),
           "rmat2k_s3": lambda: dm.Graph.generate(dm.GEN_RMAT, 2000, 8000, seed=3),
           "chunglu18k_s1": lambda: workloads.make("chunglu18k", 1),
           "rmat317k_s1": lambda: workloads.make("rmat317k", 1)}
    graphs = {"test": ROOT / "tests" / "golden" / "test.edgelist",
              "citeseer": ROOT / "tests" / "golden" / "citeseer.edgelist"}
    for name in gen:
        graphs[name] = work / f"{name}.edgelist"
    clique_ks = {"chunglu18k_s1": (4, 5, 6, 7), "rmat317k_s1": (7,)}
    motif_ks = {"rmat2k_s3": (3, 4), "chunglu18k_s1": (3, 4), "rmat317k_s1": ()}
    lb_runs = {"citeseer": (4,), "chunglu18k_s1": (4, 5, 6, 7)}
    # pattern-aware queries q_n (run with k = n), on the small graphs
    near_ns = {"test": range(4, 8), "citeseer": range(4, 14), "er2k_s1": range(4, 8), "rmat2k_s3": range(4, 10)}
    out = json.loads(Path(out_path).read_text()) if Path(out_path).exists() else {}
    for name, path in graphs.items():
        if only and name not in only:
            continue
        if name in gen:
            gen[name]().write_edgelist(path)
        info = dm.Graph.load_edgelist(path).info()
        entry = {"max_degree": info.max_degree, "clique": {}, "motifs": {}, "time_gpu_s": {}}
        for k in clique_ks.get(name, (3, 4, 5, 6)):
            c, t = _clique(path, k, 100)
            entry["clique"][str(k)] = c
            entry["time_gpu_s"][f"clique{k}"] = t
        for k in motif_ks.get(name, (3, 4, 5)):
            if not motif_buffers_hold(info.max_degree, k):
                continue
            txt = run("motifs_DM_WCLB", path, k, 100, timeout=600)
            counts = {int(a): int(b) for a, b in re.findall(r"^(\d+), (\d+)$", txt, re.M)}
            total = int(re.search(r"Aggregated: (\d+),", txt).group(1))
            entry["motifs"][str(k)] = {"classes": counts, "total": total}
            entry["time_gpu_s"][f"motifs{k}"] = float(re.search(r"Time \(GPU\): ([0-9.]+)", txt).group(1))
        if name in near_ns:
            entry["near"] = {}
            for q in near_ns[name]:
                txt = run(f"q{q}_PA", path, q, 100, timeout=600)
                entry["near"][str(q)] = int(re.search(r"Result: (\d+)\.", txt).group(1))
                entry["time_gpu_s"][f"q{q}"] = float(re.search(r"Time \(GPU\): ([0-9.]+)", txt).group(1))
        if name in lb_runs:
            entry["clique_lb_threshold30"] = {}
            for k in lb_runs[name]:
                c, t = _clique(path, k, 30)
                entry["clique_lb_threshold30"][str(k)] = c
                entry["time_gpu_s"][f"clique{k}_threshold30"] = t
        out[name] = entry
        Path(out_path).parent.mkdir(parents=True, exist_ok=True)
        Path(out_path).write_text(json.dumps(out, indent=1, sort_keys=True))
        print(name, entry["clique"], {k: v["total"] for k, v in entry["motifs"].items()}, entry["time_gpu_s"],
              flush=True)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("out", nargs="?", default=str(ROOT / "tests" / "golden" / "ref_counts.json"))
    ap.add_argument("--only", default="")
    a = ap.parse_args()
    main(a.out, set(x for x in a.only.split(",") if x) or None)
