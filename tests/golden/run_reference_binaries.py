"""Runs the reference's own GPU binaries (built by `make -C oracle ref` into oracle/_ref)
on small graphs and writes their counts as a golden fixture (default
gpurun_out/ref_counts.json; copy it to tests/golden/ref_counts.json).

Graphs: the reference's toy graph and citeseer, the 2,000-vertex ER workload (seed 1) and a
small R-MAT graph (ids < 2,000, 8,000 edges, seed 3; motifs up to k = 4 there, since its
5-vertex count is in the billions). Runs use the reference's recommended launch shape
(102400 threads, 256 per block, 16 donations) with threshold 100 (no balancing), plus one
citeseer run with threshold 30 (host-mediated balancing on).

A run is only made where the reference's per-warp extension buffers provably hold every
write: each level's buffer is nextpow2(l * max(32, dmax)) ints and a level's writes reach
index <= (l-1)*dmax + roundup32(dmax) - 1 (DuMatoCPU.cu:70-87, DuMatoGPU.cu:317-343).
"""
from __future__ import annotations

import json
import re
import subprocess
import sys
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


def run(binary: str, graph: Path, k: int, threshold: int) -> str:
    cmd = [str(EXEC / binary), str(graph), str(k), *ARGS, str(threshold)]
    res = subprocess.run(cmd, cwd=EXEC, capture_output=True, text=True, timeout=300)
    if res.returncode != 0:
        raise RuntimeError(f"{cmd} failed ({res.returncode}): {res.stdout[-500:]} {res.stderr[-500:]}")
    return res.stdout


def main(out_path: str) -> None:
    import dumato_b200 as dm
    from dumato_b200 import workloads

    work = ROOT / "gpurun_out" / "ref_graphs"
    work.mkdir(parents=True, exist_ok=True)
    graphs = {"test": ROOT / "tests" / "golden" / "test.edgelist",
              "citeseer": ROOT / "tests" / "golden" / "citeseer.edgelist"}
    g = workloads.make("er2k", 1)
    g.write_edgelist(work / "er2k_s1.edgelist")
    graphs["er2k_s1"] = work / "er2k_s1.edgelist"
    g = dm.Graph.generate(dm.GEN_RMAT, 2000, 8000, seed=3)
    g.write_edgelist(work / "rmat2k_s3.edgelist")
    graphs["rmat2k_s3"] = work / "rmat2k_s3.edgelist"
    max_motif_k = {"rmat2k_s3": 4}
    out = {}
    for name, path in graphs.items():
        info = dm.Graph.load_edgelist(path).info()
        entry = {"max_degree": info.max_degree, "clique": {}, "motifs": {}, "time_gpu_s": {}}
        for k in (3, 4, 5, 6):
            txt = run("clique_PA", path, k, 100)
            entry["clique"][str(k)] = int(re.search(r"Result: (\d+)\.", txt).group(1))
            entry["time_gpu_s"][f"clique{k}"] = float(re.search(r"Time \(GPU\): ([0-9.]+)", txt).group(1))
        for k in (3, 4, 5):
            if k > max_motif_k.get(name, 5) or not motif_buffers_hold(info.max_degree, k):
                continue
            txt = run("motifs_DM_WCLB", path, k, 100)
            counts = {int(a): int(b) for a, b in re.findall(r"^(\d+), (\d+)$", txt, re.M)}
            total = int(re.search(r"Aggregated: (\d+),", txt).group(1))
            entry["motifs"][str(k)] = {"classes": counts, "total": total}
            entry["time_gpu_s"][f"motifs{k}"] = float(re.search(r"Time \(GPU\): ([0-9.]+)", txt).group(1))
        out[name] = entry
        print(name, entry["clique"], {k: v["total"] for k, v in entry["motifs"].items()}, flush=True)
    txt = run("clique_PA", graphs["citeseer"], 4, 30)
    out["citeseer"]["clique_lb_threshold30"] = {"4": int(re.search(r"Result: (\d+)\.", txt).group(1))}
    Path(out_path).parent.mkdir(parents=True, exist_ok=True)
    Path(out_path).write_text(json.dumps(out, indent=1, sort_keys=True))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else str(ROOT / "gpurun_out" / "ref_counts.json"))
