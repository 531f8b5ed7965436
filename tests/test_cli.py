"""Drop-in executables: argument handling (CPU) and output lines against the reference's
own printed results (GPU)."""
from __future__ import annotations

import json
import re
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

BIN = ROOT / "dumato_b200" / "bin"


def run(args, cwd=None):
    return subprocess.run([str(a) for a in args], capture_output=True, text=True, cwd=cwd, timeout=600)


@pytest.mark.parametrize("exe", ["clique", "motifs", "near_clique"])
def test_wrong_argument_count(dm, exe):
    r = run([BIN / exe, GOLDEN / "test.edgelist", 3])
    assert r.returncode == 1 and "Wrong amount of parameters!" in r.stdout


def test_missing_graph_file(dm, tmp_path):
    r = run([BIN / "clique", tmp_path / "none.edgelist", 3, 102400, 256, 16, 30])
    assert r.returncode == 1 and "reading the graph" in r.stderr


def _ref():
    return json.loads((GOLDEN / "ref_counts.json").read_text())


@pytest.mark.gpu
@pytest.mark.parametrize("k", [3, 4, 5, 6])
def test_clique_result_line(dm, gpu, k):
    r = run([BIN / "clique", GOLDEN / "citeseer.edgelist", k, 102400, 256, 16, 30])
    assert r.returncode == 0, r.stderr
    assert f"Result: {_ref()['citeseer']['clique'][str(k)]}." in r.stdout
    assert re.search(r"^Time \(GPU\): [0-9.]+ secs\.$", r.stdout, re.M)


@pytest.mark.gpu
@pytest.mark.parametrize("k", [3, 4, 5])
def test_motifs_lines_with_reference_dictionary(dm, gpu, tmp_path, k):
    # the reference layout: run from exec/, tables in ../dictionaries/<k>.csv
    (tmp_path / "exec").mkdir()
    (tmp_path / "dictionaries").mkdir()
    z = np.load(GOLDEN / f"ref_dict_{k}.npz")
    q, c = z["quick_to_class"], z["class_code"]
    with open(tmp_path / "dictionaries" / f"{k}.csv", "w") as f:
        f.write(f"#quick,cg_local\n{q.size}\n" + "".join(f"{i},{x}\n" for i, x in enumerate(q)))
        f.write(f"#cg_local,cg_global\n{c.size}\n" + "".join(f"{i},{int(x)}\n" for i, x in enumerate(c)))
    r = run([BIN / "motifs", GOLDEN / "citeseer.edgelist", k, 102400, 256, 16, 100], cwd=tmp_path / "exec")
    assert r.returncode == 0, r.stderr
    ref = _ref()["citeseer"]["motifs"][str(k)]
    lines = re.findall(r"^(\d+), (\d+)$", r.stdout, re.M)
    assert {int(a): int(b) for a, b in lines} == {int(a): b for a, b in ref["classes"].items()}
    assert f"Aggregated: {ref['total']}, {len(ref['classes'])} patterns." in r.stdout


@pytest.mark.gpu
def test_motifs_without_dictionary_file_generates_one(dm, gpu, tmp_path):
    r = run([BIN / "motifs", GOLDEN / "test.edgelist", 4, 0, 256, 16, 30], cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    assert "Aggregated: 4, 3 patterns." in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("q", [4, 5, 6])
def test_near_clique_result_line(dm, orc, gpu, q):
    """`near_clique graph k ...` prints the count of the reference's q<k>_PA."""
    r = run([BIN / "near_clique", GOLDEN / "citeseer.edgelist", q, 102400, 256, 16, 30])
    assert r.returncode == 0, r.stderr
    og = orc.OracleGraph.load(GOLDEN / "citeseer.edgelist")
    assert f"Result: {orc.near_cliques(og, q)}." in r.stdout
