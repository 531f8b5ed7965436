"""Writes tests/golden/ref_dict_<k>.npz from the DuMato dictionaries (dictionaries/<k>.csv,
k = 3..6): quick -> cg_local (int32) and cg_local -> cg_global (uint64). Run where the
DuMato sources are available:

    python tests/golden/make_dictionary_fixtures.py /path/to/DuMato
    DUMATO_REF_ROOT=/path/to/DuMato python tests/golden/make_dictionary_fixtures.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np


def read_csv(path: Path):
    tok = path.read_text().split()
    i = 1
    nq = int(tok[i]); i += 1
    q2c = np.full(nq, -1, np.int32)
    for _ in range(nq):
        q, c = tok[i].split(","); i += 1
        q2c[int(q)] = int(c)
    i += 1  # header
    nc = int(tok[i]); i += 1
    code = np.zeros(nc, np.uint64)
    for _ in range(nc):
        c, g = tok[i].split(","); i += 1
        code[int(c)] = int(g)
    return q2c, code


def main(root: str) -> None:
    out = Path(__file__).resolve().parent
    for k in (3, 4, 5, 6):
        q2c, code = read_csv(Path(root) / "dictionaries" / f"{k}.csv")
        np.savez_compressed(out / f"ref_dict_{k}.npz", quick_to_class=q2c, class_code=code)
        print(k, q2c.size, code.size)


if __name__ == "__main__":
    import os

    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DUMATO_REF_ROOT")
    if not root:
        sys.exit("usage: make_dictionary_fixtures.py /path/to/DuMato (or set DUMATO_REF_ROOT)")
    main(root)
