"""Self-generated canonical dictionaries against the reference's tables (CPU)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN

CLASSES = {3: 3, 4: 10, 5: 33, 6: 155, 7: 1043}
CONNECTED = {3: 2, 4: 6, 5: 21, 6: 112, 7: 853}


def ref_tables(k):
    z = np.load(GOLDEN / f"ref_dict_{k}.npz")
    return z["quick_to_class"], z["class_code"]


@pytest.mark.parametrize("k", [3, 4, 5, 6, 7])
def test_class_and_connected_counts(dm, k):
    d = dm.Dictionary.generate(k)
    kk, nq, nc = d.shape()
    assert (kk, nq, nc) == (k, 2 ** (k * (k - 1) // 2 - 1), CLASSES[k])
    assert int(d.connected().sum()) == CONNECTED[k]


@pytest.mark.parametrize("k", [3, 4, 5, 6])
def test_partition_matches_reference(dm, k):
    q2c, _ = dm.Dictionary.generate(k).tables()
    rq2c, _ = ref_tables(k)
    # same partition of quick codes: the class maps are a bijection
    pairs = set(zip(q2c.tolist(), rq2c.tolist()))
    assert len(pairs) == CLASSES[k]
    assert len({a for a, _ in pairs}) == len({b for _, b in pairs}) == CLASSES[k]


@pytest.mark.parametrize("k", [3, 4])
def test_small_tables_identical_to_reference(dm, k):
    q2c, code = dm.Dictionary.generate(k).tables()
    rq2c, rcode = ref_tables(k)
    assert np.array_equal(q2c, rq2c) and np.array_equal(code, rcode)


def write_reference_csv(path, q2c, code):
    with open(path, "w") as f:
        f.write(f"#quick,cg_local\n{q2c.size}\n")
        for q, c in enumerate(q2c):
            f.write(f"{q},{c}\n")
        f.write(f"#cg_local,cg_global\n{code.size}\n")
        for c, g in enumerate(code):
            f.write(f"{c},{int(g)}\n")


@pytest.mark.parametrize("k", [3, 5, 6])
def test_loads_reference_format(dm, tmp_path, k):
    rq2c, rcode = ref_tables(k)
    p = tmp_path / f"{k}.csv"
    write_reference_csv(p, rq2c, rcode)
    d = dm.Dictionary.load_csv(p)
    q2c, code = d.tables()
    assert np.array_equal(q2c, rq2c) and np.array_equal(code, rcode)


@pytest.mark.parametrize("k", [4, 7])
def test_csv_round_trip(dm, tmp_path, k):
    d = dm.Dictionary.generate(k)
    p = tmp_path / "d.csv"
    d.write_csv(p)
    e = dm.Dictionary.load_csv(p)
    for a, b in zip(d.tables(), e.tables()):
        assert np.array_equal(a, b)


def test_malformed_dictionary_rejected(dm, tmp_path):
    p = tmp_path / "bad.csv"
    p.write_text("#quick,cg_local\n5\n0,0\n")
    with pytest.raises(dm.DMError) as e:
        dm.Dictionary.load_csv(p)
    assert e.value.status == -3
    with pytest.raises(dm.DMError) as e:
        dm.Dictionary.load_csv(tmp_path / "missing.csv")
    assert e.value.status == -2
