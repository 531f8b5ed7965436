"""The C ABI library loads and exports every entry point of include/dumato_b200.h (CPU)."""
from __future__ import annotations

import re
import subprocess

from conftest import ROOT


def declared_symbols():
    text = (ROOT / "include" / "dumato_b200.h").read_text()
    return re.findall(r"^DM_API [^(]*?\b(dm_\w+)\s*\(", text, re.M)


def test_header_symbols_exported(dm):
    names = declared_symbols()
    assert len(names) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", str(dm.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (dm_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    lib = dm.lib()
    for n in names:
        getattr(lib, n)


def test_binding_covers_header(dm):
    assert set(declared_symbols()) <= set(dm.exported_symbols())


def test_counting_without_device_reports_status(dm):
    if dm.device_count() > 0:
        return
    g = dm.Graph.load_edgelist(ROOT / "tests" / "golden" / "test.edgelist")
    try:
        dm.count_cliques(g, 3)
    except dm.DMError as e:
        assert e.status == -5
    else:
        raise AssertionError("counting must fail without a device (no CPU path)")


def test_bad_arguments(dm):
    g = dm.Graph.load_edgelist(ROOT / "tests" / "golden" / "test.edgelist")
    for k in (1, 13):
        try:
            dm.count_cliques(g, k)
        except dm.DMError as e:
            assert e.status in (-1, -5)
        else:
            raise AssertionError
    assert dm.lib().dm_abi_version() == 2
