"""The public GPM step library (include/dumato_b200_gpm.cuh): it compiles on its own for
sm_100a (CPU test), and its self-test program matches host results on a GPU."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "gpm" / "gpm_selftest.cu"


def _nvcc():
    for c in ("/usr/local/cuda/bin/nvcc", "nvcc"):
        if c == "nvcc" or Path(c).exists():
            return c
    return "nvcc"


def _build(tmp: Path) -> Path:
    exe = tmp / "gpm_selftest"
    cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17",
           "--extended-lambda", "-I", str(ROOT / "include"), "-o", str(exe), str(SRC)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    return exe


def test_gpm_header_compiles_standalone(tmp_path):
    assert _build(tmp_path).exists()


@pytest.mark.gpu
def test_gpm_selftest_on_gpu(tmp_path, gpu):
    exe = _build(tmp_path)
    res = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0 and "gpm selftest ok" in res.stdout, res.stdout + res.stderr
