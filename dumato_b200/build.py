"""Builds libdmb200.so (host C++ + sm_100a CUDA kernels) and the drop-in executables.

Everything is compiled in-tree with nvcc for sm_100a only; the CUDA runtime is linked
statically so the library loads with nothing but the driver on the machine.

    python -m dumato_b200.build            # library + bin/clique + bin/motifs
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libdmb200.so"
BIN = PKG / "bin"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "-I", str(PKG.parent / "include"), "-I", str(CSRC)]
LIB_SOURCES = ["graph.cpp", "dictionary.cpp", "engine.cu", "clique.cu", "clique_k7_8.cu", "clique_k9.cu",
               "clique_k10.cu", "clique_k11.cu", "clique_k12.cu", "motif.cu", "predictor.cu", "noalloc.cu", "batch.cu", "ingest.cu", "near_clique.cu"]
CLI_SOURCES = {"clique": "cli_clique.cpp", "motifs": "cli_motifs.cpp", "near_clique": "cli_near_clique.cpp"}


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ... ({res.returncode})")
    if verbose and (res.stdout or res.stderr):
        print(res.stdout + res.stderr)


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build(verbose: bool = False, ptxas_info: bool = False) -> Path:
    headers = list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + list((PKG.parent / "include").glob("*.h*"))
    sources = [CSRC / s for s in LIB_SOURCES] + [CSRC / s for s in CLI_SOURCES.values()]
    # a library and executables newer than every source need no object files (a copy of the
    # tree that carries only the built outputs)
    if not ptxas_info and not _stale(LIB, sources + headers) and \
            all(not _stale(BIN / name, [LIB, CSRC / src] + headers) for name, src in CLI_SOURCES.items()):
        return LIB
    BUILD.mkdir(exist_ok=True)
    BIN.mkdir(exist_ok=True)
    nvcc = _nvcc()
    objs = []
    jobs = []
    for src in LIB_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers) or ptxas_info:
            cmd = [nvcc, *ARCH, *COMMON, "-c", str(s), "-o", str(o)]
            if src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"] if ptxas_info else []
            else:
                cmd = [nvcc, *COMMON, "-x", "c++", "-Xcompiler", "-O3", "-c", str(s), "-o", str(o)]
            jobs.append(cmd)
    procs = []
    for cmd in jobs:
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = None
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed = (cmd, out)
        elif (verbose or ptxas_info) and out:
            print(out)
    if failed:
        sys.stderr.write(failed[1])
        raise RuntimeError(f"compile failed: {failed[0][-3]}")
    if _stale(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs),
              "-Xlinker", "-z,defs", "-lpthread", "-ldl", "-lrt"], verbose)
    for name, src in CLI_SOURCES.items():
        s = CSRC / src
        exe = BIN / name
        if _stale(exe, [s, LIB] + headers):
            _run([nvcc, *COMMON, "-x", "c++", "-o", str(exe), str(s), "-L", str(PKG), "-ldmb200",
                  "-Xlinker", "-rpath,$ORIGIN/..", "-lpthread"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
