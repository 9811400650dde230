"""Build recipe for the native parts of gstore_b200 (in-tree outputs).

* ``lib/libgstore_cuda.so`` — the sm_100a engine behind ``include/gstore_cuda.h``
* ``lib/gstoreu`` / ``lib/gstored`` — the reference-compatible command line
  (undirected half grid / directed full grid), linked against the engine.

Run ``python -m gstore_b200.build``.  nvcc cross-compiles for sm_100a without
a GPU, so this works on a build host too.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
HOST = CSRC / "host"
LIB = PKG / "lib"
INCLUDE = ROOT / "include"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_SOURCES = ["gs_api.cu", "gs_sweep.cu", "gs_bfs.cu", "gs_gen.cu", "gs_convert.cu", "gs_noalloc.cu",
                "gs_stream.cu", "gs_batch.cu",
                "gs_serve.cu", "gs_pagerank.cu", "gs_pr_blocked.cu", "gs_files.cpp"]
HOST_SOURCES = ["gstore_main.cpp", "tilefile.cpp", "algo.cpp"]


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd, quiet):
    if not quiet:
        print(" ".join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def build_engine(quiet: bool = True, force: bool = False) -> Path:
    LIB.mkdir(exist_ok=True)
    out = LIB / "libgstore_cuda.so"
    deps = [CSRC / s for s in CUDA_SOURCES] + list(CSRC.glob("*.cuh")) + [INCLUDE / "gstore_cuda.h"]
    if force or _stale(out, deps):
        _run([NVCC, "-std=c++17", "-O3", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-shared",
              "-I", INCLUDE, "-I", CSRC, "-o", out, *[CSRC / s for s in CUDA_SOURCES]], quiet)
    return out


def build_host(quiet: bool = True, force: bool = False):
    """gstoreu (HALF_GRID) and gstored (directed) — the reference's two binaries."""
    srcs = [HOST / s for s in HOST_SOURCES if (HOST / s).exists()]
    if not srcs:
        return []
    outs = []
    deps = srcs + list(HOST.glob("*.h")) + [INCLUDE / "gstore_cuda.h", LIB / "libgstore_cuda.so"]
    for name, flags in (("gstoreu", ["-DHALF_GRID"]), ("gstored", [])):
        out = LIB / name
        if force or _stale(out, deps):
            _run(["/usr/bin/g++", "-std=c++17", "-O2", *flags, "-I", INCLUDE, "-I", HOST, *srcs,
                  "-L", LIB, "-lgstore_cuda", "-Wl,-rpath,$ORIGIN", "-lpthread", "-o", out], quiet)
        outs.append(out)
    return outs


def build(quiet: bool = True, force: bool = False) -> None:
    build_engine(quiet, force)
    build_host(quiet, force)


if __name__ == "__main__":
    build(quiet=False, force="--force" in sys.argv)
