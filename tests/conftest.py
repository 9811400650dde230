"""Shared fixtures.  GPU tests are marked ``gpu`` and need a CUDA device and
the in-tree engine library; everything else runs on a CPU-only host."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(ROOT))

GOLDEN_NAMES = ["kron12", "kron12d", "spread18", "spread18d", "handmade", "handmade_d"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libgstore_cuda.so")


def load_golden(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz") as z:
        d = {k: z[k] for k in z.files}
    d["V"] = int(d["V"])
    d["directed"] = bool(d["directed"])
    return d


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle

    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def gpu_ctx_factory():
    import gstore_b200 as gs

    ctxs = {}

    def get(directed: bool):
        if directed not in ctxs:
            ctxs[directed] = gs.Context(0, 0, directed)
        return ctxs[directed]

    yield get
    for c in ctxs.values():
        c.close()


@pytest.fixture(scope="session")
def reference_layouts():
    """The reference converter's single-file (-c 1) and multi-file (-c 3)
    outputs of one edge list: Graph500 Kron 16 spread over 2^26 vertices
    (the multi-file layout needs V >= 2^25), undirected (gstoreu) and
    directed (gstored).  {kind: (single prefix, multi prefix)}."""
    V = 1 << 26
    REF = ROOT / "oracle" / "_ref"
    if not all((REF / n).exists() for n in ("gstoreu", "gstored", "kron_gen_ref")):
        pytest.skip("reference binaries not built (oracle/_ref)")
    base = "/dev/shm" if os.path.isdir("/dev/shm") else None
    work = Path(tempfile.mkdtemp(prefix="gs_c3_", dir=base))
    try:
        subprocess.run([str(REF / "kron_gen_ref"), "16", "16", str(work / "e16.bin"), "1", "2"], check=True,
                       capture_output=True)
        e = np.fromfile(work / "e16.bin", np.uint32).astype(np.uint64)
        ((e * 1021) % V).astype(np.uint32).tofile(work / "e26.bin")   # spread over 2^26 vertices
        out = {}
        for kind, exe in (("u", "gstoreu"), ("d", "gstored")):
            d3 = work / f"multi_{kind}"
            d3.mkdir()
            subprocess.run([str(REF / exe), "-s", "26", "-c", "3", "-i", str(work / "e26.bin"), "-o", str(d3)],
                           check=True, capture_output=True)
            subprocess.run([str(REF / exe), "-s", "26", "-c", "1", "-i", str(work / "e26.bin"), "-o",
                            str(work / f"single_{kind}")], check=True, capture_output=True)
            out[kind] = (work / f"single_{kind}", d3 / "gstore")
        yield out
    finally:
        shutil.rmtree(work, ignore_errors=True)
