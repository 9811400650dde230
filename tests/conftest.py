"""Shared fixtures.  GPU tests are marked ``gpu`` and need a CUDA device and
the in-tree engine library; everything else runs on a CPU-only host."""
from __future__ import annotations

import sys
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
