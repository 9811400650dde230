"""The C-ABI library: it loads, exports every symbol include/gstore_cuda.h
declares, and fails loudly (a status, no crash) without a usable GPU.  No
compute call is made here."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

import gstore_b200 as gs

ROOT = Path(__file__).resolve().parents[1]


def header_symbols():
    text = (ROOT / "include" / "gstore_cuda.h").read_text()
    return sorted(set(re.findall(r"^(?:gs_status|const char\*)\s+(gs_\w+)\(", text, re.M)))


def test_library_built():
    assert gs.LIB_PATH.exists(), "run python -m gstore_b200.build"


def test_every_declared_symbol_is_exported():
    syms = header_symbols()
    assert len(syms) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", str(gs.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r" T (gs_\w+)$", out, re.M))
    missing = [s for s in syms if s not in exported]
    assert not missing, f"declared but not exported: {missing}"
    lib = C.CDLL(str(gs.LIB_PATH))
    for s in syms:
        getattr(lib, s)


def test_python_binding_covers_the_header():
    assert sorted(gs.ABI_SYMBOLS) == header_symbols()


def test_geometry_matches_reference_rules():
    # grid::init -v: p = ceil(V / 2^24), p_s = 256 p; half grid stores
    # p_s (p_s + 1) / 2 tiles, the full grid p_s^2 (calc_total_part).
    assert gs.geometry(1 << 20) == (1, 256, 32896 + 1)
    assert gs.geometry(1 << 26) == (4, 1024, 1024 * 1025 // 2 + 1)
    assert gs.geometry(1 << 26, True) == (4, 1024, 1024 * 1024 + 1)
    assert gs.geometry((1 << 24) + 1) == (2, 512, 512 * 513 // 2 + 1)


def test_no_gpu_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(gs.GStoreError):
        gs.Context(0)
