"""The gstoreu/gstored command line: reference flags, geometry lines and the
host-side input checks (truncated or inconsistent tile files are rejected
before any device work).  GPU-free."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import load_golden

LIB = Path(__file__).resolve().parents[1] / "gstore_b200" / "lib"


def run(exe, *args):
    return subprocess.run([str(LIB / exe), *map(str, args)], capture_output=True, text=True, timeout=120)


def write_fixture(tmp_path, name="spread18"):
    g = load_golden(name)
    prefix = tmp_path / name
    g["start"].tofile(str(prefix) + ".start")
    g["grid"].tofile(str(prefix) + ".grid")
    g["degree"].tofile(str(prefix) + ".degree")
    return prefix, g


@pytest.mark.parametrize("exe", ["gstoreu", "gstored"])
def test_binaries_exist_and_help(exe):
    r = run(exe, "-h")
    assert r.returncode == 0 and "Coming soon" in r.stdout


def test_geometry_lines():
    r = run("gstoreu", "-s", 26, "-j", 999)
    assert "Total Physcial Group Count (in One Direction) = 4" in r.stdout
    assert "Total Tiles Count (in One Direction) = 1024" in r.stdout
    assert "Wrong value for -j argument" in r.stdout and r.returncode != 0


def test_requires_vertex_count():
    r = run("gstoreu", "-j", 20, "-i", "x")
    assert r.returncode != 0 and "-s or -v" in r.stderr


def test_truncated_start_is_rejected(tmp_path):
    prefix, g = write_fixture(tmp_path)
    g["start"][:-10].tofile(str(prefix) + ".start")
    r = run("gstoreu", "-v", g["V"], "-j", 20, "-i", prefix)
    assert r.returncode != 0 and "entries; the tile geometry needs" in r.stderr


def test_start_grid_mismatch_is_rejected(tmp_path):
    prefix, g = write_fixture(tmp_path)
    g["grid"][:-3].tofile(str(prefix) + ".grid")
    r = run("gstoreu", "-v", g["V"], "-j", 23, "-i", prefix)
    assert r.returncode != 0 and "records in .grid" in r.stderr


def test_wrong_geometry_is_rejected(tmp_path):
    prefix, g = write_fixture(tmp_path)
    r = run("gstoreu", "-s", 26, "-j", 20, "-i", prefix)
    assert r.returncode != 0 and "check -s/-v" in r.stderr


def test_bad_edge_list_is_rejected(tmp_path):
    f = tmp_path / "e.bin"
    np.arange(3, dtype=np.uint32).tofile(f)   # 12 bytes: not whole gedge_t pairs
    r = run("gstoreu", "-v", 1 << 16, "-c", 1, "-i", f, "-o", tmp_path / "out")
    assert r.returncode != 0 and "not a multiple of 8" in r.stderr


def test_unsupported_modes():
    assert "not provided" in run("gstoreu", "-v", 100, "-c", 2, "-i", "x").stderr
    assert "not provided" in run("gstoreu", "-v", 100, "-j", 100, "-i", "x").stdout
