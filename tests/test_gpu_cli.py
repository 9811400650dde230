"""The gstoreu command line on the GPU, beside the reference's own gstoreu
(compiled from its sources into oracle/_ref): the -c 1 converter writes the
same .start/.degree bytes and the same records per tile, and the jobs print
the reference's result lines (k-core members, WCC count, the coloured set
of -j 4) and the known BFS level counts of Graph500 Kron 16 from root 1."""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
OURS = ROOT / "gstore_b200" / "lib" / "gstoreu"
REF = ROOT / "oracle" / "_ref"


def run(exe, *args):
    r = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


@pytest.fixture(scope="module")
def kron16(tmp_path_factory):
    if not (REF / "gstoreu").exists() or not (REF / "kron_gen_ref").exists():
        pytest.skip("reference binaries not built (oracle/_ref)")
    d = tmp_path_factory.mktemp("cli")
    edges = d / "edges.bin"
    subprocess.run([str(REF / "kron_gen_ref"), "16", "16", str(edges), "1", "2"], check=True,
                   capture_output=True)
    # -s 24: one tile group, the reference's working rule for scales below 24
    run(OURS, "-s", 24, "-c", 1, "-i", edges, "-o", d / "ours")
    run(REF / "gstoreu", "-s", 24, "-c", 1, "-i", edges, "-o", d / "ref")
    return d


def test_converter_matches_reference(kron16):
    d = kron16
    for ext in (".start", ".degree"):
        assert (d / ("ours" + ext)).read_bytes() == (d / ("ref" + ext)).read_bytes(), ext
    start = np.fromfile(d / "ours.start", np.uint64)
    a = np.fromfile(d / "ours.grid", np.uint32)
    b = np.fromfile(d / "ref.grid", np.uint32)
    assert a.size == b.size == start[-1] == 1048067
    for t in np.nonzero(np.diff(start))[0]:
        assert np.array_equal(np.sort(a[start[t]:start[t + 1]]), np.sort(b[start[t]:start[t + 1]]))


def test_jobs_print_reference_results(kron16):
    d = kron16
    prefix = d / "ours"
    ours = run(OURS, "-s", 24, "-j", 22, "-a", 8, "-i", prefix)
    ref = run(REF / "gstoreu", "-s", 24, "-j", 22, "-a", 8, "-i", d / "ref")
    pat = r">= 8vertices count = (\d+)"
    assert re.search(pat, ours).group(1) == re.search(pat, ref).group(1) == "23418"
    ours = run(OURS, "-s", 24, "-j", 23, "-i", prefix)
    ref = run(REF / "gstoreu", "-s", 24, "-j", 23, "-i", d / "ref")
    pat = r"WCC count = (\d+)"
    assert re.findall(pat, ours)[-1] == re.findall(pat, ref)[-1] == "12"
    bfs = run(OURS, "-s", 24, "-j", 20, "-i", prefix)
    counts = [int(c) for c in re.findall(r"level: \d+ frontier count: (\d+)", bfs)]
    assert counts == [4, 907, 35752, 10083, 67, 0]
    assert "Half BFS time = " in bfs
    pr = run(OURS, "-s", 24, "-j", 21, "-a", 5, "-i", prefix)
    assert "Page-rank_mmap time = " in pr
    # -j 30: label-correcting BFS from 1 reaches what -j 20 reaches
    bfs2 = run(OURS, "-s", 24, "-j", 30, "-i", prefix)
    assert "reached vertices = %d" % (1 + sum(counts)) in bfs2 and "Half BFS time = " in bfs2
    # -j 4: the reference's coloured set from pivot 1 has 1 + sum(frontier counts) vertices
    ours = run(OURS, "-s", 24, "-j", 4, "-i", prefix)
    ref = run(REF / "gstoreu", "-s", 24, "-j", 4, "-i", d / "ref")
    ref_colored = 1 + sum(int(c) for c in re.findall(r"frontier count: (\d+)", ref))
    assert "coloured vertices = %d" % ref_colored in ours
    assert "Single color propagation time = " in ours


def test_semi_external_jobs_stream_from_the_grid_file(kron16):
    """Jobs 0-3 with a budget (-m 3: 3 MB) below the 4.2 MB grid leave the
    records in the .grid file and stream them through two 1.5 MB segments;
    the results are the resident jobs'."""
    d = kron16
    prefix = d / "ours"
    bfs = run(OURS, "-s", 24, "-j", 0, "-a", 1, "-m", 3, "-i", prefix)
    counts = [int(c) for c in re.findall(r"level: \d+ frontier count: (\d+)", bfs)]
    assert counts == [4, 907, 35752, 10083, 67, 0]
    kc = run(OURS, "-s", 24, "-j", 2, "-a", 8, "-m", 3, "-i", prefix)
    assert re.search(r">= 8vertices count = (\d+)", kc).group(1) == "23418"
    wcc = run(OURS, "-s", 24, "-j", 3, "-m", 3, "-i", prefix)
    assert re.findall(r"WCC count = (\d+)", wcc)[-1] == "12"
