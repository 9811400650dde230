"""A graph whose records stay in the reference's multi-file layout ("-c 3",
per-file .grid.N/.start.N) streams from those files through two HBM
segments (gs_upload_graph_files) with results equal, bit for bit, to the
same graph read from the reference's single-file output and kept resident;
PageRank within the FP64-oracle tolerance of the resident run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

V = 1 << 26
SEG = 2 << 20


@pytest.mark.parametrize("kind", ["u", "d"])
def test_streamed_from_multi_file_layout(reference_layouts, kind):
    import gstore_b200 as gs

    single, multi = reference_layouts[kind]
    directed = kind == "d"
    s1, g1, d1 = gs.read_tiles(single, V, directed)
    with gs.Context(0, directed=directed) as ctx:
        res = ctx.upload(s1, g1, d1, V)
        fg = ctx.upload_files(multi, V, SEG)
        nz = np.nonzero(d1)[0]
        for root in (int(nz[0]), int(nz[nz.size // 2])):
            assert np.array_equal(fg.bfs(root), res.bfs(root)), f"BFS from {root}"
        if not directed:
            assert np.array_equal(fg.wcc()[0], res.wcc()[0])
            assert np.array_equal(fg.kcore(8)[0], res.kcore(8)[0])
        r_f, r_r = fg.pagerank(3)[0], res.pagerank(3)[0]
        assert np.abs(r_f.astype(np.float64) - r_r).sum() <= 1e-6 * np.abs(r_r.astype(np.float64)).sum()
        st = fg.stream_stats()
        assert st["segments"] > 0 and st["bytes"] > 0
        s3, g3, _ = fg.download()                          # records read back from the files
        assert np.array_equal(s3, s1)
        for t in np.nonzero(np.diff(s1))[0][::97]:
            a, b = int(s1[t]), int(s1[t + 1])
            assert np.array_equal(np.sort(g3[a:b]), np.sort(g1[a:b]))
        fg.free()
        res.free()


def test_cli_reads_multi_file_layout(reference_layouts):
    """gstoreu -i <dir>/gstore on the "-c 3" files prints the reference's
    result lines for its "-c 1" files (k-core members, WCC count), resident
    (-j 22/23) and streamed from the files under a small -m (-j 2/3)."""
    import re
    import subprocess
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    ours, ref = root / "gstore_b200" / "lib" / "gstoreu", root / "oracle" / "_ref" / "gstoreu"
    single, multi = reference_layouts["u"]

    def run(exe, *args):
        r = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        return r.stdout

    pat_k, pat_w = r">= 8vertices count = (\d+)", r"WCC count = (\d+)"
    want_k = re.search(pat_k, run(ref, "-s", 26, "-j", 22, "-a", 8, "-i", single)).group(1)
    want_w = re.search(pat_w, run(ref, "-s", 26, "-j", 23, "-i", single)).group(1)
    for j_k, j_w, extra in ((22, 23, []), (2, 3, ["-m", 3])):
        assert re.search(pat_k, run(ours, "-s", 26, "-j", j_k, "-a", 8, "-i", multi, *extra)).group(1) == want_k
        assert re.search(pat_w, run(ours, "-s", 26, "-j", j_w, "-i", multi, *extra)).group(1) == want_w
