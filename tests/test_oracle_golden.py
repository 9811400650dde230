"""The CPU oracle (oracle/gs_oracle.c) against the golden fixtures.

The fixtures hold the reference's own outputs (tests/golden/make_golden.py):
tile files written by the reference converter and the per-vertex arrays of
its bfs_t / kcore_t / wcc2_t / pr_t / bfs2_t / traverse_t classes.  Passing here pins the oracle
that the GPU parity tests then use at sizes the fixtures do not cover.
"""
import numpy as np
import pytest

from conftest import GOLDEN_NAMES, load_golden


def _n_for(g, oracle):
    return g["V"]


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_converter_matches_reference(name, oracle_lib):
    g = load_golden(name)
    p, ps, T = oracle_lib.geometry(g["V"], g["directed"])
    assert g["start"].size == T + 1
    start, grid, degree = oracle_lib.convert(g["pairs"], p, g["directed"], g["V"])
    assert np.array_equal(start, g["start"])
    assert np.array_equal(degree, g["degree"])
    # in-tile record order is thread order in the reference: compare per tile
    for t in np.nonzero(np.diff(start))[0]:
        a, b = start[t], start[t + 1]
        assert np.array_equal(np.sort(grid[a:b]), np.sort(g["grid"][a:b])), f"tile {t}"


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_bfs_matches_reference(name, oracle_lib):
    g = load_golden(name)
    p, _, _ = oracle_lib.geometry(g["V"], g["directed"])
    for r, root in enumerate(g["bfs_roots"]):
        depth, counts, swept = oracle_lib.bfs(g["start"], g["grid"], p, g["directed"], g["V"], int(root))
        assert np.array_equal(depth, g["bfs_depth"][r]), f"root {root}"
        ref_counts = g["bfs_ref_level_counts"][r]
        assert np.array_equal(counts, ref_counts[: counts.size]), f"root {root}"
        assert (swept <= g["grid"].size).all()


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_wcc_matches_reference(name, oracle_lib):
    g = load_golden(name)
    p, _, _ = oracle_lib.geometry(g["V"], g["directed"])
    label, count = oracle_lib.wcc(g["start"], g["grid"], p, g["directed"], g["V"])
    assert np.array_equal(label, g["wcc_label"])
    assert count == int(g["wcc_count"])


@pytest.mark.parametrize("name", [n for n in GOLDEN_NAMES if not n.endswith("d")])
def test_kcore_matches_reference(name, oracle_lib):
    g = load_golden(name)
    p, _, _ = oracle_lib.geometry(g["V"], False)
    for i, k in enumerate(g["kcore_k"]):
        deg, members, _ = oracle_lib.kcore(g["start"], g["grid"], g["degree"], p, g["V"], int(k))
        assert np.array_equal(deg, g["kcore_deg"][i]), f"k={k}"
        if g["kcore_count"][i] >= 0:
            assert members == g["kcore_count"][i]


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_pagerank_compat_matches_reference(name, oracle_lib):
    """With the reference's int32 inverse degree the FP64 restatement and the
    reference's FP32 CAS accumulation agree within 1e-6 relative L1."""
    g = load_golden(name)
    p, _, _ = oracle_lib.geometry(g["V"], g["directed"])
    r, x = oracle_lib.pagerank(g["start"], g["grid"], g["degree"], p, g["directed"], g["V"], 5, compat=True)
    ref = g["pr_compat_x"].astype(np.float64)
    denom = max(np.abs(x).sum(), 1e-300)
    assert np.abs(ref - x).sum() / denom <= 1e-6


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_bfs2_and_traverse_match_reference(name, oracle_lib):
    """-j 30 (bfs2_t) and -j 4 (traverse_t) from every fixture root."""
    g = load_golden(name)
    p, _, _ = oracle_lib.geometry(g["V"], g["directed"])
    for r, root in enumerate(g["bfs_roots"]):
        depth, _ = oracle_lib.bfs2(g["start"], g["grid"], p, g["directed"], g["V"], int(root))
        assert np.array_equal(depth, g["bfs2_depth"][r]), f"root {root}"
        assert np.array_equal(depth, g["bfs_depth"][r])          # the label-correcting BFS ends at BFS depth
        cid, colored, _ = oracle_lib.traverse(g["start"], g["grid"], p, g["directed"], g["V"], int(root))
        assert np.array_equal(cid, g["traverse_cid"][r]), f"pivot {root}"
        assert colored == int(np.count_nonzero(cid == 0))


def test_bfs_level_overflow_is_an_error(oracle_lib):
    """More than 254 levels would wrap the reference's u8 depth_t to INFTY;
    the oracle (like the engine) reports it instead of producing garbage."""
    V = 1 << 16
    path = np.arange(0, 301, dtype=np.uint32)
    pairs = np.stack([path[:-1], path[1:]], 1)
    p, _, _ = oracle_lib.geometry(V)
    start, grid, _ = oracle_lib.convert(pairs, p, False, V)
    with pytest.raises(ValueError, match="status -2"):
        oracle_lib.bfs(start, grid, p, False, V, 0)
    # 254 levels are fine
    pairs = np.stack([path[:253], path[1:254]], 1)
    start, grid, _ = oracle_lib.convert(pairs, p, False, V)
    depth, counts, _ = oracle_lib.bfs(start, grid, p, False, V, 0)
    assert depth[253] == 254 and counts.size == 254


def test_tile_index_roundtrip(oracle_lib):
    for directed in (False, True):
        for V in (1 << 16, (1 << 24) + 5, 3 << 24):
            p, ps, T = oracle_lib.geometry(V, directed)
            row, col = oracle_lib.tile_coords(p, directed)
            assert row.size == T
            idx = [oracle_lib.tile_index(p, directed, int(r), int(c)) for r, c in zip(row[::997], col[::997])]
            assert idx == list(range(0, T, 997))


def test_reference_kron16_numbers(oracle_lib, tmp_path):
    """The reference's printed results for Graph500 Kron 16 (seeds 1,2,
    edgefactor 16, -c 1): 1,048,067 records ("Total Edges again",
    gstore.cpp:2907); BFS from 1 finds 4, 907, 35752, 10083, 67 ("frontier
    count", bfs.cpp:193-194); 12 components ("WCC count", wcc.cpp:336);
    23,418 vertices with degree != 0 after k-core k = 8 ("vertices count",
    gstore.cpp:2796-2803)."""
    if not oracle_lib.ref_available():
        pytest.skip("reference generator not built here")
    pairs = oracle_lib.ref_generate(16, 16, tmp_path / "k16.bin")
    p, _, _ = oracle_lib.geometry(1 << 16)
    start, grid, degree = oracle_lib.convert(pairs, p, False, 1 << 16)
    assert grid.size == 1048067
    _, counts, _ = oracle_lib.bfs(start, grid, p, False, 1 << 16, 1)
    assert counts.tolist() == [4, 907, 35752, 10083, 67, 0]
    _, n = oracle_lib.wcc(start, grid, p, False, 1 << 16)
    assert n == 12
    _, members, _ = oracle_lib.kcore(start, grid, degree, p, 1 << 16, 8)
    assert members == 23418
