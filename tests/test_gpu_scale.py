"""Parity at a benchmark size: Graph500 Kron 24 edgefactor 16 (seeds 1, 2),
the graph of the batched-query workload, 268 M records.

The reference compiled from its own sources (oracle/_ref) generates the
edge list and converts it (gstoreu -c 1, records in its threads' order
inside each tile), and its own algorithm classes run on those files through
the harness: bfs_t (bfs.cpp:56-338) from two seeded roots, kcore_t
(kcore.cpp:55-300) with k = 8, wcc2_t (wcc.cpp:57-395).  The engine then
runs on the same files through gs_upload_graph -- the drop-in case -- and on
its own converter's files of the device generator's edge list; BFS depths,
k-core degrees and the WCC partition must be equal bit for bit, and the
counts equal the reference's printed result lines ("vertices count",
gstore.cpp:2796-2803; "WCC count", wcc.cpp:336)."""
import os
import re
import shutil
import tempfile
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SCALE = 24
V = 1 << SCALE


def _splitmix64_roots(degree, count, seed=1):
    x, out = seed, []
    while len(out) < count:
        x = (x + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        z ^= z >> 31
        if degree[z % degree.size] > 0:
            out.append(int(z % degree.size))
    return out


@pytest.fixture(scope="module")
def kron24(oracle_lib):
    if not oracle_lib.ref_available() or not (oracle_lib.REF_DIR / "gstoreu").exists():
        pytest.skip("reference binaries not built (oracle/_ref)")
    base = "/dev/shm" if os.path.isdir("/dev/shm") and shutil.disk_usage("/dev/shm").free > (8 << 30) else None
    work = Path(tempfile.mkdtemp(prefix="gs_k24_", dir=base))
    try:
        edges = work / "edges.bin"
        pairs = oracle_lib.ref_generate(SCALE, 16, edges)
        prefix = work / "k24"
        oracle_lib.ref_convert(edges, prefix, V)
        edges.unlink()
        start = np.fromfile(str(prefix) + ".start", np.uint64)
        grid = np.fromfile(str(prefix) + ".grid", np.uint32)
        degree = np.fromfile(str(prefix) + ".degree", np.int32)
        roots = _splitmix64_roots(degree, 2)
        jobs = [("bfs", roots[0]), ("bfs", roots[1]), ("kcore", 8), ("wcc", 0)]
        with ThreadPoolExecutor(len(jobs)) as ex:
            res = list(ex.map(lambda j: oracle_lib.ref_run(prefix, V, j[0], j[1]), jobs))
        yield {"pairs": pairs, "start": start, "grid": grid, "degree": degree, "roots": roots,
               "bfs": {roots[0]: res[0][0], roots[1]: res[1][0]},
               "kcore8": res[2][0], "kcore8_printed": int(re.search(r"vertices count = (\d+)", res[2][1]).group(1)),
               "wcc": oracle_lib.canonical_labels(res[3][0]),
               "wcc_printed": int(re.search(r"WCC count = (\d+)", res[3][1]).group(1))}
    finally:
        shutil.rmtree(work, ignore_errors=True)


def _check_graph(graph, k):
    for r in k["roots"]:
        assert np.array_equal(graph.bfs(r), k["bfs"][r]), f"BFS depth from {r}"
    deg, members = graph.kcore(8)
    assert np.array_equal(deg, k["kcore8"]), "k-core degrees"
    assert members == k["kcore8_printed"] == 3746689
    labels, n = graph.wcc()
    assert np.array_equal(labels, k["wcc"]), "WCC partition"
    assert n == k["wcc_printed"] == 2874


def test_reference_tiles_bit_exact(kron24, gpu_ctx_factory, oracle_lib):
    """The drop-in case: the reference converter's files, unchanged.  Upload
    sorts each tile's records (the converter leaves them in its threads'
    order); the records per tile stay the same multiset.  PageRank (the
    propagation-blocked sweep at this size) is within 1e-6 relative L1 of the
    FP64 oracle."""
    k = kron24
    ctx = gpu_ctx_factory(False)
    g = ctx.upload(k["start"], k["grid"], k["degree"], V)
    assert g.n_edges == 268432653
    start, grid, _ = g.download()
    assert np.array_equal(start, k["start"])
    tiles = np.nonzero(np.diff(start))[0]
    for t in tiles[:: max(1, tiles.size // 64)]:
        a, b = int(start[t]), int(start[t + 1])
        assert np.all(np.diff(grid[a:b].astype(np.int64)) >= 0), f"tile {t} not sorted"
        assert np.array_equal(grid[a:b], np.sort(k["grid"][a:b]))
    del grid
    _check_graph(g, k)
    p, _, _ = oracle_lib.geometry(V)
    r64, _ = oracle_lib.pagerank(k["start"], k["grid"], k["degree"], p, False, V, 5)
    r, _ = g.pagerank(5)
    err = np.abs(r.astype(np.float64) - r64).sum() / np.abs(r64).sum()
    assert err <= 1e-6, f"PageRank relative L1 {err}"
    g.free()


def test_engine_converter_bit_exact(kron24, gpu_ctx_factory):
    """The device generator and converter on the same graph: the same
    .start/.degree bytes and per-tile record multisets, the same results,
    and the batched form (64 roots in one persistent launch) on it."""
    import gstore_b200 as gs

    k = kron24
    ctx = gpu_ctx_factory(False)
    gen = ctx.kron_generate(SCALE, 16)
    assert np.array_equal(gen, k["pairs"]), "device generator differs from the reference generator"
    g = ctx.convert(gen, V)
    start, grid, degree = g.download()
    assert np.array_equal(start, k["start"]) and np.array_equal(degree, k["degree"][:V])
    tiles = np.nonzero(np.diff(start))[0]
    for t in tiles[:: max(1, tiles.size // 64)]:
        a, b = int(start[t]), int(start[t + 1])
        assert np.array_equal(np.sort(grid[a:b]), np.sort(k["grid"][a:b]))
    _check_graph(g, k)
    roots = k["roots"] + _splitmix64_roots(degree, 64)[2:]
    with gs.Batch(ctx) as b:
        ids = [b.add(g, "bfs", r) for r in roots]
        b.run()
        for q, r in zip(ids[:2], roots[:2]):
            assert np.array_equal(b.download(q), k["bfs"][r]), f"batched BFS depth from {r}"
        for q, r in list(zip(ids, roots))[2::9]:
            assert np.array_equal(b.download(q), g.bfs(r)), f"batched BFS depth from {r}"
    g.free()
