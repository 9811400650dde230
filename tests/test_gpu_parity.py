"""GPU parity through the C ABI (libgstore_cuda.so) against the reference's
own outputs (golden fixtures) and the CPU oracle (oracle/gs_oracle.c).

Bars: BFS depth, WCC labels (canonical: smallest vertex id per component)
and k-core degrees are bit-exact; PageRank is within 1e-6 relative L1 of
the FP64 oracle (PR_TOL below).
"""
import numpy as np
import pytest

from conftest import GOLDEN_NAMES, load_golden

pytestmark = pytest.mark.gpu

PR_TOL = 1e-6   # relative L1, sum|gpu - fp64| / sum|fp64|


def rel_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)


@pytest.fixture(scope="module")
def gs():
    import gstore_b200

    return gstore_b200


def upload_golden(ctx_factory, name):
    g = load_golden(name)
    ctx = ctx_factory(g["directed"])
    return g, ctx.upload(g["start"], g["grid"], g["degree"], g["V"])


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_bfs_golden(name, gpu_ctx_factory):
    g, graph = upload_golden(gpu_ctx_factory, name)
    for r, root in enumerate(g["bfs_roots"]):
        with graph.state("bfs", int(root)) as s:
            s.run()
            depth = s.download()
            stats = s.bfs_stats()
        assert np.array_equal(depth, g["bfs_depth"][r]), f"root {root}"
        ref = g["bfs_ref_level_counts"][r]
        assert stats["level_counts"].tolist() == ref[: stats["level_counts"].size].tolist()


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_wcc_golden(name, gpu_ctx_factory, oracle_lib):
    g, graph = upload_golden(gpu_ctx_factory, name)
    labels, count = graph.wcc()
    assert np.array_equal(labels, g["wcc_label"])
    assert count == int(g["wcc_count"])


@pytest.mark.parametrize("name", [n for n in GOLDEN_NAMES if not n.endswith("d")])
def test_kcore_golden(name, gpu_ctx_factory):
    g, graph = upload_golden(gpu_ctx_factory, name)
    for i, k in enumerate(g["kcore_k"]):
        deg, members = graph.kcore(int(k))
        assert np.array_equal(deg, g["kcore_deg"][i]), f"k={k}"
        if g["kcore_count"][i] >= 0:
            assert members == g["kcore_count"][i]


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_pagerank_golden(name, gpu_ctx_factory, oracle_lib):
    g, graph = upload_golden(gpu_ctx_factory, name)
    p, _, _ = oracle_lib.geometry(g["V"], g["directed"])
    # reference semantics (int32 inverse degree) against the reference's own output
    r_c, x_c = graph.pagerank(5, compat=True)
    assert rel_l1(x_c, g["pr_compat_x"]) <= PR_TOL
    # intended formula against the FP64 oracle
    r, x = graph.pagerank(5)
    r64, x64 = oracle_lib.pagerank(g["start"], g["grid"], g["degree"], p, g["directed"], g["V"], 5)
    assert rel_l1(r, r64) <= PR_TOL
    assert rel_l1(x, x64) <= PR_TOL


def test_generator_matches_reference_generator(gpu_ctx_factory):
    """Graph500 generator on the device: byte-identical to the reference's
    generator output stored in the kron12 fixture."""
    g = load_golden("kron12")
    pairs = gpu_ctx_factory(False).kron_generate(12, 16, 1, 2)
    assert np.array_equal(pairs, g["pairs"])


@pytest.mark.parametrize("scale", [16, 18])
def test_generator_matches_reference_binary(scale, gpu_ctx_factory, oracle_lib, tmp_path):
    if not oracle_lib.ref_available():
        pytest.skip("reference generator binary not present")
    ref = oracle_lib.ref_generate(scale, 16, tmp_path / "k.bin")
    got = gpu_ctx_factory(False).kron_generate(scale, 16, 1, 2)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_converter_golden(name, gpu_ctx_factory):
    g = load_golden(name)
    graph = gpu_ctx_factory(g["directed"]).convert(g["pairs"], g["V"])
    start, grid, degree = graph.download()
    assert np.array_equal(start, g["start"])
    assert np.array_equal(degree, g["degree"])
    for t in np.nonzero(np.diff(start))[0]:
        a, b = start[t], start[t + 1]
        assert np.array_equal(np.sort(grid[a:b]), np.sort(g["grid"][a:b])), f"tile {t}"


@pytest.fixture(scope="module")
def kron(gpu_ctx_factory, oracle_lib):
    """Graph500 Kron 16 and 20 (edgefactor 16, seeds 1,2) generated and
    converted on the device, with host copies for the oracle."""
    out = {}
    for scale in (16, 20):
        ctx = gpu_ctx_factory(False)
        V = 1 << scale
        pairs = ctx.kron_generate(scale, 16)
        graph = ctx.convert(pairs, V)
        start, grid, degree = graph.download()
        out[scale] = dict(V=V, pairs=pairs, graph=graph, start=start, grid=grid, degree=degree)
    return out


def test_kron_converter_matches_oracle(kron, oracle_lib):
    for scale, k in kron.items():
        p, _, _ = oracle_lib.geometry(k["V"])
        start, grid, degree = oracle_lib.convert(k["pairs"], p, False, k["V"])
        assert np.array_equal(start, k["start"])
        assert np.array_equal(degree, k["degree"])
        t = np.nonzero(np.diff(start))[0]
        for tt in t[:: max(1, t.size // 40)]:
            a, b = start[tt], start[tt + 1]
            assert np.array_equal(np.sort(grid[a:b]), np.sort(k["grid"][a:b]))


def test_reference_printed_numbers(kron):
    """The reference's own printed results on Graph500 Kron 16 / Kron 20
    (seeds 1,2, edgefactor 16, converted with -c 1): "Total Edges again"
    (gstore.cpp:2907) 1,048,067 / 16,776,020 records; "WCC count"
    (wcc.cpp:336) 12 / 207; "vertices count" of -j 22 -a 8
    (gstore.cpp:2796-2803) 23,418 / 294,079; and the BFS-from-1 "frontier
    count" lines (bfs.cpp:193-194) 4/907/35752/10083/67 at Kron 16."""
    k16, k20 = kron[16]["graph"], kron[20]["graph"]
    assert k16.n_edges == 1048067 and k20.n_edges == 16776020
    with k16.state("bfs", 1) as s:
        s.run()
        assert s.bfs_stats()["level_counts"].tolist() == [4, 907, 35752, 10083, 67, 0]
    assert k16.wcc()[1] == 12 and k20.wcc()[1] == 207
    assert k16.kcore(8)[1] == 23418 and k20.kcore(8)[1] == 294079


def test_kron_bfs_matches_oracle(kron, oracle_lib):
    k = kron[20]
    p, _, _ = oracle_lib.geometry(k["V"])
    rng = np.random.default_rng(5)
    nz = np.nonzero(k["degree"])[0]
    for root in [1, *rng.choice(nz, 3, replace=False).tolist()]:
        depth_o, counts_o, swept_o = oracle_lib.bfs(k["start"], k["grid"], p, False, k["V"], int(root))
        with k["graph"].state("bfs", int(root)) as s:
            s.run()
            depth = s.download()
            st = s.bfs_stats()
        assert np.array_equal(depth, depth_o), f"root {root}"
        assert st["level_counts"].tolist() == counts_o.tolist()
        assert st["swept"].tolist() == swept_o.tolist()
        # records read: never more than the reference rule's swept tiles hold
        # (fewer once chunks with every record's ends visited are skipped)
        assert len(st["read"]) == len(st["swept"])
        assert (st["read"] <= st["swept"]).all() and st["read"][:2].sum() == st["swept"][:2].sum()


def test_kron_wcc_kcore_pr_match_oracle(kron, oracle_lib):
    k = kron[20]
    p, _, _ = oracle_lib.geometry(k["V"])
    lab_o, n_o = oracle_lib.wcc(k["start"], k["grid"], p, False, k["V"])
    lab, n = k["graph"].wcc()
    assert np.array_equal(lab, lab_o) and n == n_o
    for kk in (2, 8, 32):
        deg_o, mem_o, _ = oracle_lib.kcore(k["start"], k["grid"], k["degree"], p, k["V"], kk)
        deg, mem = k["graph"].kcore(kk)
        assert np.array_equal(deg, deg_o) and mem == mem_o, f"k={kk}"
    r64, x64 = oracle_lib.pagerank(k["start"], k["grid"], k["degree"], p, False, k["V"], 5)
    r, x = k["graph"].pagerank(5)
    assert rel_l1(r, r64) <= PR_TOL and rel_l1(x, x64) <= PR_TOL


@pytest.mark.parametrize("shift", ["0", "1", "4", "8"])
def test_kron_wcc_sampled_pass_matches_oracle(kron, oracle_lib, monkeypatch, shift):
    """WCC on a resident graph of >= 2^22 records hooks a sample of the
    records first (one 16-byte group in 2^shift), then sweeps every record
    but those with both ends in the largest sampled tree.  The sample only
    changes the order in which trees are linked: the labels (the smallest
    vertex of each component, wcc.cpp:372-390) and the count must equal the
    oracle's for any sample size, shift 0 being the plain sweep."""
    monkeypatch.setenv("GS_WCC_SAMPLE_SHIFT", shift)
    k = kron[20]
    p, _, _ = oracle_lib.geometry(k["V"])
    lab_o, n_o = oracle_lib.wcc(k["start"], k["grid"], p, False, k["V"])
    before = k["graph"].ctx.launches()
    with k["graph"].state("wcc", 0) as s:
        assert s.run() == 1                      # one sweep call, whatever the sample
        lab, n = s.download(0), s.count()
        s.reset(0)                               # a second run on the same state
        s.run()
        assert np.array_equal(s.download(0), lab)
    assert np.array_equal(lab, lab_o) and n == n_o
    # the sampled form launches the sample, the largest-tree vote, the
    # bitmap and the full pass in place of one sweep
    launches = k["graph"].ctx.launches() - before
    assert launches >= (2 * 6 if shift != "0" else 2 * 3)


def test_step_protocol_matches_run(kron):
    """algo_t protocol: sweep()/finalize() step by step equals run()."""
    g = kron[16]["graph"]
    with g.state("bfs", 1) as s:
        levels = []
        while True:
            s.sweep()
            f, done = s.finalize()
            levels.append(f)
            if done:
                break
        d1 = s.download()
    assert levels == [4, 907, 35752, 10083, 67, 0]
    assert np.array_equal(d1, g.bfs(1))
    with g.state("kcore", 8) as s:
        f, done = s.finalize()          # kcore_mmap's first iteration_finalize
        while not done:
            s.sweep()
            f, done = s.finalize()
        assert s.count() == 23418


def test_errors_are_statuses(gs, gpu_ctx_factory):
    ctx = gpu_ctx_factory(False)
    g = load_golden("spread18")
    graph = ctx.upload(g["start"], g["grid"], g["degree"], g["V"])
    with pytest.raises(gs.GStoreError, match="GS_ERR_ARG"):
        graph.state("bfs", g["V"])
    with pytest.raises(gs.GStoreError, match="GS_ERR_FORMAT"):
        ctx.upload(g["start"][:-1], g["grid"], g["degree"], g["V"])
    bad = g["start"].copy()
    bad[-1] += 1
    with pytest.raises(gs.GStoreError, match="GS_ERR_FORMAT"):
        ctx.upload(bad, g["grid"], g["degree"], g["V"])
    dctx = gpu_ctx_factory(True)
    gd = load_golden("spread18d")
    dgraph = dctx.upload(gd["start"], gd["grid"], gd["degree"], gd["V"])
    with pytest.raises(gs.GStoreError, match="GS_ERR_UNSUPPORTED"):
        dgraph.state("kcore", 8)
    # records addressing vertices >= V in the ragged last window
    h = load_golden("handmade")
    with pytest.raises(gs.GStoreError, match="GS_ERR_FORMAT"):
        ctx.upload(h["start"], h["grid"], h["degree"], h["V"] - 1)


def test_bfs_level_overflow(gs, gpu_ctx_factory):
    ctx = gpu_ctx_factory(False)
    path = np.arange(0, 301, dtype=np.uint32)
    graph = ctx.convert(np.stack([path[:-1], path[1:]], 1), 1 << 16)
    with pytest.raises(gs.GStoreError, match="GS_ERR_RANGE"):
        graph.bfs(0)
    graph = ctx.convert(np.stack([path[:253], path[1:254]], 1), 1 << 16)
    assert graph.bfs(0)[253] == 254


@pytest.mark.parametrize("iterations", [3, 10])
def test_pagerank_edgefactor32_matches_oracle(iterations, gpu_ctx_factory, oracle_lib):
    """A denser Kronecker graph (edgefactor 32, hubs of ~10^5 records): FP32
    accumulation on the GPU stays within PR_TOL of the FP64 oracle."""
    ctx = gpu_ctx_factory(False)
    V = 1 << 20
    g = ctx.convert(ctx.kron_generate(20, 32, seed1=20), V)
    start, grid, degree = g.download()
    p, _, _ = oracle_lib.geometry(V)
    r64, x64 = oracle_lib.pagerank(start, grid, degree, p, False, V, iterations)
    r, x = g.pagerank(iterations)
    assert rel_l1(r, r64) <= PR_TOL and rel_l1(x, x64) <= PR_TOL
    g.free()


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_bfs2_and_traverse_golden(name, gpu_ctx_factory):
    """-j 30 (label-correcting BFS) and -j 4 (single-colour propagation)
    against the reference's bfs2_t / traverse_t arrays, resident and
    streamed."""
    g = load_golden(name)
    ctx = gpu_ctx_factory(g["directed"])
    graphs = [ctx.upload(g["start"], g["grid"], g["degree"], g["V"]),
              ctx.upload_streamed(g["start"], g["grid"], g["degree"], g["V"], 2 * (131072 + 8) * 4)]
    for graph in graphs:
        for r, root in enumerate(g["bfs_roots"]):
            with graph.state("bfs2", int(root)) as s:
                s.run()
                assert np.array_equal(s.download(), g["bfs2_depth"][r]), f"root {root}"
                assert s.count() == int(np.count_nonzero(g["bfs2_depth"][r]))
            with graph.state("traverse", int(root)) as s:
                s.run()
                assert np.array_equal(s.download(), g["traverse_cid"][r]), f"pivot {root}"
                assert s.count() == int(np.count_nonzero(g["traverse_cid"][r] == 0))
        graph.free()


def test_bfs2_and_traverse_kron20(kron, oracle_lib):
    k = kron[20]
    p, _, _ = oracle_lib.geometry(k["V"])
    nz = np.nonzero(k["degree"])[0]
    for root in [1, int(nz[len(nz) // 3])]:
        with k["graph"].state("bfs2", root) as s:
            s.run()
            assert np.array_equal(s.download(), k["graph"].bfs(root))
        cid_o, colored_o, _ = oracle_lib.traverse(k["start"], k["grid"], p, False, k["V"], root)
        with k["graph"].state("traverse", root) as s:
            s.run()
            assert np.array_equal(s.download(), cid_o)
            assert s.count() == colored_o
