"""Batched queries (gs_batch_*) on the GPU.

Every query of a batch must give what the same query gives alone through the
plain entry point (gs_state_create / gs_run / gs_download): BFS depths and
per-level counts, WCC labels and k-core degrees bit for bit, PageRank within
PR_TOL.  BFS roots on one graph run as a multi-source BFS in 32- or 64-bit
frontier words; the autotuner tries every word width / tile order once, so
the BFS checks repeat the batch until all eight configurations have run.
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

PR_TOL = 1e-6


@pytest.fixture(scope="module")
def gs():
    import gstore_b200

    return gstore_b200


@pytest.fixture(scope="module")
def graphs(gpu_ctx_factory):
    ctx = gpu_ctx_factory(False)
    out = {}
    for scale in (16, 18, 20):
        out[scale] = ctx.convert(ctx.kron_generate(scale, 16, seed1=scale), 1 << scale)
    return out


def _roots(graph, n, seed):
    nz = np.nonzero(graph.degree())[0]
    rng = np.random.default_rng(seed)
    return [int(r) for r in rng.choice(nz, n, replace=True)]


def _plain_bfs(graph, root):
    with graph.state("bfs", root) as s:
        s.run()
        return s.download(), s.bfs_stats()["level_counts"], s.count()


@pytest.mark.parametrize("n_roots", [5, 40, 70])
def test_msbfs_matches_plain(n_roots, gs, graphs, gpu_ctx_factory):
    ctx = gpu_ctx_factory(False)
    g = graphs[20]
    roots = _roots(g, n_roots, n_roots)
    roots[1] = roots[0]                      # two queries on one root
    want = {r: _plain_bfs(g, r) for r in set(roots)}
    for rep in range(8):                     # every autotuner candidate runs once
        with gs.Batch(ctx) as b:
            ids = [b.add(g, "bfs", r) for r in roots]
            b.run()
            for qid, r in zip(ids, roots):
                depth, levels, count = want[r]
                assert np.array_equal(b.download(qid), depth), f"rep {rep} root {r}"
                assert b.bfs_levels(qid).tolist() == levels.tolist()
                assert b.count(qid) == count
            st = b.stats()
            assert st["launches"] == -(-n_roots // 32) or st["launches"] == -(-n_roots // 64)


@pytest.mark.parametrize("name", ["spread18", "spread18d", "kron12", "kron12d"])
def test_msbfs_golden(name, gs, gpu_ctx_factory):
    gd = load_golden(name)
    ctx = gpu_ctx_factory(gd["directed"])
    g = ctx.upload(gd["start"], gd["grid"], gd["degree"], gd["V"])
    with gs.Batch(ctx) as b:
        ids = [b.add(g, "bfs", int(r)) for r in gd["bfs_roots"]]
        b.run()
        for k, qid in enumerate(ids):
            assert np.array_equal(b.download(qid), gd["bfs_depth"][k])
            ref = gd["bfs_ref_level_counts"][k]
            lv = b.bfs_levels(qid)
            assert lv.tolist() == ref[: lv.size].tolist()
    g.free()


def test_wcc_kcore_batch_over_graphs(gs, graphs, gpu_ctx_factory):
    """16 WCC + 16 k-core queries over graphs of three sizes: one persistent
    launch, plus one plain run per distinct WCC query on a graph of >= 2^22
    records (whose plain WCC hooks a sample of the records first)."""
    ctx = gpu_ctx_factory(False)
    gd = load_golden("spread18")
    extra = ctx.upload(gd["start"], gd["grid"], gd["degree"], gd["V"])
    pool = [graphs[16], graphs[18], graphs[20], extra]
    rng = np.random.default_rng(3)
    queries = []
    with gs.Batch(ctx) as b:
        for i in range(16):
            g = pool[i % 4]
            queries.append((b.add(g, "wcc"), g, "wcc", 0))
            k = int(rng.integers(4, 33))
            queries.append((b.add(g, "kcore", k), g, "kcore", k))
        b.run()
        plain_wcc = {id(g) for _, g, algo, _ in queries if algo == "wcc" and g.n_edges >= 1 << 22}
        assert len(plain_wcc) == 1                       # the Kron 20 graph
        assert b.stats()["launches"] == 1 + len(plain_wcc)
        for qid, g, algo, k in queries:
            if algo == "wcc":
                lab, cnt = g.wcc()
            else:
                lab, cnt = g.kcore(k)
            assert np.array_equal(b.download(qid), lab), f"{algo} k={k}"
            assert b.count(qid) == cnt
    extra.free()


def test_mixed_batch_and_errors(gs, graphs, gpu_ctx_factory, oracle_lib):
    ctx = gpu_ctx_factory(False)
    g = graphs[18]
    with gs.Batch(ctx) as b:
        q_bfs = b.add(g, "bfs", 1)
        q_pr = b.add(g, "pagerank", 5)
        q_k = b.add(g, "kcore", 8)
        with pytest.raises(gs.GStoreError, match="GS_ERR_STATE"):
            b.download(q_bfs)
        b.run()
        assert np.array_equal(b.download(q_bfs), g.bfs(1))
        start, grid, degree = g.download()
        p, _, _ = oracle_lib.geometry(g.V)
        r64, _ = oracle_lib.pagerank(start, grid, degree, p, False, g.V, 5)
        assert np.abs(b.download(q_pr) - r64).sum() <= PR_TOL * np.abs(r64).sum()
        assert np.array_equal(b.download(q_k), g.kcore(8)[0])
        with pytest.raises(gs.GStoreError, match="GS_ERR_ARG"):
            b.add(g, "bfs", g.V)
    # a BFS over 254 levels fails alone; the other root of the group does not
    path = np.arange(0, 301, dtype=np.uint32)
    pairs = np.concatenate([np.stack([path[:-1], path[1:]], 1),
                            np.array([[400, 401], [401, 402]], np.uint32)])
    pg = ctx.convert(pairs, 1 << 16)
    with gs.Batch(ctx) as b:
        q0 = b.add(pg, "bfs", 0)
        q1 = b.add(pg, "bfs", 400)
        b.run()
        with pytest.raises(gs.GStoreError, match="GS_ERR_RANGE"):
            b.download(q0)
        assert np.array_equal(b.download(q1), pg.bfs(400))
    # streamed graphs are not batched
    gd = load_golden("spread18")
    sg = ctx.upload_streamed(gd["start"], gd["grid"], gd["degree"], gd["V"], 2 * (131072 + 8) * 4)
    with gs.Batch(ctx) as b:
        with pytest.raises(gs.GStoreError, match="GS_ERR_UNSUPPORTED"):
            b.add(sg, "bfs", 0)
    sg.free()
