"""The serving loop (gs_serve_*) on the GPU.

Requests arrive while others run (continuous batching: they join the next
step), share steps with requests on other graphs, and wait for HBM when the
state budget is full.  Each result must be the same in the mix as alone:
BFS depth, WCC labels and k-core degrees bit for bit against the plain entry
point, PageRank within PR_TOL relative L1 of the FP64 oracle (two FP32 runs
that sum in different orders each meet that bar, not a tighter one between
them).
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

PR_TOL = 1e-6


def rel_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)


@pytest.fixture(scope="module")
def gs():
    import gstore_b200

    return gstore_b200


@pytest.fixture(scope="module")
def pool(gpu_ctx_factory):
    ctx = gpu_ctx_factory(False)
    gd = load_golden("spread18")
    out = [ctx.convert(ctx.kron_generate(s, ef, seed1=s), 1 << s) for s, ef in ((16, 8), (18, 16), (20, 32))]
    out.append(ctx.upload(gd["start"], gd["grid"], gd["degree"], gd["V"]))
    return out


_ORACLE = {}


def _plain(g, algo, arg):
    """The plain entry point's result; for PageRank the FP64 oracle's ranks."""
    if algo == "bfs":
        return g.bfs(arg)
    if algo == "wcc":
        return g.wcc()[0]
    if algo == "kcore":
        return g.kcore(arg)[0]
    import oracle

    key = (id(g), arg)
    if key not in _ORACLE:
        start, grid, degree = g.download()
        p, _, _ = oracle.geometry(g.V, g.directed)
        _ORACLE[key] = oracle.pagerank(start, grid, degree, p, g.directed, g.V, arg)[0]
    return _ORACLE[key]


def _check(algo, got, want):
    if algo == "pagerank":
        assert rel_l1(got, want) <= PR_TOL
    else:
        assert np.array_equal(got, want)


def _mix(pool, n, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(n):
        gi = int(rng.integers(0, len(pool)))
        g = pool[gi]
        u = rng.random()
        if u < 0.7:
            nz = np.nonzero(g.degree())[0]
            reqs.append((gi, "bfs", int(rng.choice(nz))))
        elif u < 0.85:
            reqs.append((gi, "kcore", int(rng.integers(4, 33))))
        elif u < 0.95:
            reqs.append((gi, "wcc", 0))
        else:
            reqs.append((gi, "pagerank", 10))
    return reqs


def _drive(srv, gids, reqs, waves):
    """Submit `reqs` in `waves` groups, stepping between them; run to the end."""
    ids = [None] * len(reqs)
    chunks = np.array_split(np.arange(len(reqs)), waves)
    max_running = 0
    for c in chunks:
        for i in c:
            gi, algo, arg = reqs[i]
            ids[i] = srv.submit(gids[gi], algo, arg)
        for _ in range(2):
            na, nq = srv.step()
            max_running = max(max_running, na)
    while True:
        na, nq = srv.step()
        if na == 0 and nq == 0:
            break
    return ids, max_running


def test_serve_mix_matches_plain(gs, pool, gpu_ctx_factory, oracle_lib):
    ctx = gpu_ctx_factory(False)
    reqs = _mix(pool, 60, 1)
    reqs.append((1, "wcc", 0))               # identical requests share a run
    reqs.append((1, "wcc", 0))
    want = {}
    for gi, algo, arg in reqs:
        if (gi, algo, arg) not in want:
            want[(gi, algo, arg)] = _plain(pool[gi], algo, arg)
    with gs.Server(ctx) as srv:
        gids = [srv.add_graph(g) for g in pool]
        ids, max_running = _drive(srv, gids, reqs, waves=6)
        assert max_running > 1
        for rid, (gi, algo, arg) in zip(ids, reqs):
            assert srv.poll(rid) == gs.Server.DONE
            got, t0, t1, steps = srv.result(rid)
            _check(algo, got, want[(gi, algo, arg)])
            assert t1 >= t0 and steps >= 1
        st = srv.stats()
        assert st["graph_launches"] == st["steps"]
        assert st["hbm_in_use"] == 0


def test_serve_alone_equals_in_mix(gs, pool, gpu_ctx_factory, oracle_lib):
    """The same request alone in a server and inside a mix (PageRank: both
    within PR_TOL of the FP64 oracle)."""
    ctx = gpu_ctx_factory(False)
    reqs = _mix(pool, 24, 7)
    alone = []
    with gs.Server(ctx) as srv:
        gids = [srv.add_graph(g) for g in pool]
        for gi, algo, arg in reqs:
            rid = srv.submit(gids[gi], algo, arg)
            while srv.step() != (0, 0):
                pass
            alone.append(srv.result(rid)[0])
    with gs.Server(ctx) as srv:
        gids = [srv.add_graph(g) for g in pool]
        ids, _ = _drive(srv, gids, reqs, waves=3)
        for k, (rid, (gi, algo, arg)) in enumerate(zip(ids, reqs)):
            got = srv.result(rid)[0]
            if algo == "pagerank":
                want = _plain(pool[gi], algo, arg)
                _check(algo, got, want)
                _check(algo, alone[k], want)
            else:
                _check(algo, got, alone[k])


def test_serve_admission_by_budget(gs, pool, gpu_ctx_factory, oracle_lib):
    """A budget for about one large request at a time: requests queue, all
    finish, and the state in use never exceeds the budget."""
    ctx = gpu_ctx_factory(False)
    g = pool[2]                                   # 2^20 vertices
    budget = 12 * g.V + (1 << 20)                 # one k-core / WCC / PR state
    reqs = [(2, "kcore", 8), (2, "kcore", 9), (2, "wcc", 0), (2, "kcore", 12), (2, "pagerank", 3)]
    with gs.Server(ctx, state_budget=budget) as srv:
        gids = [srv.add_graph(x) for x in pool]
        ids = [srv.submit(gids[gi], algo, arg) for gi, algo, arg in reqs]
        saw_queue = False
        while True:
            na, nq = srv.step()
            saw_queue |= nq > 0
            assert srv.stats()["hbm_in_use"] <= budget
            if na == 0 and nq == 0:
                break
        assert saw_queue
        for rid, (gi, algo, arg) in zip(ids, reqs):
            _check(algo, srv.result(rid)[0], _plain(pool[gi], algo, arg))


def test_serve_failure_is_per_request(gs, gpu_ctx_factory):
    ctx = gpu_ctx_factory(False)
    path = np.arange(0, 301, dtype=np.uint32)
    pairs = np.concatenate([np.stack([path[:-1], path[1:]], 1), np.array([[400, 401], [401, 402]], np.uint32)])
    pg = ctx.convert(pairs, 1 << 16)
    with gs.Server(ctx) as srv:
        gid = srv.add_graph(pg)
        bad = srv.submit(gid, "bfs", 0)          # over 254 levels
        good = srv.submit(gid, "bfs", 400)
        while srv.step() != (0, 0):
            pass
        assert srv.poll(bad) == gs.Server.FAILED
        with pytest.raises(gs.GStoreError, match="GS_ERR_RANGE"):
            srv.result(bad)
        assert np.array_equal(srv.result(good)[0], pg.bfs(400))
        with pytest.raises(gs.GStoreError, match="GS_ERR_ARG"):
            srv.submit(gid, "bfs", pg.V)
    pg.free()


def test_serve_completion_queue_and_side_streams(gs, pool, gpu_ctx_factory, oracle_lib):
    """A client that takes results as they land (gs_serve_completed) gets
    every request exactly once, with the plain entry point's results, on one
    side stream; the side-stream count can only change while no WCC /
    k-core / PageRank request runs."""
    ctx = gpu_ctx_factory(False)
    reqs = _mix(pool, 30, 11) + [(3, "kcore", 6), (2, "wcc", 0), (1, "pagerank", 4)]
    with gs.Server(ctx) as srv:
        gids = [srv.add_graph(g) for g in pool]
        srv.set_side_streams(1)
        with pytest.raises(gs.GStoreError, match="GS_ERR_ARG"):
            srv.set_side_streams(0)
        ids = {}
        for i, (gi, algo, arg) in enumerate(reqs):
            ids[srv.submit(gids[gi], algo, arg)] = i
        with pytest.raises(gs.GStoreError, match="GS_ERR_STATE"):
            srv.step()
            srv.set_side_streams(2)
        seen = []
        while True:
            na, nq = srv.step()
            for rid in srv.completed():
                seen.append(rid)
                gi, algo, arg = reqs[ids[rid]]
                _check(algo, srv.result(rid)[0], _plain(pool[gi], algo, arg))
            if na == 0 and nq == 0:
                break
        for rid in srv.completed():
            seen.append(rid)
            gi, algo, arg = reqs[ids[rid]]
            _check(algo, srv.result(rid)[0], _plain(pool[gi], algo, arg))
        assert sorted(seen) == sorted(ids)
        assert srv.completed() == []
        srv.set_side_streams(8)                  # nothing runs now


def test_serve_result_views(gs, pool, gpu_ctx_factory, oracle_lib):
    """A result read in place (gs_serve_result_view) is the copied result;
    release forgets the request; a failed request fails the view."""
    ctx = gpu_ctx_factory(False)
    reqs = [(0, "bfs", 1), (1, "wcc", 0), (3, "kcore", 5), (2, "pagerank", 3), (1, "bfs", 7)]
    with gs.Server(ctx) as srv:
        gids = [srv.add_graph(g) for g in pool]
        ids = [srv.submit(gids[gi], algo, arg) for gi, algo, arg in reqs]
        while srv.step() != (0, 0):
            pass
        for rid, (gi, algo, arg) in zip(ids, reqs):
            view, t0, t1, steps = srv.result_view(rid)
            _check(algo, view, _plain(pool[gi], algo, arg))
            assert t1 >= t0 and steps >= 1
            srv.release(rid)
            with pytest.raises(gs.GStoreError, match="GS_ERR_ARG"):
                ctx._check(gs.lib().gs_serve_release(srv._h, rid))   # already forgotten
    path = np.arange(0, 301, dtype=np.uint32)
    pg = ctx.convert(np.stack([path[:-1], path[1:]], 1), 1 << 16)
    with gs.Server(ctx) as srv:
        bad = srv.submit(srv.add_graph(pg), "bfs", 0)     # over 254 levels
        while srv.step() != (0, 0):
            pass
        with pytest.raises(gs.GStoreError, match="GS_ERR_RANGE"):
            srv.result_view(bad)
    pg.free()


def test_serve_result_arena(gs, pool, gpu_ctx_factory, oracle_lib):
    """Results are carved from one pinned arena.  With enough host memory
    reserved up front, two rounds of requests whose results are all held at
    once and released out of order pin nothing more, and every held result
    stays intact until it is released (a block freed early must not be handed
    to a result that is still being read)."""
    ctx = gpu_ctx_factory(False)
    picks = (0, 1, 3)
    reqs = []
    for gi in picks:
        nz = np.nonzero(pool[gi].degree())[0]
        reqs += [(gi, "kcore", 6), (gi, "wcc", 0), (gi, "bfs", int(nz[0])), (gi, "bfs", int(nz[-1]))]
    want = [_plain(pool[gi], algo, arg) for gi, algo, arg in reqs]
    rng = np.random.default_rng(3)
    with gs.Server(ctx) as srv:
        gids = [srv.add_graph(g) for g in pool]
        srv.reserve_host(64 << 20)
        for _ in range(2):
            ids = [srv.submit(gids[gi], algo, arg) for gi, algo, arg in reqs]
            while srv.step() != (0, 0):
                pass
            views = [srv.result_view(rid)[0] for rid in ids]
            order = rng.permutation(len(ids))
            for n, k in enumerate(order):
                for j in order[n:]:           # every result not yet released
                    _check(reqs[j][1], views[j], want[j])
                srv.release(ids[k])
        prof = srv.profile()
        assert prof["pinned_allocs"] == 0     # every result fit the reservation
        assert srv.stats()["hbm_in_use"] == 0
