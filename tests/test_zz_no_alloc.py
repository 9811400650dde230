"""gs_bfs_noalloc: BFS for callers that may not allocate device memory.

Some callers cannot let a library call cudaMalloc while they run queries —
a host framework whose memory pool already owns the GPU, or a serving loop
that cannot take cudaMalloc's device-wide synchronisation.  For them the C
ABI has gs_bfs_noalloc, which keeps its scratch state in a fixed array inside
the library and writes depths into a device buffer the caller owns.  These
tests call it through the C ABI and check it against the regular BFS entry
point (gs_state_create / gs_run / gs_download) bit for bit, on two calls in a
row, since every call reuses the same scratch array.

This file is named to be collected last, so a run stopping at the first
failure has already run every other test.
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch

    import gstore_b200 as gs

    ctx = gs.Context(0)
    yield gs, ctx, torch
    ctx.close()


def _check_two_calls(gs, ctx, torch, graph, roots):
    out = torch.empty(graph.V, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    for root in roots:                      # consecutive calls share the scratch array
        out.fill_(0xAB)                     # stale bytes must not leak into the result
        torch.cuda.synchronize()
        sweeps = graph.bfs_noalloc(root, out.data_ptr())
        got = out.cpu().numpy()
        want = graph.bfs(root)              # the regular entry point
        assert np.array_equal(got, want), f"root {root}"
        assert sweeps == int(want.max())    # one sweep per level, the last finds nothing


def test_noalloc_matches_regular_bfs_golden(env):
    gs, ctx, torch = env
    g = load_golden("spread18")
    graph = ctx.upload(g["start"], g["grid"], g["degree"], g["V"])
    roots = [int(r) for r in g["bfs_roots"][:2]]
    _check_two_calls(gs, ctx, torch, graph, roots)
    assert np.array_equal(graph.bfs(roots[0]), g["bfs_depth"][0])
    graph.free()


def test_noalloc_matches_regular_bfs_directed_golden(env):
    """The directed grid (push v0 -> v1 only, every tile of the full grid)."""
    gs, _, torch = env
    g = load_golden("spread18d")
    with gs.Context(0, directed=True) as dctx:
        graph = dctx.upload(g["start"], g["grid"], g["degree"], g["V"])
        roots = [int(r) for r in g["bfs_roots"][:2]]
        _check_two_calls(gs, dctx, torch, graph, roots)
        assert np.array_equal(graph.bfs(roots[0]), g["bfs_depth"][0])
        graph.free()


def test_noalloc_rejects_bad_root_and_streamed_graph(env):
    gs, ctx, torch = env
    g = load_golden("spread18")
    V = int(g["V"])
    out = torch.empty(V, dtype=torch.uint8, device="cuda")
    graph = ctx.upload(g["start"], g["grid"], g["degree"], V)
    with pytest.raises(gs.GStoreError, match="GS_ERR_ARG"):
        graph.bfs_noalloc(V, out.data_ptr())          # root == V
    graph.free()
    streamed = ctx.upload_streamed(g["start"], g["grid"], g["degree"], V, segment_bytes=2 << 20)
    with pytest.raises(gs.GStoreError, match="GS_ERR_UNSUPPORTED"):
        streamed.bfs_noalloc(0, out.data_ptr())
    streamed.free()


def test_noalloc_matches_regular_bfs_kron20(env):
    gs, ctx, torch = env
    V = 1 << 20
    graph = ctx.convert(ctx.kron_generate(20, 16), V)
    deg = graph.degree()
    nz = np.nonzero(deg)[0]
    _check_two_calls(gs, ctx, torch, graph, [int(nz[7]), int(nz[len(nz) // 2])])
    graph.free()


def test_noalloc_rejects_graphs_over_its_limit(env):
    gs, ctx, torch = env
    V = (1 << 24) + 1                        # one vertex over the fixed scratch size
    graph = ctx.convert(np.array([[0, 1], [1, V - 1]], np.uint32), V)
    out = torch.empty(16, dtype=torch.uint8, device="cuda")
    with pytest.raises(gs.GStoreError, match="GS_ERR_RANGE"):
        graph.bfs_noalloc(0, out.data_ptr())
    graph.free()
