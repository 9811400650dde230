"""The multi-rank logic of bench.py (one process per GPU under torchrun) on
the host: world_size 2 over gloo.  Ranks time their own BFS roots (disjoint
slices of one seeded stream), the reported time is the max over ranks and
the work the sum."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    try:
        import bench

        d = bench.Dist(world, backend="gloo")
        mx = d.reduce(float(rank + 1), "max")
        sm = d.reduce(float(rank + 1), "sum")
        d.barrier()
        degree = np.ones(1 << 16, np.int32)
        degree[::3] = 0
        roots = bench.splitmix64_roots(degree, 4, seed=1, skip=rank * 4)
        d.close()
        q.put((rank, mx, sm, roots, None))
    except Exception as e:  # reported to the parent
        q.put((rank, None, None, None, repr(e)))


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        rank, mx, sm, roots, err = q.get(timeout=120)
        assert err is None, err
        out[rank] = (mx, sm, roots)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0] == 2.0
    assert out[0][1] == out[1][1] == 3.0
    import bench

    degree = np.ones(1 << 16, np.int32)
    degree[::3] = 0
    stream = bench.splitmix64_roots(degree, 8, seed=1)
    assert out[0][2] == stream[:4] and out[1][2] == stream[4:]
    assert all(degree[r] > 0 for r in stream)
