"""gstore_b200 — B200-native engine for G-Store's tile-grid edge scan.

Python face of ``libgstore_cuda.so`` (declared in ``include/gstore_cuda.h``):
a thin ctypes layer over the C ABI, used by the tests and the benchmark.  The
reference-compatible host (``gstoreu``/``gstored`` and the ``algo_t`` adapters)
is C++ under ``csrc/host``; this module mirrors the same objects:

* :class:`Context`  — ``gs_create``: device, HBM tile budget, directed flag
* :class:`Graph`    — a resident tile grid (``read_grid_in_mem`` +
  ``read_degree_in_mem``, gstore.cpp:2953-3011)
* :class:`State`    — one algorithm run with the ``algo_t`` protocol
  (``init`` / ``algo_mem_part`` = :meth:`State.sweep` /
  ``iteration_finalize`` = :meth:`State.finalize`, algo.h:38-44)

There is no CPU fallback: if the CUDA library is missing or no GPU is
present, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libgstore_cuda.so"

GS_ALGO_BFS, GS_ALGO_PAGERANK, GS_ALGO_KCORE, GS_ALGO_WCC, GS_ALGO_BFS2, GS_ALGO_TRAVERSE = 0, 1, 2, 3, 4, 5
ALGOS = {"bfs": GS_ALGO_BFS, "pagerank": GS_ALGO_PAGERANK, "pr": GS_ALGO_PAGERANK,
         "kcore": GS_ALGO_KCORE, "wcc": GS_ALGO_WCC, "bfs2": GS_ALGO_BFS2, "traverse": GS_ALGO_TRAVERSE}
_RESULT_DTYPE = {GS_ALGO_BFS: np.uint8, GS_ALGO_PAGERANK: np.float32, GS_ALGO_KCORE: np.int32,
                 GS_ALGO_WCC: np.uint32, GS_ALGO_BFS2: np.uint8, GS_ALGO_TRAVERSE: np.uint32}
STATUS = {0: "GS_OK", 1: "GS_ERR_CUDA", 2: "GS_ERR_OOM", 3: "GS_ERR_FORMAT", 4: "GS_ERR_TIMEOUT",
          5: "GS_ERR_ARG", 6: "GS_ERR_RANGE", 7: "GS_ERR_STATE", 8: "GS_ERR_UNSUPPORTED"}

# Every exported symbol of the C ABI, as declared in include/gstore_cuda.h.
ABI_SYMBOLS = [
    "gs_create", "gs_destroy", "gs_last_error", "gs_set_stream", "gs_profile", "gs_kernel_time",
    "gs_launch_count",
    "gs_geometry", "gs_upload_graph", "gs_upload_graph_device", "gs_graph_free", "gs_graph_info",
    "gs_graph_degree", "gs_state_create", "gs_state_free", "gs_state_reset", "gs_sweep", "gs_finalize", "gs_run",
    "gs_download", "gs_result_count", "gs_bfs_stats", "gs_bfs_records_read", "gs_pagerank_compat",
    "gs_kron_generate_device", "gs_kron_generate", "gs_convert", "gs_graph_download",
    "gs_bfs_noalloc", "gs_upload_graph_streamed", "gs_upload_graph_file", "gs_stream_stats",
    "gs_read_tile_files", "gs_upload_graph_files",
    "gs_batch_create", "gs_batch_add", "gs_batch_run", "gs_batch_download", "gs_batch_result_count",
    "gs_batch_bfs_levels", "gs_batch_stats", "gs_batch_free",
    "gs_serve_create", "gs_serve_add_graph", "gs_serve_submit", "gs_serve_step", "gs_serve_poll",
    "gs_serve_result", "gs_serve_clock", "gs_serve_stats", "gs_serve_free", "gs_serve_completed",
    "gs_serve_set_side_streams", "gs_serve_result_view", "gs_serve_release", "gs_serve_profile",
    "gs_serve_reserve_host",
]


class GStoreError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


_lib = None


def lib():
    """Load libgstore_cuda.so (built in-tree by ``python -m gstore_b200.build``)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"CUDA engine not built: {LIB_PATH} is missing "
                               "(run python -m gstore_b200.build)")
        L = C.CDLL(str(LIB_PATH))
        vp, u64, i64, i32 = C.c_void_p, C.c_uint64, C.c_int64, C.c_int
        pvp = C.POINTER(C.c_void_p)
        pu64 = C.POINTER(C.c_uint64)
        sig = {
            "gs_create": [pvp, i32, u64, i32],
            "gs_destroy": [vp],
            "gs_set_stream": [vp, vp],
            "gs_profile": [vp, i32],
            "gs_kernel_time": [vp, i32, pu64, C.POINTER(C.c_double), pu64],
            "gs_launch_count": [vp, pu64],
            "gs_geometry": [u64, i32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), pu64],
            "gs_upload_graph": [vp, vp, u64, vp, u64, vp, u64, pvp],
            "gs_upload_graph_device": [vp, vp, u64, vp, u64, vp, u64, pvp],
            "gs_graph_free": [vp],
            "gs_graph_info": [vp, pu64, pu64, pu64, pu64],
            "gs_graph_degree": [vp, vp],
            "gs_state_create": [vp, i32, i64, pvp],
            "gs_state_free": [vp],
            "gs_state_reset": [vp, i64],
            "gs_sweep": [vp, vp, i32],
            "gs_finalize": [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int)],
            "gs_run": [vp, C.POINTER(C.c_int64)],
            "gs_download": [vp, i32, vp, u64],
            "gs_result_count": [vp, pu64],
            "gs_bfs_stats": [vp, pu64, vp, i32, C.POINTER(C.c_int), vp],
            "gs_bfs_records_read": [vp, vp, i32, C.POINTER(C.c_int)],
            "gs_pagerank_compat": [vp, i32],
            "gs_kron_generate_device": [vp, i32, i64, u64, u64, vp],
            "gs_kron_generate": [vp, i32, i64, u64, u64, vp],
            "gs_convert": [vp, vp, u64, i32, u64, pvp],
            "gs_graph_download": [vp, vp, vp, vp],
            "gs_bfs_noalloc": [vp, u64, vp, C.POINTER(C.c_int64)],
            "gs_upload_graph_streamed": [vp, vp, u64, vp, u64, vp, u64, u64, pvp],
            "gs_upload_graph_file": [vp, vp, u64, C.c_char_p, u64, vp, u64, u64, pvp],
            "gs_stream_stats": [vp, pu64, pu64, pu64, pu64],
            "gs_read_tile_files": [vp, C.c_char_p, u64, i32, vp, u64, vp, u64, vp, pu64],
            "gs_upload_graph_files": [vp, C.c_char_p, u64, u64, pvp],
            "gs_batch_create": [vp, pvp],
            "gs_batch_add": [vp, vp, i32, i64, C.POINTER(C.c_int)],
            "gs_batch_run": [vp],
            "gs_batch_download": [vp, i32, i32, vp, u64],
            "gs_batch_result_count": [vp, i32, pu64],
            "gs_batch_bfs_levels": [vp, i32, vp, i32, C.POINTER(C.c_int)],
            "gs_batch_stats": [vp, pu64, C.POINTER(C.c_double)],
            "gs_batch_free": [vp],
            "gs_serve_create": [vp, u64, pvp],
            "gs_serve_add_graph": [vp, vp, C.POINTER(C.c_int)],
            "gs_serve_submit": [vp, i32, i32, i64, pu64],
            "gs_serve_step": [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)],
            "gs_serve_poll": [vp, u64, C.POINTER(C.c_int)],
            "gs_serve_result": [vp, u64, vp, u64, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                C.POINTER(C.c_int64)],
            "gs_serve_clock": [vp, C.POINTER(C.c_double)],
            "gs_serve_stats": [vp, pu64, pu64, pu64, pu64],
            "gs_serve_free": [vp],
            "gs_serve_completed": [vp, pu64, i32, C.POINTER(C.c_int)],
            "gs_serve_set_side_streams": [vp, i32],
            "gs_serve_result_view": [vp, u64, C.POINTER(C.c_void_p), pu64, C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), C.POINTER(C.c_int64)],
            "gs_serve_release": [vp, u64],
            "gs_serve_profile": [vp, C.POINTER(C.c_double), i32],
            "gs_serve_reserve_host": [vp, u64],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int32
        L.gs_last_error.argtypes = [vp]
        L.gs_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays must be C-contiguous"
    return a.ctypes.data_as(C.c_void_p)


def geometry(V: int, directed: bool = False):
    """(p, p_s, number of .start entries) for vertex count V (grid::init -v)."""
    p, ps, n = C.c_uint32(), C.c_uint32(), C.c_uint64()
    lib().gs_geometry(V, int(directed), C.byref(p), C.byref(ps), C.byref(n))
    return p.value, ps.value, n.value


def part_id(gi: int, gj: int, si: int, sj: int, p: int) -> int:
    """The reference's part id of tile (si, sj) in group (gi, gj):
    group_full_index << 16 | si << 8 | sj (get_ij, gstore.h:199-220)."""
    return ((gi * p + gj) << 16) | (si << 8) | sj


def read_tile_files(prefix, V: int | None = None, with_degree: bool = True):
    """Read <prefix>.start / .grid / .degree as the reference writes them."""
    prefix = str(prefix)
    start = np.fromfile(prefix + ".start", np.uint64)
    grid = np.fromfile(prefix + ".grid", np.uint32)
    degree = None
    if with_degree and os.path.exists(prefix + ".degree"):
        degree = np.fromfile(prefix + ".degree", np.int32, count=-1 if V is None else V)
    return start, grid, degree


def read_tiles(prefix, V: int, directed: bool = False, with_grid: bool = True, ctx=None):
    """(start, grid, degree) of the tile files at `prefix` through the C ABI
    (gs_read_tile_files): the single .start/.grid layout, or the per-file
    .start.N/.grid.N layout of the reference's "-c 3" converter decoded into
    the single-file .start and record order.  Host-only: needs no GPU."""
    n = C.c_uint64()
    pre = str(prefix).encode()
    h = ctx._h if ctx is not None else None

    def check(st):
        if st != 0:
            msg = lib().gs_last_error(h).decode() if h else "see the status"
            raise GStoreError(st, f"reading {prefix}: {msg}")

    check(lib().gs_read_tile_files(h, pre, V, int(directed), None, 0, None, 0, None, C.byref(n)))
    start = np.empty(geometry(V, directed)[2], np.uint64)
    grid = np.empty(n.value if with_grid else 0, np.uint32)
    degree = np.empty(V, np.int32)
    check(lib().gs_read_tile_files(h, pre, V, int(directed), _ptr(start), start.size,
                                   _ptr(grid) if with_grid else None, grid.size, _ptr(degree), C.byref(n)))
    return start, (grid if with_grid else None), degree


def write_tile_files(prefix, start, grid, degree):
    """Write .grid/.start/.degree (grid::save_grid, gstore.cpp:2818-2917)."""
    prefix = str(prefix)
    np.ascontiguousarray(grid, np.uint32).tofile(prefix + ".grid")
    np.ascontiguousarray(start, np.uint64).tofile(prefix + ".start")
    if degree is not None:
        np.ascontiguousarray(degree, np.int32).tofile(prefix + ".degree")


class Context:
    """A device context (gs_create)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0, directed: bool = False):
        self._h = C.c_void_p()
        self._children = weakref.WeakSet()   # graphs, states, batches made from this context
        st = lib().gs_create(C.byref(self._h), device, hbm_budget, int(directed))
        if st != 0:
            raise GStoreError(st, "gs_create failed (no usable CUDA device?)")
        self.directed = bool(directed)

    def _check(self, st):
        if st != 0:
            raise GStoreError(st, lib().gs_last_error(self._h).decode())

    def close(self):
        """Free every object made from this context, then the context
        (gs_destroy does not free graphs, states or batches)."""
        if self._h:
            kids = list(self._children)
            for kind in (State, Batch, Server, Graph):
                for k in kids:
                    if isinstance(k, kind):
                        k.free()
            lib().gs_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, cuda_stream_ptr: int | None):
        self._check(lib().gs_set_stream(self._h, C.c_void_p(cuda_stream_ptr or 0)))

    def profile(self, enable: bool = True):
        self._check(lib().gs_profile(self._h, int(enable)))

    def kernel_time(self, algo: int):
        n, ms, b = C.c_uint64(), C.c_double(), C.c_uint64()
        self._check(lib().gs_kernel_time(self._h, algo, C.byref(n), C.byref(ms), C.byref(b)))
        return n.value, ms.value, b.value

    def launches(self) -> int:
        """Kernels launched by this context so far."""
        n = C.c_uint64()
        self._check(lib().gs_launch_count(self._h, C.byref(n)))
        return n.value

    def upload(self, start, grid, degree, V: int) -> "Graph":
        start = np.ascontiguousarray(start, np.uint64)
        grid = np.ascontiguousarray(grid, np.uint32)
        if degree is not None:
            degree = np.ascontiguousarray(degree, np.int32)
            assert degree.size >= V, "degree array shorter than V"
        h = C.c_void_p()
        self._check(lib().gs_upload_graph(self._h, _ptr(start), start.size, _ptr(grid), grid.size,
                                          _ptr(degree), V, C.byref(h)))
        # over the HBM budget the graph streams from `grid`: keep it alive
        return Graph(self, h, keep=grid)

    def upload_streamed(self, start, grid, degree, V: int, segment_bytes: int) -> "Graph":
        """A graph whose records stay in host memory (`grid`, pinned by the
        library unless it already is) and stream through two HBM segments of
        segment_bytes each on every sweep."""
        start = np.ascontiguousarray(start, np.uint64)
        if not (isinstance(grid, np.ndarray) and grid.dtype == np.uint32 and grid.flags["C_CONTIGUOUS"]):
            grid = np.ascontiguousarray(grid, np.uint32)
        if degree is not None:
            degree = np.ascontiguousarray(degree, np.int32)
            assert degree.size >= V, "degree array shorter than V"
        h = C.c_void_p()
        self._check(lib().gs_upload_graph_streamed(self._h, _ptr(start), start.size, _ptr(grid), grid.size,
                                                   _ptr(degree), V, segment_bytes, C.byref(h)))
        return Graph(self, h, keep=grid)

    def upload_file(self, start, grid_path, n_edges: int, degree, V: int, segment_bytes: int) -> "Graph":
        """A graph whose records stay in the .grid file at grid_path and are
        read into two pinned staging buffers, then copied through two HBM
        segments of segment_bytes each, on every sweep."""
        start = np.ascontiguousarray(start, np.uint64)
        if degree is not None:
            degree = np.ascontiguousarray(degree, np.int32)
            assert degree.size >= V, "degree array shorter than V"
        h = C.c_void_p()
        self._check(lib().gs_upload_graph_file(self._h, _ptr(start), start.size, str(grid_path).encode(), n_edges,
                                               _ptr(degree), V, segment_bytes, C.byref(h)))
        return Graph(self, h)

    def read_tile_files(self, prefix, V: int, with_grid: bool = True):
        """read_tiles(prefix, V, directed=this context's grid kind)."""
        return read_tiles(prefix, V, self.directed, with_grid, ctx=self)

    def upload_files(self, prefix, V: int, segment_bytes: int) -> "Graph":
        """A graph whose records stay in the tile file(s) at `prefix` (either
        layout) and stream through two HBM segments (gs_upload_graph_files)."""
        h = C.c_void_p()
        self._check(lib().gs_upload_graph_files(self._h, str(prefix).encode(), V, segment_bytes, C.byref(h)))
        return Graph(self, h)

    def upload_device(self, d_start: int, n_start: int, d_grid: int, n_edges: int, d_degree: int | None,
                      V: int) -> "Graph":
        h = C.c_void_p()
        self._check(lib().gs_upload_graph_device(self._h, C.c_void_p(d_start), n_start, C.c_void_p(d_grid),
                                                 n_edges, C.c_void_p(d_degree or 0), V, C.byref(h)))
        return Graph(self, h)

    def kron_generate(self, scale: int, edgefactor: int = 16, seed1: int = 1, seed2: int = 2) -> np.ndarray:
        out = np.empty(((edgefactor << scale), 2), np.uint32)
        self._check(lib().gs_kron_generate(self._h, scale, edgefactor, seed1, seed2, _ptr(out)))
        return out

    def kron_generate_device(self, scale: int, edgefactor: int, seed1: int, seed2: int, d_pairs: int):
        self._check(lib().gs_kron_generate_device(self._h, scale, edgefactor, seed1, seed2,
                                                  C.c_void_p(d_pairs)))

    def convert(self, pairs, V: int, n_pairs: int | None = None) -> "Graph":
        """Edge pairs (numpy (m,2) uint32 on the host, or an int device pointer
        with n_pairs) -> resident graph (the "-c 1" converter)."""
        h = C.c_void_p()
        if isinstance(pairs, int):
            self._check(lib().gs_convert(self._h, C.c_void_p(pairs), n_pairs, 1, V, C.byref(h)))
        else:
            pairs = np.ascontiguousarray(pairs, np.uint32)
            self._check(lib().gs_convert(self._h, _ptr(pairs), pairs.size // 2, 0, V, C.byref(h)))
        return Graph(self, h)


class Batch:
    """Queries run together (gs_batch): multi-source BFS groups, WCC and
    k-core queries over several graphs in one persistent launch."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        self._h = C.c_void_p()
        ctx._check(lib().gs_batch_create(ctx._h, C.byref(self._h)))
        self._graphs = {}
        ctx._children.add(self)

    def add(self, graph: "Graph", algo, arg: int = 0) -> int:
        a = ALGOS[algo] if isinstance(algo, str) else int(algo)
        qid = C.c_int()
        self.ctx._check(lib().gs_batch_add(self._h, graph._h, a, arg, C.byref(qid)))
        self._graphs[qid.value] = (graph, a)
        return qid.value

    def run(self):
        self.ctx._check(lib().gs_batch_run(self._h))

    def download(self, qid: int, what: int = 0) -> np.ndarray:
        graph, a = self._graphs[qid]
        dt = _RESULT_DTYPE[a]
        out = np.empty(graph.V, dt)
        self.ctx._check(lib().gs_batch_download(self._h, qid, what, _ptr(out), out.nbytes))
        return out

    def count(self, qid: int) -> int:
        c = C.c_uint64()
        self.ctx._check(lib().gs_batch_result_count(self._h, qid, C.byref(c)))
        return c.value

    def bfs_levels(self, qid: int) -> np.ndarray:
        out = np.zeros(256, np.uint64)
        n = C.c_int()
        self.ctx._check(lib().gs_batch_bfs_levels(self._h, qid, _ptr(out), 256, C.byref(n)))
        return out[: n.value].copy()

    def stats(self):
        n, ms = C.c_uint64(), C.c_double()
        self.ctx._check(lib().gs_batch_stats(self._h, C.byref(n), C.byref(ms)))
        return {"launches": n.value, "kernel_ms": ms.value}

    def free(self):
        if self._h:
            lib().gs_batch_free(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.free()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Server:
    """Request loop over resident graphs (gs_serve_*): continuous batching of
    BFS / WCC / k-core / PageRank requests, admitted by HBM footprint."""

    QUEUED, RUNNING, DONE, FAILED = 0, 1, 2, 3

    def __init__(self, ctx: Context, state_budget: int = 0):
        self.ctx = ctx
        self._h = C.c_void_p()
        ctx._check(lib().gs_serve_create(ctx._h, state_budget, C.byref(self._h)))
        self._graphs = []
        self._req = {}
        ctx._children.add(self)

    def add_graph(self, graph: "Graph") -> int:
        gid = C.c_int()
        self.ctx._check(lib().gs_serve_add_graph(self._h, graph._h, C.byref(gid)))
        self._graphs.append(graph)
        return gid.value

    def submit(self, gid: int, algo, arg: int = 0) -> int:
        a = ALGOS[algo] if isinstance(algo, str) else int(algo)
        rid = C.c_uint64()
        self.ctx._check(lib().gs_serve_submit(self._h, gid, a, arg, C.byref(rid)))
        self._req[rid.value] = (gid, a)
        return rid.value

    def step(self):
        """One serving step; returns (running, queued)."""
        na, nq = C.c_int(), C.c_int()
        self.ctx._check(lib().gs_serve_step(self._h, C.byref(na), C.byref(nq)))
        return na.value, nq.value

    def completed(self, max_ids: int = 4096):
        """Ids of requests finished since the last call, oldest first."""
        buf = (C.c_uint64 * max_ids)()
        n = C.c_int()
        out = []
        while True:
            self.ctx._check(lib().gs_serve_completed(self._h, buf, max_ids, C.byref(n)))
            out.extend(buf[: n.value])
            if n.value < max_ids:
                return out

    def set_side_streams(self, n: int) -> None:
        self.ctx._check(lib().gs_serve_set_side_streams(self._h, n))

    def poll(self, rid: int) -> int:
        st = C.c_int()
        self.ctx._check(lib().gs_serve_poll(self._h, rid, C.byref(st)))
        return st.value

    def result(self, rid: int, want_data: bool = True):
        """(result array or None, t_submit, t_done, steps); forgets the request."""
        gid, a = self._req.pop(rid)
        V = self._graphs[gid].V
        dt = _RESULT_DTYPE[a]
        out = np.empty(V, dt) if want_data else None
        ts, td, n = C.c_double(), C.c_double(), C.c_int64()
        self.ctx._check(lib().gs_serve_result(self._h, rid, _ptr(out), 0 if out is None else out.nbytes,
                                              C.byref(ts), C.byref(td), C.byref(n)))
        return out, ts.value, td.value, n.value

    def result_view(self, rid: int):
        """(result array viewing the server's pinned buffer, t_submit, t_done,
        steps) without a copy; the array is valid until release(rid)."""
        gid, a = self._req[rid]
        dt = np.dtype(_RESULT_DTYPE[a])
        p, nb = C.c_void_p(), C.c_uint64()
        ts, td, n = C.c_double(), C.c_double(), C.c_int64()
        try:
            self.ctx._check(lib().gs_serve_result_view(self._h, rid, C.byref(p), C.byref(nb), C.byref(ts),
                                                       C.byref(td), C.byref(n)))
        except GStoreError:
            self._req.pop(rid)        # a failed request is forgotten by the server
            raise
        buf = (C.c_char * nb.value).from_address(p.value)
        return np.frombuffer(buf, dt), ts.value, td.value, n.value

    def release(self, rid: int) -> None:
        self._req.pop(rid)
        self.ctx._check(lib().gs_serve_release(self._h, rid))

    def clock(self) -> float:
        t = C.c_double()
        self.ctx._check(lib().gs_serve_clock(self._h, C.byref(t)))
        return t.value

    def stats(self):
        a, b, c, d = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint64()
        self.ctx._check(lib().gs_serve_stats(self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(d)))
        return {"steps": a.value, "graph_launches": b.value, "kernel_launches": c.value, "hbm_in_use": d.value}

    def profile(self):
        """Host seconds in gs_serve_step by phase, and the pool misses
        (pinned host and device allocations) made inside those phases."""
        out = (C.c_double * 8)()
        self.ctx._check(lib().gs_serve_profile(self._h, out, 8))
        return {"admit_s": out[0], "step_launch_s": out[1], "side_s": out[2], "step_finish_s": out[3],
                "pinned_alloc_s": out[4], "pinned_allocs": int(out[5]), "device_alloc_s": out[6],
                "device_allocs": int(out[7])}

    def reserve_host(self, nbytes: int):
        """Pins nbytes into the server's result arena ahead of the requests."""
        self.ctx._check(lib().gs_serve_reserve_host(self._h, int(nbytes)))

    def free(self):
        if self._h:
            lib().gs_serve_free(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.free()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Graph:
    """A resident tile grid (gs_graph)."""

    def __init__(self, ctx: Context, handle, keep=None):
        self.ctx = ctx
        self._h = handle
        self._keep = keep        # host records of a streamed graph
        ctx._children.add(self)
        e, t, i, v = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint64()
        ctx._check(lib().gs_graph_info(self._h, C.byref(e), C.byref(t), C.byref(i), C.byref(v)))
        self.n_edges, self.n_tiles, self.n_items, self.V = e.value, t.value, i.value, v.value
        self.directed = ctx.directed

    def free(self):
        if self._h:
            lib().gs_graph_free(self._h)
            self._h = None
        self._keep = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def stream_stats(self) -> dict:
        """Host-to-device traffic of a streamed graph since upload."""
        b, c, sg, r = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint64()
        self.ctx._check(lib().gs_stream_stats(self._h, C.byref(b), C.byref(c), C.byref(sg), C.byref(r)))
        return {"bytes": b.value, "copies": c.value, "segments": sg.value, "reused": r.value}

    def degree(self) -> np.ndarray:
        out = np.empty(self.V, np.int32)
        self.ctx._check(lib().gs_graph_degree(self._h, _ptr(out)))
        return out

    def download(self):
        _, _, ns = geometry(self.V, self.directed)
        start = np.empty(ns, np.uint64)
        grid = np.empty(self.n_edges, np.uint32)
        degree = np.empty(self.V, np.int32)
        self.ctx._check(lib().gs_graph_download(self._h, _ptr(start), _ptr(grid), _ptr(degree)))
        return start, grid, degree

    def state(self, algo, arg: int = 0) -> "State":
        a = ALGOS[algo] if isinstance(algo, str) else int(algo)
        h = C.c_void_p()
        self.ctx._check(lib().gs_state_create(self._h, a, arg, C.byref(h)))
        return State(self, h, a)

    def bfs_noalloc(self, root: int, d_depth: int) -> int:
        """BFS into a caller-owned device buffer (uint8, V bytes) without any
        allocation by the library; returns the number of sweeps."""
        n = C.c_int64()
        self.ctx._check(lib().gs_bfs_noalloc(self._h, root, C.c_void_p(d_depth), C.byref(n)))
        return n.value

    # convenience: whole runs ------------------------------------------------
    def bfs(self, root: int) -> np.ndarray:
        with self.state("bfs", root) as s:
            s.run()
            return s.download()

    def pagerank(self, iterations: int = 5, compat: bool = False):
        with self.state("pagerank", iterations) as s:
            if compat:
                s.compat()
            s.run()
            return s.download(0), s.download(1)

    def wcc(self):
        with self.state("wcc") as s:
            s.run()
            return s.download(), s.count()

    def kcore(self, k: int):
        with self.state("kcore", k) as s:
            s.run()
            return s.download(), s.count()


class State:
    """One algorithm run (gs_state): the algo_t protocol on the device."""

    def __init__(self, graph: Graph, handle, algo: int):
        self.graph = graph
        self._h = handle
        self.algo = algo
        graph.ctx._children.add(self)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.free()

    def free(self):
        if self._h:
            lib().gs_state_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def _check(self, st):
        self.graph.ctx._check(st)

    def reset(self, arg: int):
        """Start a new run (new root / iterations / k) reusing the device arrays."""
        self._check(lib().gs_state_reset(self._h, arg))

    def compat(self, enable: bool = True):
        self._check(lib().gs_pagerank_compat(self._h, int(enable)))

    def sweep(self, parts=None):
        """algo_mem_part (algo.h:40) over every tile, or over the tiles of
        the given part ranges [(part_start, part_end), ...] (inclusive, in
        file order; ids from part_id)."""
        if not parts:
            self._check(lib().gs_sweep(self._h, None, 0))
            return
        arr = np.ascontiguousarray(np.asarray(parts, np.uint64).reshape(-1, 2))
        self._check(lib().gs_sweep(self._h, _ptr(arr), arr.shape[0]))

    def finalize(self):
        """iteration_finalize(): returns (frontier, done)."""
        f, d = C.c_int64(), C.c_int()
        self._check(lib().gs_finalize(self._h, C.byref(f), C.byref(d)))
        return f.value, bool(d.value)

    def run(self) -> int:
        n = C.c_int64()
        self._check(lib().gs_run(self._h, C.byref(n)))
        return n.value

    def download(self, what: int = 0) -> np.ndarray:
        V = self.graph.V
        dt = _RESULT_DTYPE[self.algo]
        out = np.empty(V, dt)
        self._check(lib().gs_download(self._h, what, _ptr(out), out.nbytes))
        return out

    def download_into(self, out: np.ndarray, what: int = 0) -> np.ndarray:
        """Download into a caller-provided (e.g. pinned) host array."""
        self._check(lib().gs_download(self._h, what, _ptr(out), out.nbytes))
        return out

    def count(self) -> int:
        c = C.c_uint64()
        self._check(lib().gs_result_count(self._h, C.byref(c)))
        return c.value

    def bfs_stats(self, max_levels: int = 256):
        e = C.c_uint64()
        swept = np.zeros(max_levels, np.uint64)
        counts = np.zeros(max_levels, np.uint64)
        nl = C.c_int()
        self._check(lib().gs_bfs_stats(self._h, C.byref(e), _ptr(swept), max_levels, C.byref(nl),
                                       _ptr(counts)))
        n = nl.value
        read = np.zeros(max_levels, np.uint64)
        nr = C.c_int()
        self._check(lib().gs_bfs_records_read(self._h, _ptr(read), max_levels, C.byref(nr)))
        return {"edges_in_component": e.value, "swept": swept[:n].copy(), "level_counts": counts[:n].copy(),
                "read": read[:min(n, nr.value)].copy()}
