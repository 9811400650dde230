"""CPU oracle for the G-Store tile-grid hot path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import this package, and only as the
checker.  The product (``gstore_b200`` and its C-ABI library) never uses it.

Two layers:

* ``liboracle.so`` (``gs_oracle.c``): a sequential C restatement of the
  reference algorithms (BFS ``bfs.cpp``, PageRank ``pr.cpp`` in FP64, WCC
  ``wcc.cpp`` as a partition, k-core ``kcore.cpp`` with its exact int16/negative
  degree rules, the ``-c 1`` converter ``gstore.cpp:1245-1458``).
* ``_ref/``: the reference itself compiled from its own sources (``make ref``)
  -- ``gstoreu``/``gstored``, a harness that dumps the reference's per-vertex
  arrays, and the Graph500 generator driver.  Absent where the reference
  sources are absent; callers check ``ref_available()``.

Parity pins: the restatement is checked against the reference harness and the
committed golden fixtures under ``tests/golden``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"
REF_DIR = HERE / "_ref"

_lib = None


def build(quiet: bool = True, reference_dir: str | None = None) -> None:
    """Compile liboracle.so, and the reference itself under _ref when the
    directory of its sources is given (``reference_dir``, else the
    ``GS_REFERENCE_DIR`` environment variable; there is no default).  A
    directory that is given but holds no reference sources is an error."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", str(HERE), "all"], check=True, stdout=out)
    ref = reference_dir or os.environ.get("GS_REFERENCE_DIR")
    if ref:
        if not (Path(ref) / "gstore.cpp").is_file():
            raise FileNotFoundError(f"oracle.build: {ref} holds no reference sources (gstore.cpp)")
        subprocess.run(["make", "-C", str(HERE), "ref", f"REF={ref}"], check=True, stdout=out)


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        u64p = C.POINTER(C.c_uint64)
        u32p = C.POINTER(C.c_uint32)
        L.orc_geometry.argtypes = [C.c_uint64, C.c_int, u32p, u32p, u64p]
        L.orc_tile_coords.argtypes = [C.c_uint32, C.c_int, C.c_void_p, C.c_void_p]
        L.orc_tile_index.argtypes = [C.c_uint32, C.c_int, C.c_uint32, C.c_uint32]
        L.orc_tile_index.restype = C.c_uint64
        L.orc_bfs.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_uint64,
                              C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                              C.POINTER(C.c_int)]
        L.orc_pagerank.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_int,
                                   C.c_uint64, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        L.orc_wcc.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_uint64,
                              C.c_void_p, u64p]
        L.orc_kcore.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_int,
                                C.c_void_p, u64p, C.c_void_p, C.c_int, C.POINTER(C.c_int)]
        L.orc_convert.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32, C.c_int, C.c_uint64,
                                  C.c_void_p, C.c_void_p, C.c_void_p, u64p]
        L.orc_edges_reached.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_void_p]
        L.orc_edges_reached.restype = C.c_uint64
        L.orc_bfs2.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_uint64, C.c_uint64,
                               C.c_void_p, C.POINTER(C.c_int)]
        L.orc_traverse.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_uint64, C.c_uint64,
                                   C.c_void_p, u64p, C.POINTER(C.c_int)]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)


def geometry(V: int, directed: bool = False):
    p, ps, T = C.c_uint32(), C.c_uint32(), C.c_uint64()
    lib().orc_geometry(V, int(directed), C.byref(p), C.byref(ps), C.byref(T))
    return p.value, ps.value, T.value


def tile_coords(p: int, directed: bool = False):
    _, _, T = geometry(p << 24, directed)
    row = np.empty(T, np.uint32)
    col = np.empty(T, np.uint32)
    lib().orc_tile_coords(p, int(directed), _ptr(row), _ptr(col))
    return row, col


def tile_index(p: int, directed: bool, row: int, col: int) -> int:
    return lib().orc_tile_index(p, int(directed), row, col)


def bfs(start, grid, p, directed, n, root, max_levels=256):
    start = np.ascontiguousarray(start, np.uint64)
    grid = np.ascontiguousarray(grid, np.uint32)
    depth = np.empty(n, np.uint8)
    counts = np.zeros(max_levels, np.uint64)
    swept = np.zeros(max_levels, np.uint64)
    nl = C.c_int()
    st = lib().orc_bfs(_ptr(start), _ptr(grid), p, int(directed), n, root, _ptr(depth),
                       _ptr(counts), _ptr(swept), max_levels, C.byref(nl))
    if st != 0:
        raise ValueError(f"orc_bfs status {st}")
    return depth, counts[: nl.value].copy(), swept[: nl.value].copy()


def edges_reached(start, grid, p, directed, depth) -> int:
    """Records with both ends reached (depth != 0): the GTEPS numerator."""
    start = np.ascontiguousarray(start, np.uint64)
    grid = np.ascontiguousarray(grid, np.uint32)
    depth = np.ascontiguousarray(depth, np.uint8)
    return int(lib().orc_edges_reached(_ptr(start), _ptr(grid), p, int(directed), _ptr(depth)))


def bfs2(start, grid, p, directed, n, root):
    """Label-correcting BFS (-j 30): (u8 depth, sweeps)."""
    start = np.ascontiguousarray(start, np.uint64)
    grid = np.ascontiguousarray(grid, np.uint32)
    depth = np.empty(n, np.uint8)
    ns = C.c_int()
    st = lib().orc_bfs2(_ptr(start), _ptr(grid), p, int(directed), n, root, _ptr(depth), C.byref(ns))
    if st != 0:
        raise ValueError(f"orc_bfs2 status {st}")
    return depth, ns.value


def traverse(start, grid, p, directed, n, pivot):
    """Single-colour propagation (-j 4): (u32 cid, coloured count, sweeps)."""
    start = np.ascontiguousarray(start, np.uint64)
    grid = np.ascontiguousarray(grid, np.uint32)
    cid = np.empty(n, np.uint32)
    cnt, ns = C.c_uint64(), C.c_int()
    st = lib().orc_traverse(_ptr(start), _ptr(grid), p, int(directed), n, pivot, _ptr(cid), C.byref(cnt),
                            C.byref(ns))
    if st != 0:
        raise ValueError(f"orc_traverse status {st}")
    return cid, cnt.value, ns.value


def pagerank(start, grid, degree, p, directed, n, iterations, compat=False):
    start = np.ascontiguousarray(start, np.uint64)
    grid = np.ascontiguousarray(grid, np.uint32)
    degree = np.ascontiguousarray(degree, np.int32)
    r = np.empty(n, np.float64)
    x = np.empty(n, np.float64)
    st = lib().orc_pagerank(_ptr(start), _ptr(grid), _ptr(degree), p, int(directed), n,
                            iterations, int(compat), _ptr(r), _ptr(x))
    if st != 0:
        raise ValueError(f"orc_pagerank status {st}")
    return r, x


def wcc(start, grid, p, directed, n):
    start = np.ascontiguousarray(start, np.uint64)
    grid = np.ascontiguousarray(grid, np.uint32)
    label = np.empty(n, np.uint32)
    cnt = C.c_uint64()
    st = lib().orc_wcc(_ptr(start), _ptr(grid), p, int(directed), n, _ptr(label), C.byref(cnt))
    if st != 0:
        raise ValueError(f"orc_wcc status {st}")
    return label, cnt.value


def kcore(start, grid, degree, p, n, k, max_rounds=4096):
    start = np.ascontiguousarray(start, np.uint64)
    grid = np.ascontiguousarray(grid, np.uint32)
    deg = np.array(degree, np.int32, copy=True)
    mem = C.c_uint64()
    swept = np.zeros(max_rounds, np.uint64)
    nr = C.c_int()
    st = lib().orc_kcore(_ptr(start), _ptr(grid), p, n, k, _ptr(deg), C.byref(mem),
                         _ptr(swept), max_rounds, C.byref(nr))
    if st != 0:
        raise ValueError(f"orc_kcore status {st}")
    return deg, mem.value, swept[: nr.value].copy()


def convert(edges, p, directed, n):
    """edges: (m, 2) uint32 array of (v0, v1) pairs (gedge_t)."""
    edges = np.ascontiguousarray(edges, np.uint32)
    _, _, T = geometry(p << 24, directed)
    start = np.empty(T + 1, np.uint64)
    degree = np.empty(n, np.int32)
    nrec = C.c_uint64()
    L = lib()
    st = L.orc_convert(_ptr(edges), edges.shape[0], p, int(directed), n, _ptr(start), None,
                       _ptr(degree), C.byref(nrec))
    if st != 0:
        raise ValueError(f"orc_convert status {st}")
    grid = np.empty(nrec.value, np.uint32)
    L.orc_convert(_ptr(edges), edges.shape[0], p, int(directed), n, _ptr(start), _ptr(grid),
                  _ptr(degree), C.byref(nrec))
    return start, grid, degree


def canonical_labels(label: np.ndarray) -> np.ndarray:
    """Map any WCC labelling to min-vertex-id per component; 0xFFFFFFFF kept."""
    label = np.asarray(label, np.uint32)
    out = np.full(label.shape, 0xFFFFFFFF, np.uint32)
    valid = label != 0xFFFFFFFF
    idx = np.nonzero(valid)[0]
    if idx.size:
        lab = label[idx]
        order = np.argsort(lab, kind="stable")
        lab_s = lab[order]
        idx_s = idx[order]
        first = np.ones(lab_s.size, bool)
        first[1:] = lab_s[1:] != lab_s[:-1]
        grp = np.cumsum(first) - 1
        mins = np.minimum.reduceat(idx_s, np.nonzero(first)[0])
        out[idx_s] = mins[grp].astype(np.uint32)
    return out


# ------------------------------------------------------ reference (_ref) ---
def ref_available() -> bool:
    return (REF_DIR / "ref_harness_u").exists() and (REF_DIR / "kron_gen_ref").exists()


def ref_generate(scale: int, edgefactor: int, out: Path, seed1: int = 1, seed2: int = 2) -> np.ndarray:
    subprocess.run([str(REF_DIR / "kron_gen_ref"), str(scale), str(edgefactor), str(out),
                    str(seed1), str(seed2)], check=True)
    return np.fromfile(out, np.uint32).reshape(-1, 2)


def ref_convert(edge_file: Path, prefix: Path, V: int, directed: bool = False) -> str:
    exe = REF_DIR / ("gstored" if directed else "gstoreu")
    r = subprocess.run([str(exe), "-v", str(V), "-c", "1", "-i", str(edge_file), "-o", str(prefix)],
                       check=True, capture_output=True, text=True)
    return r.stdout


def ref_run(prefix: Path, V: int, algo: str, arg: int, directed: bool = False):
    """Run the reference's own algorithm class on tile files; returns (array, stdout).
    Runs with different (algo, arg) may go on concurrently."""
    exe = REF_DIR / ("ref_harness_d" if directed else "ref_harness_u")
    out = Path(str(prefix) + f".{algo}.{arg}.out")
    r = subprocess.run([str(exe), str(prefix), str(V), algo, str(arg), str(out)],
                       check=True, capture_output=True, text=True)
    dt = {"bfs": np.uint8, "kcore": np.int32, "wcc": np.uint32, "pr": np.float32, "bfs2": np.uint8,
          "traverse": np.uint32}[algo]
    arr = np.fromfile(out, dt)
    out.unlink()
    return arr, r.stdout
