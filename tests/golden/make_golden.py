"""Generate the golden fixtures under tests/golden from the reference itself.

Runs in a container that has the reference sources: ``make -C oracle ref``
compiles the G-Store reference (gstoreu/gstored, a harness around its
algorithm classes) and the Graph500 generator from their own sources into
``oracle/_ref``.  Each fixture holds the tile files the reference converter
wrote and the per-vertex arrays the reference's own code computed on them:

  bfs_depth[r]   bfs_t depth_t array for root bfs_roots[r]     (bfs.cpp)
  kcore_deg[i]   kcore_t final vert_degree for k = kcore_k[i]   (kcore.cpp)
  wcc_label      wcc2_t vert_cid, canonicalised to the smallest vertex id
                 of each component                              (wcc.cpp)
  pr_compat_x    pr_t vert_rank_prior after 5 iterations        (pr.cpp),
                 i.e. with the reference's int32 inverse degree
  bfs2_depth[r]  bfs2_t depth_t array for root bfs_roots[r]    (bfs2.cpp)
  traverse_cid[r] traverse_t vert_cid from pivot bfs_roots[r]  (traverse.cpp)

Graphs: Graph500 Kronecker (seeds 1, 2) and small hand-made edge lists that
exercise several tile windows, a ragged last window, self-loops, duplicates,
isolated vertices and a long path.

usage: python tests/golden/make_golden.py
"""
from __future__ import annotations

import re
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent


def spread(pairs: np.ndarray, factor: int, bits: int) -> np.ndarray:
    """Injective relabelling v -> (v * factor + v % factor) mod 2^bits that
    spreads a small graph's ids over several 2^16-vertex tile windows."""
    v = pairs.astype(np.uint64)
    out = (v * factor + (v % factor)) % (1 << bits)
    return out.astype(np.uint32)


def handmade() -> tuple[np.ndarray, int]:
    """Edge cases: ragged last window, self-loops, duplicates, isolated
    vertices, a 200-edge path, a star hub, edges touching vertex V-1."""
    V = 2 * 65536 + 37
    rng = np.random.default_rng(7)
    e = []
    path = np.arange(1000, 1000 + 201 * 211, 211) % V          # 200-edge path across windows
    e += list(zip(path[:-1], path[1:]))
    hub = 70000
    e += [(hub, int(x)) for x in rng.integers(0, V, 500)]       # star
    e += [(5, 5), (131000, 131000)]                              # self-loops (dropped)
    e += [(1, 2)] * 5                                            # duplicates
    e += [(V - 1, 3), (V - 1, V - 2), (65535, 65536)]            # window borders, last vertex
    e += [(int(a), int(b)) for a, b in rng.integers(0, V, (2000, 2))]
    e += [(120000, 120001), (120001, 120002)]                    # a small separate component
    pairs = np.array(e, np.uint32)
    return pairs, V


def reference_arrays(prefix: Path, V: int, directed: bool, roots, ks):
    d = {}
    depth = []
    levels = []
    for r in roots:
        arr, out = O.ref_run(prefix, V, "bfs", int(r), directed)
        depth.append(arr)
        levels.append([int(m) for m in re.findall(r"frontier count: (\d+)", out)])
    d["bfs_roots"] = np.array(roots, np.uint64)
    d["bfs_depth"] = np.stack(depth)
    d["bfs_ref_level_counts"] = np.array([np.pad(l, (0, 256 - len(l))) for l in levels], np.int64)
    cid, out = O.ref_run(prefix, V, "wcc", 0, directed)
    d["wcc_label"] = O.canonical_labels(cid)
    d["wcc_count"] = np.int64(re.search(r"WCC count = (\d+)", out).group(1))
    if not directed:
        kd, counts = [], []
        for k in ks:
            arr, out = O.ref_run(prefix, V, "kcore", int(k), directed)
            kd.append(arr)
            m = re.search(r"vertices count = (\d+)", out)
            counts.append(int(m.group(1)) if m else -1)
        d["kcore_k"] = np.array(ks, np.int32)
        d["kcore_deg"] = np.stack(kd)
        d["kcore_count"] = np.array(counts, np.int64)
    x, _ = O.ref_run(prefix, V, "pr", 5, directed)
    d["pr_compat_x"] = x
    d["bfs2_depth"] = np.stack([O.ref_run(prefix, V, "bfs2", int(r), directed)[0] for r in roots])
    d["traverse_cid"] = np.stack([O.ref_run(prefix, V, "traverse", int(r), directed)[0] for r in roots])
    return d


def make(name: str, pairs: np.ndarray, V: int, directed: bool, roots, ks, tmp: Path):
    edge_file = tmp / f"{name}.bin"
    pairs.astype(np.uint32).tofile(edge_file)
    prefix = tmp / name
    O.ref_convert(edge_file, prefix, V, directed)
    start = np.fromfile(str(prefix) + ".start", np.uint64)
    grid = np.fromfile(str(prefix) + ".grid", np.uint32)
    degree = np.fromfile(str(prefix) + ".degree", np.int32)
    d = dict(V=np.int64(V), directed=np.int64(directed), pairs=pairs.astype(np.uint32),
             start=start, grid=grid, degree=degree)
    d.update(reference_arrays(prefix, V, directed, roots, ks))
    np.savez_compressed(OUT / f"{name}.npz", **d)
    print(f"{name}: V={V} records={grid.size} tiles={np.count_nonzero(np.diff(start))}")


def main():
    if not O.ref_available():
        O.build(quiet=False)
    assert O.ref_available(), "the reference could not be built (oracle/_ref)"
    with tempfile.TemporaryDirectory() as t:
        tmp = Path(t)
        k12 = O.ref_generate(12, 16, tmp / "k12.bin")
        deg = np.bincount(k12.ravel(), minlength=4096)
        rng = np.random.default_rng(1)
        roots = [1] + [int(x) for x in rng.choice(np.nonzero(deg)[0], 3, replace=False)]
        make("kron12", k12, 4096, False, roots, [2, 4, 8, 16, 32], tmp)
        make("kron12d", k12, 4096, True, roots, [], tmp)
        s18 = spread(k12, 64, 18)
        deg = np.bincount(s18.ravel(), minlength=1 << 18)
        roots = [int(s18[0, 0])] + [int(x) for x in rng.choice(np.nonzero(deg)[0], 3, replace=False)]
        make("spread18", s18, 1 << 18, False, roots, [2, 8, 16], tmp)
        make("spread18d", s18, 1 << 18, True, roots, [], tmp)
        hm, V = handmade()
        make("handmade", hm, V, False, [1000, 70000, V - 1, 120000], [2, 3, 8], tmp)
        make("handmade_d", hm, V, True, [1000, 70000], [], tmp)


if __name__ == "__main__":
    main()
