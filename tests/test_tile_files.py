"""The reference's on-disk layouts read through the C ABI (gs_read_tile_files,
host code only): the single .start/.grid of "-c 1", and the per-file
.start.N/.grid.N directory layout of "-c 3" (grid::post_grid_dir and
save_start_files(is_odir), gstore.cpp:688-879, 2837-2898), written here by
the reference's own converter.  The multi-file layout only exists for
V >= 2^25 (file blocks of 2^25 vertices), so a Graph500 Kron 16 edge list is
spread over 2^26 vertices; decoded, it must give the same .start, .degree
and per-tile records as the reference's "-c 1" output of the same edges."""
import os

import numpy as np
import pytest

V = 1 << 26


@pytest.mark.parametrize("kind", ["u", "d"])
def test_multi_file_layout_matches_single_file(reference_layouts, kind):
    import gstore_b200 as gs

    single, multi = reference_layouts[kind]
    directed = kind == "d"
    nfiles = len(list(multi.parent.glob("gstore.grid.*")))
    assert nfiles == (4 if directed else 3)               # 2 x 2 file blocks (upper triangle for gstoreu)
    s1, g1, d1 = gs.read_tiles(single, V, directed)
    s3, g3, d3 = gs.read_tiles(multi, V, directed)
    assert np.array_equal(s1, s3)
    assert np.array_equal(d1, d3)
    assert g1.size == g3.size == s1[-1]
    for t in np.nonzero(np.diff(s1))[0]:
        a, b = int(s1[t]), int(s1[t + 1])
        assert np.array_equal(np.sort(g1[a:b]), np.sort(g3[a:b])), f"tile {t}"
    # the decoder needs the writer's running sums, not an ordinary prefix sum
    raw = np.fromfile(str(multi) + ".start.0", np.uint64)
    assert raw[-1] > np.fromfile(str(multi) + ".grid.0", np.uint32).size


def test_multi_file_layout_errors(reference_layouts, tmp_path):
    import gstore_b200 as gs

    _, multi = reference_layouts["u"]
    bad = tmp_path / "gstore"
    for f in multi.parent.glob("gstore.*"):
        if f.name != "gstore.grid.1":
            os.symlink(f, tmp_path / f.name)
    with pytest.raises(gs.GStoreError, match="GS_ERR_ARG"):      # a missing .grid.N
        gs.read_tiles(bad, V)
    g1 = np.fromfile(multi.parent / "gstore.grid.1", np.uint32)
    g1[:-1].tofile(tmp_path / "gstore.grid.1")                     # one record short
    with pytest.raises(gs.GStoreError, match="GS_ERR_FORMAT"):
        gs.read_tiles(bad, V)
