// Tile files on disk (host code of libgstore_cuda.so): the reference's loaders
// read_start_in_mem / read_grid_in_mem / read_degree_in_mem
// (gstore.cpp:2953-3011, 3799-3813) for the single-file layout that "-c 1"
// and "-c 2" write, and a reader for the multi-file layout that "-c 3" writes
// into a directory (grid::post_grid_dir + save_start_files(is_odir),
// gstore.cpp:688-879, 2837-2898), which the reference itself never reads back.
//
// The multi-file layout.  With p groups per side and p_v = V >> 25 file
// blocks per side (bit_shift0, gstore.h:82), file block (a, b) -- a <= b for
// the half grid -- holds the groups of rows [a np, (a+1) np) and columns
// [b np, (b+1) np), np = p / p_v, and is file F = calc_index(a, b, p_v)
// (gstore.h:107-113 half, 146-150 full):
//   * <prefix>.grid.F: for each group row c of the block, the groups (c, d)
//     of the block in column order (the diagonal block from d = c), each
//     group's records in the tile order of the single .grid;
//   * <prefix>.start.F: one u64 per tile of those group rows, in the same
//     order, no closing entry.  The writer accumulates a running sum of the
//     per-row prefix sums: within a row of tc tiles, entry d minus entry d-1
//     is cum(d) = the records of the row's first d tiles, and the next row's
//     first entry closes the row (entry tc, cum(tc)); the file's last row is
//     closed by the .grid.F size.  Counts follow as cum(d+1) - cum(d); the
//     u64 arithmetic is exact modulo 2^64, which the differences tolerate.
// A row's records are contiguous in its file and in the single .grid order,
// so the records of the graph map to one (file, offset) piece per row.
#include "gs_internal.cuh"

#include <algorithm>
#include <cstdio>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

namespace {

bool file_bytes(const std::string& path, uint64_t* bytes) {
    struct stat st;
    if (stat(path.c_str(), &st) != 0) return false;
    *bytes = (uint64_t)st.st_size;
    return true;
}

template <class T>
bool read_file(const std::string& path, std::vector<T>* out, uint64_t count) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    out->resize(count);
    const uint64_t got = count ? std::fread(out->data(), sizeof(T), count, f) : 0;
    std::fclose(f);
    return got == count;
}

gs_status single_layout(gs_ctx* ctx, const std::string& prefix, uint64_t T_all, gs_tile_layout* L) {
    uint64_t sb = 0, gb = 0;
    if (!file_bytes(prefix + ".start", &sb)) return gs_fail(ctx, GS_ERR_ARG, "cannot stat " + prefix + ".start");
    if (sb % 8 || sb / 8 != T_all + 1)
        return gs_fail(ctx, GS_ERR_FORMAT,
                       prefix + ".start has " + std::to_string(sb / 8) + " entries; the tile geometry needs " +
                           std::to_string(T_all + 1) + " (check the vertex count)");
    if (!file_bytes(prefix + ".grid", &gb)) return gs_fail(ctx, GS_ERR_ARG, "cannot stat " + prefix + ".grid");
    if (gb % 4) return gs_fail(ctx, GS_ERR_FORMAT, prefix + ".grid size is not a multiple of 4");
    if (!read_file(prefix + ".start", &L->start, sb / 8)) return gs_fail(ctx, GS_ERR_ARG, "cannot read .start");
    if (L->start.back() != gb / 4)
        return gs_fail(ctx, GS_ERR_FORMAT, "last .start entry " + std::to_string(L->start.back()) +
                                                " != records in .grid " + std::to_string(gb / 4));
    L->files = {prefix + ".grid"};
    L->pieces.clear();
    if (gb) L->pieces.push_back(gs_grid_piece{0, gb / 4, 0, 0, 0});
    return GS_OK;
}

gs_status multi_layout(gs_ctx* ctx, const std::string& prefix, uint64_t V, int directed, uint32_t p,
                       uint64_t T_all, gs_tile_layout* L) {
    const uint64_t p_v = V >> 25;
    if (p_v == 0 || p % p_v != 0)
        return gs_fail(ctx, GS_ERR_FORMAT, "the multi-file layout needs V >= 2^25 and p divisible by V >> 25");
    const uint64_t np = p / p_v;
    std::vector<uint64_t> count(T_all, 0);
    struct Row {
        uint64_t tile0, n_rec, file_rec;
        uint32_t file;
    };
    std::vector<Row> rows;
    L->files.clear();
    for (uint64_t a = 0; a < p_v; ++a) {
        for (uint64_t b = directed ? 0 : a; b < p_v; ++b) {
            const uint64_t f = directed ? a * p_v + b : gs_calc_index_half(a, b, p_v);
            const std::string sp = prefix + ".start." + std::to_string(f), gp = prefix + ".grid." + std::to_string(f);
            uint64_t sb = 0, gb = 0;
            if (!file_bytes(sp, &sb) || !file_bytes(gp, &gb))
                return gs_fail(ctx, GS_ERR_ARG, "multi-file layout: cannot stat " + sp + " or " + gp);
            if (sb % 8 || gb % 4) return gs_fail(ctx, GS_ERR_FORMAT, sp + " or " + gp + " has a partial entry");
            std::vector<uint64_t> ent;
            if (!read_file(sp, &ent, sb / 8)) return gs_fail(ctx, GS_ERR_ARG, "cannot read " + sp);
            const uint64_t R = gb / 4;
            if (L->files.size() <= f) L->files.resize(f + 1);
            L->files[f] = gp;
            uint64_t idx = 0, used = 0;
            for (uint64_t c = a * np; c < (a + 1) * np; ++c) {
                const uint64_t base = (!directed && a == b) ? gs_group_base(c, c, p, directed)
                                                            : gs_group_base(c, b * np, p, directed);
                const uint64_t tc = gs_group_base(c, b * np + np, p, directed) - base;
                if (idx + tc > ent.size()) return gs_fail(ctx, GS_ERR_FORMAT, sp + " has too few entries");
                const bool last = c + 1 == (a + 1) * np;
                if (last != (idx + tc == ent.size()))
                    return gs_fail(ctx, GS_ERR_FORMAT, sp + " does not match the tile geometry");
                uint64_t prev_cum = 0;
                for (uint64_t d = 0; d < tc; ++d) {
                    // cum(d + 1): entry d+1 - entry d, or for the row's last tile the
                    // next row's first entry (the file size for the last row)
                    uint64_t cum;
                    if (d + 1 < tc) cum = ent[idx + d + 1] - ent[idx + d];
                    else if (!last) cum = ent[idx + tc] - ent[idx + tc - 1];
                    else cum = R - used;
                    if (cum < prev_cum)
                        return gs_fail(ctx, GS_ERR_FORMAT, sp + ": tile counts do not decode (entry " +
                                                               std::to_string(idx + d) + ")");
                    count[base + d] = cum - prev_cum;
                    prev_cum = cum;
                }
                rows.push_back(Row{base, prev_cum, used, (uint32_t)f});
                used += prev_cum;
                idx += tc;
            }
            if (used != R)
                return gs_fail(ctx, GS_ERR_FORMAT, gp + " holds " + std::to_string(R) + " records; " + sp +
                                                       " counts " + std::to_string(used));
        }
    }
    L->start.assign(T_all + 1, 0);
    for (uint64_t t = 0; t < T_all; ++t) L->start[t + 1] = L->start[t] + count[t];
    L->pieces.clear();
    for (const Row& r : rows)
        if (r.n_rec) L->pieces.push_back(gs_grid_piece{L->start[r.tile0], r.n_rec, r.file_rec, r.file, 0});
    std::sort(L->pieces.begin(), L->pieces.end(),
              [](const gs_grid_piece& x, const gs_grid_piece& y) { return x.rec_beg < y.rec_beg; });
    return GS_OK;
}

}  // namespace

gs_status gs_read_layout(gs_ctx* ctx, const std::string& prefix, uint64_t V, int directed, gs_tile_layout* L) {
    if (V == 0 || V > (1ull << 32)) return gs_fail(ctx, GS_ERR_ARG, "bad vertex count");
    uint32_t p = 0, ps = 0;
    uint64_t T_all = 0;
    gs_geometry_of(V, directed, &p, &ps, &T_all);
    uint64_t b = 0;
    if (file_bytes(prefix + ".grid", &b) || !file_bytes(prefix + ".grid.0", &b))
        return single_layout(ctx, prefix, T_all, L);
    return multi_layout(ctx, prefix, V, directed, p, T_all, L);
}

gs_status gs_read_degree(gs_ctx* ctx, const std::string& prefix, uint64_t V, int32_t* degree) {
    uint64_t db = 0;
    if (!file_bytes(prefix + ".degree", &db)) return gs_fail(ctx, GS_ERR_ARG, "cannot stat " + prefix + ".degree");
    // read_degree_in_mem reads vert_count entries (gstore.cpp:2999-3010); a
    // shorter file leaves the tail at zero as calloc does there
    const uint64_t n = std::min<uint64_t>(db / 4, V);
    FILE* f = std::fopen((prefix + ".degree").c_str(), "rb");
    if (!f) return gs_fail(ctx, GS_ERR_ARG, "cannot open " + prefix + ".degree");
    const uint64_t got = n ? std::fread(degree, 4, n, f) : 0;
    std::fclose(f);
    if (got != n) return gs_fail(ctx, GS_ERR_ARG, "short read on " + prefix + ".degree");
    std::fill(degree + n, degree + V, 0);
    return GS_OK;
}

extern "C" gs_status gs_read_tile_files(gs_ctx* ctx, const char* prefix, uint64_t V, int directed,
                                        uint64_t* start, uint64_t n_start, uint32_t* grid, uint64_t grid_capacity,
                                        int32_t* degree, uint64_t* n_edges) {
    if (!prefix || !n_edges) return gs_fail(ctx, GS_ERR_ARG, "null argument");
    gs_tile_layout L;
    GS_TRY(gs_read_layout(ctx, prefix, V, directed, &L));
    *n_edges = L.start.back();
    if (start) {
        if (n_start != L.start.size())
            return gs_fail(ctx, GS_ERR_ARG, "start holds " + std::to_string(n_start) + " entries; the geometry needs " +
                                                std::to_string(L.start.size()));
        std::copy(L.start.begin(), L.start.end(), start);
    }
    if (grid) {
        if (grid_capacity < L.start.back()) return gs_fail(ctx, GS_ERR_ARG, "grid buffer too small");
        std::vector<int> fds;
        for (const std::string& path : L.files) fds.push_back(path.empty() ? -1 : open(path.c_str(), O_RDONLY));
        bool ok = true;
        for (int fd : fds) ok = ok && fd >= 0;
        if (ok && L.start.back()) ok = gs_read_pieces(fds, L.pieces, grid, 0, L.start.back());
        for (int fd : fds)
            if (fd >= 0) close(fd);
        if (!ok) return gs_fail(ctx, GS_ERR_FORMAT, std::string("reading the records of ") + prefix + " failed");
    }
    if (degree) GS_TRY(gs_read_degree(ctx, prefix, V, degree));
    return GS_OK;
}
