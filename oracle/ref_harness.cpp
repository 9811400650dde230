/*
 * Oracle harness around the G-Store reference, compiled from the reference's
 * own sources (gstore.cpp with main renamed, bfs.cpp, pr.cpp, wcc.cpp,
 * kcore.cpp, ...).  TEST INFRASTRUCTURE ONLY: the product never links it.
 *
 * The reference prints no per-vertex results, so this harness drives the
 * reference's algorithm classes (bfs_t, kcore_t, wcc2_t, pr_t) through the
 * same in-memory tile loop as its "-j 2x" drivers and dumps their arrays:
 *
 *   bfs   : depth_t (u8) per vertex          (bfs_t,   bfs.cpp:56-338)
 *   kcore : final vert_degree (i32)          (kcore_t, kcore.cpp:55-300)
 *   wcc   : vert_cid (u32) per vertex        (wcc2_t,  wcc.cpp:57-395)
 *   pr    : vert_rank_prior (f32) after the  (pr_t,    pr.cpp:82-303;
 *           last iteration_finalize             its int32 inverse-degree
 *                                               truncation included)
 *   bfs2  : depth_t (u8) per vertex          (bfs2_t,  bfs2.cpp:56-181)
 *   traverse : vert_cid (u32) per vertex     (traverse_t, traverse.cpp:56-212)
 *
 * The tile loop follows grid::bfs_mmap / kcore_mmap / wcc_mmap /
 * pagerank_mmap (gstore.cpp:2502-2804): every stored tile of the half
 * (HALF_GRID) or full grid, in file order, with the same row/column
 * activity dispatch.  It runs on one thread so the run is deterministic.
 *
 * usage: ref_harness <prefix> <vert_count> <bfs|kcore|wcc|pr> <arg> <out.bin>
 *   arg = root (bfs), k (kcore), iterations (pr), unused (wcc)
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <iostream>
#include <omp.h>

#include "gstore.h"
#include "bfs.h"
#include "pr.h"
#include "wcc.h"
#include "kcore.h"
#include "bfs2.h"
#include "traverse.h"

extern grid* g;
extern cache_driver* cache;
extern io_driver* io;

template <class F>
static void for_each_tile(F f)
{
    for (index_t gi = 0; gi < p; ++gi) {
#ifdef HALF_GRID
        for (index_t gj = gi; gj < p; ++gj)
#else
        for (index_t gj = 0; gj < p; ++gj)
#endif
        {
            for (index_t m = 0; m < p_p; ++m) {
                index_t n0 = 0;
#ifdef HALF_GRID
                if (gi == gj) n0 = m;
#endif
                for (index_t n = n0; n < p_p; ++n) {
                    index_t idx;
#ifdef HALF_GRID
                    if (gi == gj)
                        idx = beg_edge_offset1(gi) + calc_index(m, n, p_p);
                    else
                        idx = beg_edge_offset2(gi, gj) + m * p_p + n;
#else
                    idx = beg_edge_offset2(gi, gj) + m * p_p + n;
#endif
                    edge_t* e = g->_edges + g->_s_start_edge[idx];
                    index_t cnt = g->_s_start_edge[idx + 1] - g->_s_start_edge[idx];
                    f(e, cnt, (part_t)(gi * p_p + m), (part_t)(gj * p_p + n));
                }
            }
        }
    }
}

static void write_out(const char* path, const void* data, size_t bytes)
{
    FILE* f = fopen(path, "wb");
    if (!f) { perror("open out"); exit(2); }
    if (bytes && fwrite(data, 1, bytes, f) != bytes) { perror("write out"); exit(2); }
    fclose(f);
}

int main(int argc, char* argv[])
{
    if (argc != 6) {
        fprintf(stderr, "usage: %s prefix vert_count bfs|kcore|wcc|pr|bfs2|traverse arg out\n", argv[0]);
        return 2;
    }
    std::string prefix = argv[1];
    vertex_t V = strtoull(argv[2], 0, 10);
    std::string algo = argv[3];
    long arg = strtol(argv[4], 0, 10);
    const char* out = argv[5];

    g = new grid;
    cache = new cache_driver;
    io = new io_driver;

    /* -v semantics of grid::init (gstore.cpp:152-161) */
    p = (V >> bit_shift1) + (0 != (V & part_mask1_2));
    if (p == 0) p = 1;
    p_s = p_p * p;
    g->read_part = new bitmap_t(p_s);
    g->read_part_next = new bitmap_t(p_s);
    g->read_part_next->reset();

    /* BFS and k-core index depth/bitmaps up to p_s << 16 (bfs.cpp:431-440),
     * so their arrays are sized to the whole tile range. */
    vertex_t alloc = V;
    if (algo == "bfs" || algo == "kcore" || algo == "bfs2") {
        vertex_t full = (vertex_t)p_s << bit_shift2;
        if (full > alloc) alloc = full;
    }
    g->vert_count = alloc;

    g->read_grid_in_mem(prefix);

    if (algo == "bfs") {
        bfs_t bf;
        bf.init(alloc, (vertex_t)arg, g->read_part);
        while (true) {
            index_t fc = 0;
            for_each_tile([&](edge_t* e, index_t c, part_t i, part_t j) {
                bitmap_t* rp = g->read_part;
#ifdef HALF_GRID
                bool ri = rp->get_bit(i), rj = rp->get_bit(j);
                if (ri && rj) fc += bf.bfs_onepart(e, c, i, j);
                else if (rj) fc += bf.bfs_onepart_col(e, c, i, j);
                else if (ri) fc += bf.bfs_onepart_row(e, c, i, j);
#else
                if (rp->get_bit(i)) fc += bf.bfs_onepart(e, c, i, j);
#endif
            });
            bf.front_count[0] += fc;
            if (bf.iteration_finalize()) break;
        }
        write_out(out, bf.depth, V);
    } else if (algo == "kcore") {
#ifndef HALF_GRID
        fprintf(stderr, "kcore not applicable for directed graphs\n");
        return 3;
#else
        g->read_degree_in_mem(prefix);
        kcore_t kc;
        kc.init(alloc, (int)arg, g->vert_degree, g->read_part);
        if (0 != kc.iteration_finalize()) {
            while (true) {
                for_each_tile([&](edge_t* e, index_t c, part_t i, part_t j) {
                    bitmap_t* rp = g->read_part;
                    bool ri = rp->get_bit(i), rj = rp->get_bit(j);
                    if (ri && rj) kc.kcore_onepart(e, c, i, j);
                    else if (ri) kc.kcore_onepart_row(e, c, i, j);
                    else if (rj) kc.kcore_onepart_col(e, c, i, j);
                });
                if (0 == kc.iteration_finalize()) break;
            }
        }
        vertex_t total = 0;
        for (vertex_t v = 0; v < alloc; ++v) total += (g->vert_degree[v] != 0);
        std::cout << ">= " << arg << "vertices count = " << total << std::endl;
        write_out(out, g->vert_degree, V * sizeof(int32_t));
#endif
    } else if (algo == "wcc") {
        wcc2_t w;
        w.init(alloc);
        int iteration = 0;
        while (true) {
            index_t fc = 0;
            for_each_tile([&](edge_t* e, index_t c, part_t i, part_t j) {
                if (iteration == 0) fc += w.wcc_onepart(e, c, i, j);
                else fc += w.wcc_onepart2(e, c, i, j);
            });
            w.front_count[0] += fc;
            if (0 == w.iteration_finalize()) break;
            ++iteration;
        }
        write_out(out, w.vert_cid, V * sizeof(uint32_t));
    } else if (algo == "pr") {
        g->read_degree_in_mem(prefix);
        pr_t pr;
        int iters = arg > 0 ? (int)arg : 5;
        pr.init(alloc, iters);
        for (int it = 0; it < iters; ++it) {
            for_each_tile([&](edge_t* e, index_t c, part_t i, part_t j) {
                pr.pagerank_onepart(e, c, i, j);
            });
            pr.iteration_finalize(it);
        }
        write_out(out, pr.vert_rank_prior, V * sizeof(float));
    } else if (algo == "bfs2") {
        /* label-correcting BFS (bfs2.cpp:56-181): every tile each sweep,
         * until a sweep changes nothing */
        bfs2_t bf;
        bf.init(alloc, (vertex_t)arg, g->read_part);
        while (true) {
            index_t fc = 0;
            for_each_tile([&](edge_t* e, index_t c, part_t i, part_t j) { fc += bf.bfs_onepart(e, c, i, j); });
            bf.front_count[0] += fc;
            if (0 == bf.iteration_finalize()) break;
        }
        write_out(out, bf.depth, V);
    } else if (algo == "traverse") {
        /* single-colour propagation from pivot `arg`, colour 0
         * (traverse.cpp:56-212) */
        traverse_t tr;
        tr.init(alloc, (vertex_t)arg, 0);
        while (true) {
            index_t fc = 0;
            for_each_tile([&](edge_t* e, index_t c, part_t i, part_t j) { fc += tr.traverse_onepart(e, c, i, j); });
            tr.front_count[0] += fc;
            if (0 == tr.iteration_finalize()) break;
        }
        write_out(out, tr.vert_cid, V * sizeof(uint32_t));
    } else {
        fprintf(stderr, "unknown algo %s\n", algo.c_str());
        return 2;
    }
    return 0;
}
