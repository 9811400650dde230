/*
 * gs_oracle — CPU restatement of the G-Store tile-grid hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests, the smoke check and the benchmark's
 * CPU-baseline leg may load this library, and only as the checker.  The
 * product (libgstore_cuda.so and the gstoreu/gstored host) never links it.
 *
 * Every function restates the reference algorithm it cites, in plain
 * sequential C, on the reference's own file formats:
 *   .start : u64 edge offsets, calc_total_part(p_s)+1 entries
 *   .grid  : u32 records  v0 | v1 << 16  (edge_t, gstore.h:311-334)
 *   .degree: i32 per vertex
 * Arrays indexed by vertex are sized `n` = the caller's vertex count; every
 * record must address a vertex below n (checked, GS-style status returned).
 *
 * Status: 0 ok, -1 bad argument / record out of range, -2 BFS depth would
 * overflow the u8 depth_t (more than 254 levels), -3 not applicable.
 */
#ifndef GS_ORACLE_H
#define GS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Tile-grid geometry for vertex count V (grid::init -v, gstore.cpp:152-161). */
void orc_geometry(uint64_t V, int directed, uint32_t* p, uint32_t* p_s,
                  uint64_t* n_tiles);

/* Global (row, col) tile coordinates of every stored tile, in file order
 * (the loops of grid::*_mmap, gstore.cpp:2520-2559). */
int orc_tile_coords(uint32_t p, int directed, uint32_t* row, uint32_t* col);

/* Index of tile (row, col) in .start (calc_index/beg_edge_offset1/2,
 * gstore.h:107-180), or UINT64_MAX if the tile is not stored. */
uint64_t orc_tile_index(uint32_t p, int directed, uint32_t row, uint32_t col);

/* BFS (bfs.cpp:56-338, grid::bfs_mmap gstore.cpp:2631-2713).
 * depth[n] u8: root = 1, unreached = 0.  level_counts[l-1] = vertices
 * discovered while sweeping level l; swept[l-1] = records in the tiles the
 * reference sweeps at level l.  *n_levels = number of sweeps (last has 0). */
int orc_bfs(const uint64_t* start, const uint32_t* grid, uint32_t p,
            int directed, uint64_t n, uint64_t root, uint8_t* depth,
            uint64_t* level_counts, uint64_t* swept, int max_levels,
            int* n_levels);

/* Records whose two ends both have depth != 0: the GTEPS numerator of a
 * BFS (the records of the root's component on an undirected grid).  The
 * reference prints no such count; bfs.cpp:193-194 prints vertices per level. */
uint64_t orc_edges_reached(const uint64_t* start, const uint32_t* grid, uint32_t p,
                           int directed, const uint8_t* depth);

/* Label-correcting BFS, "-j 30" (bfs2.cpp:56-181): every tile each sweep;
 * a record lowers the depth of an end to the other end's depth + 1 (u8,
 * root 1, 0 = unreached), until a sweep changes nothing.  The result is the
 * BFS depth; *n_sweeps counts the sweeps in file order. */
int orc_bfs2(const uint64_t* start, const uint32_t* grid, uint32_t p, int directed,
             uint64_t n, uint64_t root, uint8_t* depth, int* n_sweeps);

/* Single-colour propagation, "-j 4" (traverse.cpp:56-212): cid[pivot] = 0,
 * others 0xFFFFFFFF; a record colours v1 from v0 (one direction, in the
 * half grid too) until a sweep colours nothing.  *colored = vertices with
 * colour 0. */
int orc_traverse(const uint64_t* start, const uint32_t* grid, uint32_t p, int directed,
                 uint64_t n, uint64_t pivot, uint32_t* cid, uint64_t* colored, int* n_sweeps);

/* PageRank in FP64 (pr.cpp:82-303, grid::pagerank_mmap gstore.cpp:2572-2629).
 * x0 = 1/n; per iteration s[v] = sum over records of the other end's x;
 * r = 0.15 + 0.85 s; x = r * inv.  inv = 1/deg (deg > 0) else 0; with
 * compat != 0, inv = (int32)(1.0/deg) as the reference stores it
 * (pr.cpp:112-114).  Outputs r (after the last iteration) and x. */
int orc_pagerank(const uint64_t* start, const uint32_t* grid,
                 const int32_t* degree, uint32_t p, int directed, uint64_t n,
                 int iterations, int compat, double* r_out, double* x_out);

/* WCC partition (wcc.cpp:57-395): label[v] = smallest vertex id of v's
 * component for vertices touched by a record, 0xFFFFFFFF otherwise.
 * *count = number of components ("WCC count", wcc.cpp:324-337). */
int orc_wcc(const uint64_t* start, const uint32_t* grid, uint32_t p,
            int directed, uint64_t n, uint32_t* label, uint64_t* count);

/* k-core with the reference's exact rules (kcore.cpp:55-300,
 * grid::kcore_mmap gstore.cpp:2716-2804): a round removes every vertex with
 * 0 < (int16)deg < k (deg := 0), then every record with a removed endpoint
 * decrements the other endpoint's degree (removed ones go negative).
 * degree_io: in = .degree, out = final degrees.  *members = count(deg != 0).
 * swept[r] = records in the tiles swept in round r (max_rounds entries). */
int orc_kcore(const uint64_t* start, const uint32_t* grid, uint32_t p,
              uint64_t n, int k, int32_t* degree_io, uint64_t* members,
              uint64_t* swept, int max_rounds, int* n_rounds);

/* In-memory converter "-c 1" (grid::pre_grid + proc_grid,
 * gstore.cpp:1245-1458): drops self-loops, orders (min,max) for the half
 * grid, counts tiles and degrees, prefix-sums .start and scatters records.
 * In-tile order here is the input order (the reference's is thread-order). */
int orc_convert(const uint32_t* edges, uint64_t n_pairs, uint32_t p,
                int directed, uint64_t n, uint64_t* start_out,
                uint32_t* grid_out, int32_t* degree_out, uint64_t* n_records);

#ifdef __cplusplus
}
#endif
#endif
