/*
 * gs_oracle.c — sequential CPU restatement of the G-Store tile-grid hot path.
 * TEST INFRASTRUCTURE ONLY (see gs_oracle.h): the product never links it.
 * Each function cites the reference file:line it restates.
 */
#include "gs_oracle.h"
#include <stdlib.h>
#include <string.h>

#define TILE_BITS 16                 /* bit_shift2, gstore.h:77          */
#define GROUP_TILES 256              /* p_p, gstore.h:89                 */

/* calc_index for the half grid (gstore.h:109-113). */
static inline uint64_t calc_index_half(uint64_t i, uint64_t j, uint64_t pc)
{
    return ((i * ((pc << 1) - i - 1)) >> 1) + j;
}

/* beg_edge_offset1/2 (gstore.h:128-141 half, 167-178 full): first .start
 * index of group (i,i) resp. (i,j). */
static uint64_t group_base(uint64_t gi, uint64_t gj, uint64_t p, int directed)
{
    if (directed) return (gi * p + gj) << 16;
    if (gi == gj) return ((calc_index_half(gi, gi, p) - gi) << 16) + ((gi * 257) << 7);
    return ((calc_index_half(gi, gj, p) - gi - 1) << 16) + (((gi + 1) * 257) << 7);
}

void orc_geometry(uint64_t V, int directed, uint32_t* p, uint32_t* p_s,
                  uint64_t* n_tiles)
{
    uint64_t pp = (V >> 24) + ((V & 0xFFFFFF) != 0);
    if (pp == 0) pp = 1;
    uint64_t ps = pp * GROUP_TILES;
    if (p) *p = (uint32_t)pp;
    if (p_s) *p_s = (uint32_t)ps;
    if (n_tiles) *n_tiles = directed ? ps * ps : ps * (ps + 1) / 2;
}

uint64_t orc_tile_index(uint32_t p, int directed, uint32_t row, uint32_t col)
{
    uint64_t ps = (uint64_t)p * GROUP_TILES;
    if (row >= ps || col >= ps) return UINT64_MAX;
    if (!directed && row > col) return UINT64_MAX;
    uint64_t gi = row >> 8, gj = col >> 8, m = row & 255, n = col & 255;
    uint64_t base = group_base(gi, gj, p, directed);
    if (!directed && gi == gj) return base + calc_index_half(m, n, GROUP_TILES);
    return base + m * GROUP_TILES + n;
}

int orc_tile_coords(uint32_t p, int directed, uint32_t* row, uint32_t* col)
{
    uint64_t t = 0;
    for (uint64_t gi = 0; gi < p; ++gi) {
        for (uint64_t gj = directed ? 0 : gi; gj < p; ++gj) {
            for (uint64_t m = 0; m < GROUP_TILES; ++m) {
                uint64_t n0 = (!directed && gi == gj) ? m : 0;
                for (uint64_t n = n0; n < GROUP_TILES; ++n) {
                    row[t] = (uint32_t)(gi * GROUP_TILES + m);
                    col[t] = (uint32_t)(gj * GROUP_TILES + n);
                    ++t;
                }
            }
        }
    }
    return 0;
}

typedef struct {
    uint64_t T;
    uint32_t* row;
    uint32_t* col;
} tiles_t;

static int tiles_make(uint32_t p, int directed, tiles_t* tl)
{
    uint32_t ps;
    orc_geometry((uint64_t)p << 24, directed, 0, &ps, &tl->T);
    tl->row = (uint32_t*)malloc(tl->T * sizeof(uint32_t));
    tl->col = (uint32_t*)malloc(tl->T * sizeof(uint32_t));
    if (!tl->row || !tl->col) return -1;
    return orc_tile_coords(p, directed, tl->row, tl->col);
}

static void tiles_free(tiles_t* tl)
{
    free(tl->row);
    free(tl->col);
}

/* Every record must address a vertex below n. */
static int check_range(const uint64_t* start, const uint32_t* grid,
                       const tiles_t* tl, uint64_t n)
{
    for (uint64_t t = 0; t < tl->T; ++t) {
        if (start[t + 1] < start[t]) return -1;
        if (start[t + 1] == start[t]) continue;
        uint64_t b0 = (uint64_t)tl->row[t] << TILE_BITS;
        uint64_t b1 = (uint64_t)tl->col[t] << TILE_BITS;
        for (uint64_t e = start[t]; e < start[t + 1]; ++e) {
            if (b0 + (grid[e] & 0xFFFF) >= n || b1 + (grid[e] >> 16) >= n) return -1;
        }
    }
    return 0;
}

/* ---------------------------------------------------------------- BFS --- */
int orc_bfs(const uint64_t* start, const uint32_t* grid, uint32_t p,
            int directed, uint64_t n, uint64_t root, uint8_t* depth,
            uint64_t* level_counts, uint64_t* swept, int max_levels,
            int* n_levels)
{
    tiles_t tl;
    if (root >= n || tiles_make(p, directed, &tl)) return -1;
    if (check_range(start, grid, &tl, n)) { tiles_free(&tl); return -1; }
    uint64_t ps = (uint64_t)p * GROUP_TILES;
    uint8_t* act = (uint8_t*)calloc(ps, 1);
    uint8_t* nxt = (uint8_t*)calloc(ps, 1);
    memset(depth, 0, n);                       /* INFTY = 0, bfs.cpp:54 */
    depth[root] = 1;                           /* bfs.cpp:70-71 */
    uint8_t level = 1;
    act[root >> TILE_BITS] = 1;                /* calc_part_needed, bfs.cpp:324-338 */
    int status = 0, lv = 0;
    for (;;) {
        uint64_t front = 0, sw = 0;
        memset(nxt, 0, ps);
        for (uint64_t t = 0; t < tl.T; ++t) {
            uint64_t r = tl.row[t], c = tl.col[t];
            int ri = act[r], rj = act[c];
            /* tile dispatch of grid::bfs_mmap (gstore.cpp:2671-2698) */
            int fwd, bwd;
            if (directed) { fwd = ri; bwd = 0; }
            else { fwd = ri; bwd = rj; }
            if (!fwd && !bwd) continue;
            sw += start[t + 1] - start[t];
            uint8_t* d0 = depth + (r << TILE_BITS);
            uint8_t* d1 = depth + (c << TILE_BITS);
            int ni = 0, nj = 0;
            for (uint64_t e = start[t]; e < start[t + 1]; ++e) {
                uint32_t v0 = grid[e] & 0xFFFF, v1 = grid[e] >> 16;
                /* bfs_onepart / _row / _col, bfs.cpp:138-185, 77-136 */
                if (fwd && d0[v0] == level && d1[v1] == 0) {
                    d1[v1] = (uint8_t)(level + 1); ++front; nj = 1;
                } else if (bwd && d1[v1] == level && d0[v0] == 0) {
                    d0[v0] = (uint8_t)(level + 1); ++front; ni = 1;
                }
            }
            if (ni) nxt[r] = 1;
            if (nj) nxt[c] = 1;
        }
        if (lv < max_levels) {
            if (level_counts) level_counts[lv] = front;
            if (swept) swept[lv] = sw;
        }
        ++lv;
        if (front == 0) break;                 /* iteration_finalize, bfs.cpp:187-224 */
        if (level == 254) { status = -2; break; }
        ++level;
        uint8_t* tmp = act; act = nxt; nxt = tmp;
    }
    if (n_levels) *n_levels = lv;
    free(act); free(nxt); tiles_free(&tl);
    return status;
}

uint64_t orc_edges_reached(const uint64_t* start, const uint32_t* grid, uint32_t p,
                           int directed, const uint8_t* depth)
{
    tiles_t tl;
    if (tiles_make(p, directed, &tl)) return 0;
    uint64_t total = 0;
    for (uint64_t t = 0; t < tl.T; ++t) {
        const uint8_t* d0 = depth + ((uint64_t)tl.row[t] << TILE_BITS);
        const uint8_t* d1 = depth + ((uint64_t)tl.col[t] << TILE_BITS);
        for (uint64_t e = start[t]; e < start[t + 1]; ++e)
            total += (d0[grid[e] & 0xFFFF] != 0) & (d1[grid[e] >> 16] != 0);
    }
    tiles_free(&tl);
    return total;
}

/* --------------------------------------------------------------- bfs2 --- */
int orc_bfs2(const uint64_t* start, const uint32_t* grid, uint32_t p, int directed,
             uint64_t n, uint64_t root, uint8_t* depth, int* n_sweeps)
{
    tiles_t tl;
    if (root >= n || tiles_make(p, directed, &tl)) return -1;
    if (check_range(start, grid, &tl, n)) { tiles_free(&tl); return -1; }
    memset(depth, 0, n);                       /* INFTY = 0 (bfs.cpp:54) */
    depth[root] = 1;                           /* bfs2.cpp:73 */
    int status = 0, sweeps = 0;
    for (;;) {
        uint64_t changed = 0;
        for (uint64_t t = 0; t < tl.T && status == 0; ++t) {
            uint8_t* d0 = depth + ((uint64_t)tl.row[t] << TILE_BITS);
            uint8_t* d1 = depth + ((uint64_t)tl.col[t] << TILE_BITS);
            for (uint64_t e = start[t]; e < start[t + 1]; ++e) {
                uint32_t v0 = grid[e] & 0xFFFF, v1 = grid[e] >> 16;
                int l0 = d0[v0], l1 = d1[v1];
                /* relax either end (bfs2_t::bfs_onepart, bfs2.cpp:102-117) */
                if (l0 != 0 && (l1 == 0 || l1 - l0 > 1)) {
                    if (l0 == 255) { status = -2; break; }
                    d1[v1] = (uint8_t)(l0 + 1); ++changed;
                } else if (!directed && l1 != 0 && (l0 == 0 || l0 - l1 > 1)) {
                    if (l1 == 255) { status = -2; break; }
                    d0[v0] = (uint8_t)(l1 + 1); ++changed;
                }
            }
        }
        ++sweeps;
        if (status || changed == 0) break;     /* bfs2_t::iteration_finalize */
    }
    if (n_sweeps) *n_sweeps = sweeps;
    tiles_free(&tl);
    return status;
}

/* ----------------------------------------------------------- traverse --- */
int orc_traverse(const uint64_t* start, const uint32_t* grid, uint32_t p, int directed,
                 uint64_t n, uint64_t pivot, uint32_t* cid, uint64_t* colored, int* n_sweeps)
{
    tiles_t tl;
    if (pivot >= n || tiles_make(p, directed, &tl)) return -1;
    if (check_range(start, grid, &tl, n)) { tiles_free(&tl); return -1; }
    for (uint64_t v = 0; v < n; ++v) cid[v] = 0xFFFFFFFFu;   /* invalid_cid, traverse.cpp:66-70 */
    cid[pivot] = 0;                                          /* colour 0 */
    uint64_t total = 1;
    int sweeps = 0;
    for (;;) {
        uint64_t changed = 0;
        for (uint64_t t = 0; t < tl.T; ++t) {
            uint32_t* c0 = cid + ((uint64_t)tl.row[t] << TILE_BITS);
            uint32_t* c1 = cid + ((uint64_t)tl.col[t] << TILE_BITS);
            for (uint64_t e = start[t]; e < start[t + 1]; ++e) {
                uint32_t v0 = grid[e] & 0xFFFF, v1 = grid[e] >> 16;
                /* traverse_onepart (traverse.cpp:173-188): v0 -> v1 only */
                if (c0[v0] == 0 && c1[v1] == 0xFFFFFFFFu) { c1[v1] = 0; ++changed; }
            }
        }
        ++sweeps;
        total += changed;
        if (changed == 0) break;               /* traverse_t::iteration_finalize */
    }
    if (colored) *colored = total;
    if (n_sweeps) *n_sweeps = sweeps;
    tiles_free(&tl);
    return 0;
}

/* ----------------------------------------------------------- PageRank --- */
/* Tiles grouped by one of their windows (counting sort of tile indices by
 * row or by column), so that one thread can own a window's sums. */
static void tiles_by_window(const tiles_t* tl, uint64_t nw, int by_col, uint64_t* off, uint64_t* idx)
{
    memset(off, 0, (nw + 1) * sizeof(uint64_t));
    for (uint64_t t = 0; t < tl->T; ++t) ++off[(by_col ? tl->col[t] : tl->row[t]) + 1];
    for (uint64_t w = 0; w < nw; ++w) off[w + 1] += off[w];
    uint64_t* pos = (uint64_t*)malloc(nw * sizeof(uint64_t));
    memcpy(pos, off, nw * sizeof(uint64_t));
    for (uint64_t t = 0; t < tl->T; ++t) idx[pos[by_col ? tl->col[t] : tl->row[t]]++] = t;
    free(pos);
}

int orc_pagerank(const uint64_t* start, const uint32_t* grid,
                 const int32_t* degree, uint32_t p, int directed, uint64_t n,
                 int iterations, int compat, double* r_out, double* x_out)
{
    tiles_t tl;
    if (n == 0 || iterations < 1 || tiles_make(p, directed, &tl)) return -1;
    if (check_range(start, grid, &tl, n)) { tiles_free(&tl); return -1; }
    const uint64_t nw = (uint64_t)p * GROUP_TILES;
    double* x = (double*)malloc(n * sizeof(double));
    double* s = (double*)malloc(n * sizeof(double));
    double* inv = (double*)malloc(n * sizeof(double));
    uint64_t* col_off = (uint64_t*)malloc((nw + 1) * sizeof(uint64_t));
    uint64_t* row_off = (uint64_t*)malloc((nw + 1) * sizeof(uint64_t));
    uint64_t* col_idx = (uint64_t*)malloc((tl.T + 1) * sizeof(uint64_t));
    uint64_t* row_idx = (uint64_t*)malloc((tl.T + 1) * sizeof(uint64_t));
    tiles_by_window(&tl, nw, 1, col_off, col_idx);
    tiles_by_window(&tl, nw, 0, row_off, row_idx);
    for (uint64_t v = 0; v < n; ++v) {
        x[v] = 1.0 / (double)n;                /* pr.cpp:105-110 */
        int32_t d = degree[v];
        if (d == 0) inv[v] = 0.0;
        else if (compat) inv[v] = (double)(int32_t)(1.0 / d);   /* pr.cpp:112-114 */
        else inv[v] = 1.0 / (double)d;
    }
    for (int it = 0; it < iterations; ++it) {
        memset(s, 0, n * sizeof(double));
        /* s[v1] += x[v0] (pr.cpp:145-146): a thread owns the sums of one
         * column window; deterministic order (tiles in file order) */
        #pragma omp parallel for schedule(dynamic, 1)
        for (uint64_t w = 0; w < nw; ++w) {
            for (uint64_t k = col_off[w]; k < col_off[w + 1]; ++k) {
                const uint64_t t = col_idx[k];
                const uint64_t b0 = (uint64_t)tl.row[t] << TILE_BITS, b1 = w << TILE_BITS;
                for (uint64_t e = start[t]; e < start[t + 1]; ++e)
                    s[b1 + (grid[e] >> 16)] += x[b0 + (grid[e] & 0xFFFF)];
            }
        }
        /* s[v0] += x[v1] (pr.cpp:147-150, half grid): one row window each */
        if (!directed) {
            #pragma omp parallel for schedule(dynamic, 1)
            for (uint64_t w = 0; w < nw; ++w) {
                for (uint64_t k = row_off[w]; k < row_off[w + 1]; ++k) {
                    const uint64_t t = row_idx[k];
                    const uint64_t b0 = w << TILE_BITS, b1 = (uint64_t)tl.col[t] << TILE_BITS;
                    for (uint64_t e = start[t]; e < start[t + 1]; ++e)
                        s[b0 + (grid[e] & 0xFFFF)] += x[b1 + (grid[e] >> 16)];
                }
            }
        }
        #pragma omp parallel for
        for (uint64_t v = 0; v < n; ++v) {     /* pr.cpp:281-302 */
            double r = 0.15 + 0.85 * s[v];
            if (r_out) r_out[v] = r;
            x[v] = r * inv[v];
        }
    }
    if (x_out) memcpy(x_out, x, n * sizeof(double));
    free(x); free(s); free(inv); free(col_off); free(row_off); free(col_idx); free(row_idx);
    tiles_free(&tl);
    return 0;
}

/* ---------------------------------------------------------------- WCC --- */
static uint64_t uf_find(uint64_t* par, uint64_t v)
{
    while (par[v] != v) {
        par[v] = par[par[v]];
        v = par[v];
    }
    return v;
}

int orc_wcc(const uint64_t* start, const uint32_t* grid, uint32_t p,
            int directed, uint64_t n, uint32_t* label, uint64_t* count)
{
    tiles_t tl;
    if (tiles_make(p, directed, &tl)) return -1;
    if (check_range(start, grid, &tl, n)) { tiles_free(&tl); return -1; }
    uint64_t* par = (uint64_t*)malloc(n * sizeof(uint64_t));
    uint8_t* touched = (uint8_t*)calloc(n, 1);
    for (uint64_t v = 0; v < n; ++v) par[v] = v;
    for (uint64_t t = 0; t < tl.T; ++t) {
        uint64_t b0 = (uint64_t)tl.row[t] << TILE_BITS;
        uint64_t b1 = (uint64_t)tl.col[t] << TILE_BITS;
        for (uint64_t e = start[t]; e < start[t + 1]; ++e) {
            uint64_t a = b0 + (grid[e] & 0xFFFF), b = b1 + (grid[e] >> 16);
            touched[a] = touched[b] = 1;       /* wcc.cpp:203-217 label creation */
            uint64_t ra = uf_find(par, a), rb = uf_find(par, b);
            if (ra < rb) par[rb] = ra; else if (rb < ra) par[ra] = rb;
        }
    }
    uint64_t comps = 0;
    for (uint64_t v = 0; v < n; ++v) {
        if (!touched[v]) { label[v] = 0xFFFFFFFFu; continue; }   /* wcc.cpp:54, 66-68 */
        uint64_t r = uf_find(par, v);
        label[v] = (uint32_t)r;                /* root = smallest id (min-hooking) */
        if (r == v) ++comps;
    }
    if (count) *count = comps;
    free(par); free(touched); tiles_free(&tl);
    return 0;
}

/* ------------------------------------------------------------- k-core --- */
int orc_kcore(const uint64_t* start, const uint32_t* grid, uint32_t p,
              uint64_t n, int k, int32_t* deg, uint64_t* members,
              uint64_t* swept, int max_rounds, int* n_rounds)
{
    tiles_t tl;
    if (tiles_make(p, 0, &tl)) return -1;
    if (check_range(start, grid, &tl, n)) { tiles_free(&tl); return -1; }
    uint64_t ps = (uint64_t)p * GROUP_TILES;
    uint8_t* active = (uint8_t*)calloc(n, 1);
    uint8_t* act = (uint8_t*)calloc(ps, 1);
    int rounds = 0;
    for (;;) {
        /* kcore_t::iteration_finalize, kcore.cpp:179-217 */
        uint64_t removed = 0;
        memset(act, 0, ps);
        for (uint64_t v = 0; v < n; ++v) {
            int16_t m = (int16_t)deg[v];       /* sdegree_t truncation, kcore.cpp:189 */
            active[v] = 0;
            if (m < k && m > 0) {
                deg[v] = 0;                    /* GONE */
                active[v] = 1;
                act[v >> TILE_BITS] = 1;
                ++removed;
            }
        }
        if (removed == 0) break;
        /* sweep, grid::kcore_mmap dispatch gstore.cpp:2769-2783 */
        uint64_t sw = 0;
        for (uint64_t t = 0; t < tl.T; ++t) {
            uint64_t r = tl.row[t], c = tl.col[t];
            int ri = act[r], rj = act[c];
            if (!ri && !rj) continue;
            sw += start[t + 1] - start[t];
            uint64_t b0 = r << TILE_BITS, b1 = c << TILE_BITS;
            for (uint64_t e = start[t]; e < start[t + 1]; ++e) {
                uint64_t a = b0 + (grid[e] & 0xFFFF), b = b1 + (grid[e] >> 16);
                if (ri && active[a]) deg[b] -= 1;   /* kcore.cpp:77-78 */
                if (rj && active[b]) deg[a] -= 1;   /* kcore.cpp:90-91 */
            }
        }
        if (swept && rounds < max_rounds) swept[rounds] = sw;
        ++rounds;
    }
    uint64_t mem = 0;
    for (uint64_t v = 0; v < n; ++v) mem += (deg[v] != 0);   /* gstore.cpp:2796-2800 */
    if (members) *members = mem;
    if (n_rounds) *n_rounds = rounds;
    free(active); free(act); tiles_free(&tl);
    return 0;
}

/* ---------------------------------------------------------- converter --- */
int orc_convert(const uint32_t* edges, uint64_t n_pairs, uint32_t p,
                int directed, uint64_t n, uint64_t* start, uint32_t* grid,
                int32_t* degree, uint64_t* n_records)
{
    uint64_t T;
    uint32_t ps;
    orc_geometry((uint64_t)p << 24, directed, 0, &ps, &T);
    memset(start, 0, (T + 1) * sizeof(uint64_t));
    memset(degree, 0, n * sizeof(int32_t));
    for (uint64_t k = 0; k < n_pairs; ++k) {   /* pre_grid, gstore.cpp:1270-1312 */
        uint64_t u = edges[2 * k], v = edges[2 * k + 1];
        if (u == v) continue;
        if (u >= n || v >= n) return -1;
        uint64_t a = u, b = v;
        if (!directed && a > b) { a = v; b = u; }
        uint64_t t = orc_tile_index(p, directed, (uint32_t)(a >> TILE_BITS),
                                    (uint32_t)(b >> TILE_BITS));
        if (t == UINT64_MAX) return -1;
        start[t] += 1;
        degree[u] += 1;
        if (!directed) degree[v] += 1;
    }
    uint64_t sum = 0;                          /* gstore.cpp:1316-1324 */
    for (uint64_t t = 0; t < T; ++t) {
        uint64_t c = start[t];
        start[t] = sum;
        sum += c;
    }
    start[T] = sum;
    if (n_records) *n_records = sum;
    if (!grid) return 0;
    uint64_t* cur = (uint64_t*)calloc(T, sizeof(uint64_t));
    for (uint64_t k = 0; k < n_pairs; ++k) {   /* proc_grid scatter, :1403-1447 */
        uint64_t u = edges[2 * k], v = edges[2 * k + 1];
        if (u == v) continue;
        uint64_t a = u, b = v;
        if (!directed && a > b) { a = v; b = u; }
        uint64_t t = orc_tile_index(p, directed, (uint32_t)(a >> TILE_BITS),
                                    (uint32_t)(b >> TILE_BITS));
        grid[start[t] + cur[t]++] = (uint32_t)(a & 0xFFFF) | ((uint32_t)(b & 0xFFFF) << 16);
    }
    free(cur);
    return 0;
}
