/*
 * gstore_cuda.h — C ABI of libgstore_cuda.so, the B200 (sm_100a) engine for
 * G-Store's tile-grid edge scan.
 *
 * The library replaces the hot path of the G-Store reference: the per-level /
 * per-iteration sweep over the 2D grid of SNB tiles that drives BFS, PageRank,
 * WCC and k-core.  Host code (the gstoreu/gstored CLI, the algo_t adapters, or
 * any FFI caller) drives it through the plain-C entry points below: plain
 * pointers and sizes, no C++ or framework types.
 *
 * Formats (identical to the reference's files):
 *   start  : uint64 edge offsets, one per stored tile plus one
 *            (grid::save_start_files, gstore.cpp:2899-2908)
 *   grid   : uint32 records, v0 | v1 << 16, tile after tile
 *            (edge_t, gstore.h:311-334; grid::save_grid, gstore.cpp:2818-2829)
 *   degree : int32 per vertex (grid::save_degree_files, gstore.cpp:2911-2917)
 * Geometry (grid::init -v, gstore.cpp:152-161): p = ceil(V / 2^24) groups per
 * dimension, p_s = 256 p tiles per dimension; the undirected layout ("gstoreu",
 * HALF_GRID) stores the upper triangle, p_s (p_s + 1) / 2 tiles; the directed
 * one ("gstored") stores p_s^2 tiles.
 *
 * Ownership: the library owns every device allocation and pinned staging
 * buffer it makes.  The caller owns host arrays and keeps them alive until the
 * call that takes them returns.  All calls are synchronous unless named
 * otherwise.
 * Errors: every call returns gs_status; no call exits or asserts (unlike the
 * reference's handle_error, gstore.h:43-44).  gs_last_error() gives the text
 * of the last failure on a context.
 * Threading: a gs_ctx and everything made from it is single-threaded.
 */
#ifndef GSTORE_CUDA_H
#define GSTORE_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t gs_status;
#define GS_OK 0
#define GS_ERR_CUDA 1      /* a CUDA runtime call failed                     */
#define GS_ERR_OOM 2       /* device or pinned memory exhausted / over budget */
#define GS_ERR_FORMAT 3    /* start/grid/degree inconsistent or out of range  */
#define GS_ERR_TIMEOUT 4   /* a bounded device-side wait gave up              */
#define GS_ERR_ARG 5       /* invalid argument                                */
#define GS_ERR_RANGE 6     /* BFS would exceed 254 levels (u8 depth_t)        */
#define GS_ERR_STATE 7     /* call out of order for this object              */
#define GS_ERR_UNSUPPORTED 8 /* e.g. k-core on a directed grid               */

typedef enum gs_algo {
    GS_ALGO_BFS = 0,      /* bfs_t   (bfs.cpp)   arg = root                 */
    GS_ALGO_PAGERANK = 1, /* pr_t    (pr.cpp)    arg = iterations           */
    GS_ALGO_KCORE = 2,    /* kcore_t (kcore.cpp) arg = k                    */
    GS_ALGO_WCC = 3,      /* wcc2_t  (wcc.cpp)   arg unused                 */
    GS_ALGO_BFS2 = 4,     /* bfs2_t  (bfs2.cpp)  arg = root ("-j 30")       */
    GS_ALGO_TRAVERSE = 5  /* traverse_t (traverse.cpp) arg = pivot ("-j 4") */
} gs_algo;

typedef struct gs_ctx gs_ctx;
typedef struct gs_graph gs_graph;
typedef struct gs_state gs_state;
typedef struct gs_batch gs_batch;
typedef struct gs_server gs_server;

/* A run of consecutive stored tiles, mirroring part_meta_t (gstore.h:563-568):
 * part ids use the reference's encoding (group_full_index << 16 | i << 8 | j,
 * gstore.h:199-220) and start..end is inclusive in file order.  Used by the
 * streamed (semi-external) sweep. */
typedef struct gs_segment {
    uint64_t part_start;
    uint64_t part_end;
} gs_segment;

/* ------------------------------------------------------------ context --- */
/* Replaces: grid::init / read_aio_init set-up (gstore.cpp:132-186, 3044-3119).
 * hbm_budget_bytes bounds the tile bytes kept resident (0 = no bound); it is
 * the "-m" memory budget of the reference reused for HBM. */
gs_status gs_create(gs_ctx** out, int device, uint64_t hbm_budget_bytes, int directed);
gs_status gs_destroy(gs_ctx* ctx);
const char* gs_last_error(const gs_ctx* ctx);
/* Launch all work of this context on an existing cudaStream_t (NULL = the
 * context's own stream). */
gs_status gs_set_stream(gs_ctx* ctx, void* cuda_stream);
/* Enable per-kernel CUDA-event timing (kind: 0 = main sweep kernel). */
gs_status gs_profile(gs_ctx* ctx, int enable);
gs_status gs_kernel_time(gs_ctx* ctx, int algo, uint64_t* launches, double* total_ms,
                         uint64_t* bytes);

/* Number of kernels this context has launched so far (all entry points). */
gs_status gs_launch_count(const gs_ctx* ctx, uint64_t* launches);

/* Geometry of the tile files for vertex count V (grid::init -v). */
gs_status gs_geometry(uint64_t V, int directed, uint32_t* p, uint32_t* p_s,
                      uint64_t* n_start_entries);

/* -------------------------------------------------------------- graph --- */
/* Replaces: read_grid_in_mem + read_degree_in_mem (gstore.cpp:2953-3011).
 * Copies host start[n_start], grid[n_edges] and degree[V] (degree may be NULL:
 * it is then counted on the device from the records) into HBM and builds the
 * tile tables.  Checks: n_start matches the geometry, start is monotone,
 * start[last] == n_edges, every record addresses a vertex below V.  A
 * resident graph whose tiles hold their records out of ascending order (the
 * reference converter writes them in its threads' order, gstore.cpp:1403-1447)
 * has every tile sorted on the device after the copy (the sweeps run about
 * twice as fast on sorted tiles; results do not depend on the order), so
 * gs_graph_download then returns the records sorted inside each tile. */
gs_status gs_upload_graph(gs_ctx* ctx, const uint64_t* start, uint64_t n_start,
                          const uint32_t* grid, uint64_t n_edges,
                          const int32_t* degree, uint64_t V, gs_graph** out);
/* When the context's HBM budget is set and the grid is larger, the graph is
 * streamed (gs_upload_graph_streamed with segment_bytes = budget / 2), and
 * grid must then stay valid and unchanged until gs_graph_free. */

/* Replaces: the semi-external mode of the reference (-m budget: two IO
 * segments refilled by libaio, read_aio_init / fetch_mem_part,
 * gstore.cpp:3044-3119, 3867-3918).  The records stay in host memory (grid
 * is pinned with cudaHostRegister unless it already is; it must stay valid
 * and unchanged until gs_graph_free); every sweep plans the tile runs its
 * skip rule needs and copies them through two HBM buffers of segment_bytes
 * each on a side stream, overlapped with the sweep kernels.  segment_bytes
 * >= 1 MiB + 64 bytes. */
gs_status gs_upload_graph_streamed(gs_ctx* ctx, const uint64_t* start, uint64_t n_start,
                                   const uint32_t* grid, uint64_t n_edges, const int32_t* degree,
                                   uint64_t V, uint64_t segment_bytes, gs_graph** out);
/* Replaces: the disk side of the same mode (records read from the .grid file
 * by libaio into the IO segments, prep_read_aio_*, gstore.cpp:3130-3620).
 * The records stay in the file at grid_path (uint32 records from byte 0,
 * n_edges of them); every sweep plans the runs its skip rule needs, reads
 * them with pread into two pinned staging buffers of segment_bytes each and
 * copies each staged segment to one of two HBM buffers on a side stream: the
 * host reads segment k+1 while the GPU sweeps segment k.  The file must stay
 * unchanged until gs_graph_free.  segment_bytes >= 1 MiB + 64 bytes. */
gs_status gs_upload_graph_file(gs_ctx* ctx, const uint64_t* start, uint64_t n_start, const char* grid_path,
                               uint64_t n_edges, const int32_t* degree, uint64_t V, uint64_t segment_bytes,
                               gs_graph** out);

/* Replaces: read_start_in_mem + read_grid_in_mem + read_degree_in_mem
 * (gstore.cpp:2953-3011, 3799-3813) for both layouts the reference's
 * converters write: the single <prefix>.start / <prefix>.grid of "-c 1" and
 * "-c 2", and the directory layout of "-c 3" -- <prefix>.start.N and
 * <prefix>.grid.N per block of file groups (grid::post_grid_dir,
 * save_start_files(is_odir), gstore.cpp:688-879, 2837-2898), which the
 * reference writes but never reads back.  Their per-file .start.N entries
 * (a running sum of per-row prefix sums) are decoded back to tile counts.
 * Fills start[n_start] (the single-file .start; n_start from gs_geometry),
 * grid[grid_capacity] with the records in single-file order, and degree[V]
 * (.degree, zero past its end); each may be NULL.  *n_edges: the record
 * count.  directed: the full grid of gstored, else the half grid.  No device
 * work: ctx may be NULL (then only the status reports a failure). */
gs_status gs_read_tile_files(gs_ctx* ctx, const char* prefix, uint64_t V, int directed, uint64_t* start,
                             uint64_t n_start, uint32_t* grid, uint64_t grid_capacity, int32_t* degree,
                             uint64_t* n_edges);

/* Replaces: read_aio_init + read_degree_in_mem (gstore.cpp:3044-3119,
 * 2971-3011) over either layout: a graph whose records stay in the file(s)
 * at `prefix` and stream through two HBM segments of segment_bytes each, as
 * gs_upload_graph_file does for one .grid file.  <prefix>.degree is read when
 * present, else the degrees are counted from the records. */
gs_status gs_upload_graph_files(gs_ctx* ctx, const char* prefix, uint64_t V, uint64_t segment_bytes,
                                gs_graph** out);
/* Host-to-device traffic of a streamed graph since upload: bytes copied,
 * cudaMemcpyAsync calls, segments swept, segments found already in HBM
 * (all 0 for a resident graph). */
gs_status gs_stream_stats(const gs_graph* g, uint64_t* bytes_copied, uint64_t* copies,
                          uint64_t* segments, uint64_t* segments_reused);
/* The same from device pointers (e.g. produced by gs_convert_device); the
 * library copies them, the caller keeps ownership. */
gs_status gs_upload_graph_device(gs_ctx* ctx, const uint64_t* d_start, uint64_t n_start,
                                 const uint32_t* d_grid, uint64_t n_edges,
                                 const int32_t* d_degree, uint64_t V, gs_graph** out);
gs_status gs_graph_free(gs_graph* g);
/* Counts: records, non-empty tiles, work items, vertex count. */
gs_status gs_graph_info(const gs_graph* g, uint64_t* n_edges, uint64_t* n_tiles,
                        uint64_t* n_items, uint64_t* V);
/* Copy the graph's degree array (V int32) to the host. */
gs_status gs_graph_degree(const gs_graph* g, int32_t* host_degree);

/* ------------------------------------------------- algo_t plug-in layer --- */
/* Replaces: bfs_t/pr_t/kcore_t/wcc2_t/bfs2_t/traverse_t ::init (bfs.cpp:56-75,
 * pr.cpp:82-117, kcore.cpp:55-61, wcc.cpp:57-83, bfs2.cpp:56-78,
 * traverse.cpp:56-72).  arg: BFS / BFS2 root, PageRank iterations, k-core k,
 * TRAVERSE pivot; unused for WCC.  The state lives in HBM. */
gs_status gs_state_create(gs_graph* g, gs_algo algo, int64_t arg, gs_state** out);
gs_status gs_state_free(gs_state* s);
/* Re-initialise a state for a new run (new root / iterations / k) without
 * reallocating its device arrays. */
gs_status gs_state_reset(gs_state* s, int64_t arg);
/* Replaces: algo_t::algo_mem_part(segment*) (algo.h:40): sweeps the tiles of
 * the given part ranges (segs, n_segs), or every tile when n_segs == 0,
 * applying the algorithm's own tile-skip rule.  As in the reference, one
 * level or iteration may be swept by several calls (one per segment); the
 * next gs_finalize closes it.  With n_segs == 0 a streamed graph plans its
 * own segments from the skip rule and streams them. */
gs_status gs_sweep(gs_state* s, const gs_segment* segs, int n_segs);
/* Replaces: iteration_finalize() (bfs.cpp:187-224, pr.cpp:229-303,
 * kcore.cpp:179-217, wcc.cpp:281-395).  frontier_out: BFS vertices found in
 * the last sweep, k-core vertices removed, WCC labels changed, PageRank the
 * iteration just finished.  done_out: 1 when the algorithm has finished. */
gs_status gs_finalize(gs_state* s, int64_t* frontier_out, int* done_out);
/* Sweep + finalize until done, all on the device (one 8-byte read per step).
 * steps_out: number of sweeps. */
gs_status gs_run(gs_state* s, int64_t* steps_out);

/* Results.  BFS and BFS2: uint8 depth[V] (root 1, unreached 0, bfs.cpp:54;
 * the label-correcting bfs2 ends at the same depths).  TRAVERSE: uint32
 * cid[V], 0 for vertices reached from the pivot along records v0 -> v1,
 * 0xFFFFFFFF for the others (traverse.cpp:56-188).
 * PageRank: float rank[V] = 0.15 + 0.85 s after the last iteration
 * (what = 0) or float x[V] = rank * inv_degree (what = 1, the reference's
 * vert_rank_prior after its final swap).  k-core: int32 degree[V] (final,
 * removed vertices 0 or negative, kcore.cpp:179-217).  WCC: uint32 label[V],
 * the smallest vertex id of the component, 0xFFFFFFFF for vertices without
 * records (wcc.cpp:54). */
gs_status gs_download(gs_state* s, int what, void* host_dst, uint64_t bytes);
/* Scalar summary: BFS / BFS2 reached vertices, k-core members (deg != 0,
 * gstore.cpp:2796-2803), WCC component count (wcc.cpp:324-336), TRAVERSE
 * vertices with colour 0. */
gs_status gs_result_count(gs_state* s, uint64_t* count);
/* BFS: records with both endpoints reached (the GTEPS numerator) and the
 * records swept per level under the reference's tile-skip rule. */
gs_status gs_bfs_stats(gs_state* s, uint64_t* edges_in_component, uint64_t* swept_records,
                       int max_levels, int* n_levels, uint64_t* level_counts);
/* BFS: records the sweep kernel actually read per level (resident graphs
 * skip 256-record chunks whose records all had both ends visited at an
 * earlier level: such a record can discover nothing, so depths are the
 * same; a streamed graph reads every record of the swept tiles).  Same
 * reference rule otherwise as gs_bfs_stats; no counterpart in the
 * reference, which reads every record of a swept tile. */
gs_status gs_bfs_records_read(gs_state* s, uint64_t* read_records, int max_levels, int* n_levels);

/* BFS without any allocation (no counterpart in the reference; added for
 * callers that may not allocate device memory while they run queries, such
 * as a host framework whose memory pool already owns the GPU, or a serving
 * loop that cannot take the device-wide synchronisation of cudaMalloc).
 * Runs the same sweep kernels as gs_run on a BFS state, keeps its scratch
 * state in a fixed array inside the library (about 6 MiB per GPU, for the
 * life of the process) and writes uint8 depth[V] (root 1, unreached 0) into
 * the caller's device buffer d_depth.  Limit: V <= 16777216 (else
 * GS_ERR_RANGE).  The first call on a device looks the array up; make it
 * before any stream capture.  Calls overlapping on one GPU share the array
 * and race: issue them one after another.  d_depth is cleared and written on
 * the context's stream (gs_set_stream); the caller must have finished any
 * other use of that buffer before the call, or ordered that use before it on
 * the context's stream (for instance with an event the stream waits on).
 * The call is synchronous: when it returns, d_depth holds the result.
 * levels_out (may be NULL): sweeps done. */
gs_status gs_bfs_noalloc(gs_graph* g, uint64_t root, uint8_t* d_depth, int64_t* levels_out);

/* ------------------------------------------------------------ batching --- */
/* Replaces: one gstoreu process per query (the job dispatch of
 * gstore.cpp:250-333 runs a single BFS / WCC / k-core / PageRank).  A batch
 * collects queries on resident graphs of one context and runs them with few
 * launches: BFS roots on the same graph run as a multi-source BFS (one bit
 * per query in 32- or 64-bit frontier words, one persistent launch per
 * group, word width and tile order picked per graph by a measuring
 * autotuner); all k-core queries, and WCC queries on graphs of fewer
 * than 2^22 records, over any graphs, share one persistent launch; WCC
 * queries on larger graphs (whose plain WCC hooks a sample of the records
 * first and then skips the records inside the largest tree) and PageRank
 * queries run as plain gs_run; identical queries
 * (same graph, algorithm and argument) run once.  Results per
 * query equal gs_run's on the same graph and argument (BFS depth, WCC
 * labels, k-core degrees bit for bit).  arg: BFS root, k-core k, PageRank
 * iterations (ignored for WCC).  gs_batch_run runs every query added since
 * the last run; query ids stay valid until gs_batch_free. */
gs_status gs_batch_create(gs_ctx* ctx, gs_batch** out);
gs_status gs_batch_add(gs_batch* b, gs_graph* g, gs_algo algo, int64_t arg, int* query_id);
gs_status gs_batch_run(gs_batch* b);
/* Same formats as gs_download / gs_result_count; a query that failed
 * returns its status (e.g. GS_ERR_RANGE for a BFS over 254 levels). */
gs_status gs_batch_download(gs_batch* b, int query_id, int what, void* host_dst, uint64_t bytes);
gs_status gs_batch_result_count(gs_batch* b, int query_id, uint64_t* count);
/* BFS query: vertices found per level (iteration_finalize's frontier
 * counts; the last level found none). */
gs_status gs_batch_bfs_levels(gs_batch* b, int query_id, uint64_t* level_counts, int max_levels,
                              int* n_levels);
/* Launches so far: the persistent launches plus one per query run as a
 * plain gs_run (PageRank, and WCC on graphs of >= 2^22 records); kernel_ms
 * is the persistent launches' device time. */
gs_status gs_batch_stats(const gs_batch* b, uint64_t* launches, double* kernel_ms);
gs_status gs_batch_free(gs_batch* b);

/* ------------------------------------------------------------- serving --- */
/* Replaces: one gstoreu process per query (gstore.cpp:250-333), as a
 * request loop.  Graphs are registered resident graphs; requests (BFS root,
 * k-core k, PageRank iterations, WCC) are queued by gs_serve_submit and
 * advanced by gs_serve_step, which never blocks on side work.  Each step
 * admits queued requests in arrival order while their device state fits
 * state_budget_bytes (0 = 32 GiB) and a slot is free; runs one level of
 * every graph's BFS group (up to 64 BFS requests per graph share
 * bit-parallel frontier words and join at any level) in one CUDA-graph
 * launch; and advances the WCC / k-core / PageRank requests, which run to
 * completion on lower-priority side streams in chunks of iterations (64
 * slots).  Finished requests are retired into pinned host buffers and
 * listed by gs_serve_completed.  A request identical to one queued or
 * running (same graph, algorithm and argument) shares its run.  Results
 * equal gs_run's for the same query (BFS/WCC/k-core bit for bit, PageRank
 * within float rounding).  Times are seconds of the server's steady clock
 * (gs_serve_clock).  States: 0 queued, 1 running, 2 done, 3 failed. */
gs_status gs_serve_create(gs_ctx* ctx, uint64_t state_budget_bytes, gs_server** out);
gs_status gs_serve_add_graph(gs_server* s, gs_graph* g, int* graph_id);
gs_status gs_serve_submit(gs_server* s, int graph_id, gs_algo algo, int64_t arg, uint64_t* request_id);
gs_status gs_serve_step(gs_server* s, int* n_active, int* n_queued);
gs_status gs_serve_poll(gs_server* s, uint64_t request_id, int* state);
/* Ids of requests finished (done or failed) since the last call, oldest
 * first, at most max_ids of them; *n = how many were written. */
gs_status gs_serve_completed(gs_server* s, uint64_t* ids, int max_ids, int* n);
/* Side streams the WCC / k-core / PageRank requests spread over (1-8,
 * default 8); only while none of those requests is running. */
gs_status gs_serve_set_side_streams(gs_server* s, int n);
/* Copies a finished request's result (gs_download's format; host_dst may be
 * NULL) and forgets the request.  A failed request returns its status. */
gs_status gs_serve_result(gs_server* s, uint64_t request_id, void* host_dst, uint64_t bytes,
                          double* t_submit, double* t_done, int64_t* steps);
/* The same result without a copy: *data points to *bytes bytes in the
 * server's pinned host buffer (gs_download's format), valid until
 * gs_serve_release(s, request_id), which forgets the request.  A failed
 * request returns its status and is forgotten at once. */
gs_status gs_serve_result_view(gs_server* s, uint64_t request_id, const void** data, uint64_t* bytes,
                               double* t_submit, double* t_done, int64_t* steps);
gs_status gs_serve_release(gs_server* s, uint64_t request_id);
gs_status gs_serve_clock(const gs_server* s, double* seconds);
gs_status gs_serve_stats(const gs_server* s, uint64_t* steps, uint64_t* graph_launches,
                         uint64_t* kernel_launches, uint64_t* hbm_in_use);
/* Host seconds spent in gs_serve_step so far, by phase (up to n of them):
 * [0] admission, [1] BFS step launch, [2] side requests (WCC / k-core /
 * PageRank chunks, their polling and retirement), [3] BFS step finish (the
 * wait for the step, retirement of BFS slots); then, counted inside those
 * phases, [4] seconds and [5] number of pinned host allocations (result
 * arena misses; gs_serve_reserve_host is not one), [6] seconds and [7]
 * number of device allocations (pool misses). */
gs_status gs_serve_profile(const gs_server* s, double* seconds, int n);
/* Pins `bytes` of host memory into the server's result arena now, so that
 * results up to that total land without pinning pages while requests are
 * served (pinning runs at a few GB/s on the host).  Results are carved from
 * the arena best-fit; a miss pins a further chunk of at least 64 MiB.  No
 * counterpart in the reference, which answers one query per process. */
gs_status gs_serve_reserve_host(gs_server* s, uint64_t bytes);
gs_status gs_serve_free(gs_server* s);

/* PageRank with the reference's int32 inverse-degree truncation
 * (pr.cpp:112-114) instead of the real inverse; must precede gs_run. */
gs_status gs_pagerank_compat(gs_state* s, int enable);

/* ------------------------------------------- generator and converter --- */
/* Graph500 Kronecker generator (graph500-generator/graph_generator.c,
 * make_graph.c), byte-identical output: 2 * (edgefactor << scale) uint32
 * written to device memory d_pairs (caller-allocated). */
gs_status gs_kron_generate_device(gs_ctx* ctx, int scale, int64_t edgefactor,
                                  uint64_t seed1, uint64_t seed2, uint32_t* d_pairs);
/* The same into host memory. */
gs_status gs_kron_generate(gs_ctx* ctx, int scale, int64_t edgefactor, uint64_t seed1,
                           uint64_t seed2, uint32_t* host_pairs);
/* Converter "-c 1" (grid::pre_grid + proc_grid, gstore.cpp:1245-1458) on the
 * device: edge pairs (host or device pointer, is_device) -> a resident graph.
 * Self-loops dropped, duplicates kept, (min,max) order for the half grid.
 * In-tile record order is not specified (the reference's is thread order). */
gs_status gs_convert(gs_ctx* ctx, const uint32_t* pairs, uint64_t n_pairs, int is_device,
                     uint64_t V, gs_graph** out);
/* Copy a resident graph back into host start/grid/degree arrays (sizes from
 * gs_graph_info / gs_geometry), e.g. to write .start/.grid/.degree files. */
gs_status gs_graph_download(const gs_graph* g, uint64_t* host_start, uint32_t* host_grid,
                            int32_t* host_degree);

#ifdef __cplusplus
}
#endif
#endif
