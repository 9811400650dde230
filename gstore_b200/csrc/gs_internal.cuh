// Internal declarations of libgstore_cuda.so (not part of the C ABI).
#pragma once

#include "gstore_cuda.h"

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <vector>

// Tile geometry constants of the reference (gstore.h:77-104).
constexpr int kTileBits = 16;          // bit_shift2: a tile spans 2^16 vertices
constexpr uint32_t kGroupTiles = 256;  // p_p: tiles per physical group side
constexpr int kGroupBits = 24;         // bit_shift1: a group spans 2^24 vertices
// Upper bound of records per work item (a slice of one tile).
constexpr uint32_t kItemRecords = 4096;

// One work item: records [beg, beg + cnt) of the tile at global tile row
// `row`, column `col` (every record of an item lies in that one tile).
struct alignas(16) gs_item {
    uint64_t beg;
    uint32_t cnt;
    uint32_t rc;  // row << 16 | col
};

// Upper bound of records per run.
constexpr uint64_t kRunRecords = 131072;
// Zeroed records after the last one, so 16-byte-rounded bulk copies of a
// record range stay inside the allocation.
constexpr uint64_t kRecPad = 4;

// One run: consecutive non-empty tiles [tile_beg, tile_end) of the tile table
// that share a tile row and a group (contiguous in the file), restricted to
// records [rec_beg, rec_end).  A tile larger than kRunRecords is cut into
// several single-tile runs.
struct alignas(8) gs_tile_run {
    uint64_t rec_beg;
    uint64_t rec_end;
    uint32_t tile_beg;
    uint32_t tile_end;
    uint32_t unit_beg;   // the run's units [unit_beg, unit_end) of the unit table
    uint32_t unit_end;
};

// Records per BFS unit.
constexpr uint32_t kUnitRecords = 2048;
// Side of a block of the L2-blocked sweep order, in windows.
constexpr uint32_t kBlockWindows = 64;
constexpr uint32_t kBlockWindowsSmall = 32;
// Units per run of the L2-blocked order.
constexpr uint32_t kBlockRunUnits = 8;
constexpr uint32_t kBfsMinRunUnits = 8;     // BFS sweep: smallest run piece
constexpr uint64_t kBfsRunsPerCta = 4;      // BFS sweep: run pieces wanted per CTA
constexpr int kBfsCtasPerSm = 5;            // BFS sweep: resident CTAs per SM

// One unit: records [rec_beg, rec_beg + n) of the tile at row rc >> 16,
// column rc & 0xFFFF (n <= kUnitRecords; units follow the file order).
struct alignas(16) gs_unit {
    uint64_t rec_beg;
    uint32_t n;
    uint32_t rc;
};

// One entry of a segment sweep: units [unit_beg, unit_end) of run `run`,
// whose records sit in the segment buffer at (file record index + delta).
// delta is a multiple of 4, so 16-byte record alignment carries over.
struct alignas(8) gs_seg_run {
    uint32_t run;
    uint32_t unit_beg;
    uint32_t unit_end;
    uint32_t pad;
    int64_t delta;
};

// The segment a sweep currently works on (list == nullptr: every run of the
// resident graph).
struct SegView {
    const gs_seg_run* list = nullptr;
    uint32_t n = 0;
    const uint32_t* buf = nullptr;
};

// PageRank row-slice layout (gs_pagerank.cu): a second copy of the records,
// each tile's records grouped by row slice (v0 >> 13, 8 slices of 8192
// vertices) and sorted by v1 inside a slice; work items are (row window,
// slice, block of kPrColBlock column windows), their units <= kUnitRecords
// records of one tile and slice.
constexpr int kPrSliceBits = 13;
constexpr uint32_t kPrColBlock = 32;
struct gs_pr_item {
    uint32_t unit_beg, unit_end;
    uint32_t row, slice;
};
struct gs_pr_layout {
    uint32_t* d_rec = nullptr;
    gs_unit* d_units = nullptr;
    gs_pr_item* d_items = nullptr;
    uint64_t n_units = 0, n_items = 0;
    bool built = false;
};

// PageRank propagation-blocked layout (gs_pr_blocked.cu): one entry per
// (record, direction), sorted by (source slice, destination bin); u16 offsets
// of the source in its slice and of the destination in its bin, one float
// value per entry written by the gather pass, and for the accumulate pass the
// list of every bin's 8-entry groups (its blocks in slice order).
constexpr int kPbSrcBits = 14;   // source slice: 16,384 vertices (x staged in shared memory)
constexpr int kPbDstBits = 14;   // destination bin: 16,384 vertices (sums in shared memory)
struct gs_pb_item1 {             // gather item: entries [e0, e0 + n) of source slice `slice`
    uint64_t e0;
    uint32_t n, slice;
};
struct gs_pb_item2 {             // accumulate item: groups [b0, b1) of the group list, all of bin `bin`
    uint32_t b0, b1, bin, whole;
};
struct gs_pb_block {             // entries [e0, e0 + n) of one (slice, bin) block
    uint64_t e0;
    uint32_t n, pad;
};
struct gs_pb_layout {
    uint16_t* d_src = nullptr;
    uint16_t* d_dst = nullptr;
    float* d_val = nullptr;
    uint32_t* d_groups = nullptr;   // per bin, in slice order: the 8-entry groups of its blocks (entry index / 8)
    gs_pb_item1* d_items1 = nullptr;
    gs_pb_item2* d_items2 = nullptr;
    uint64_t n_entries = 0, n_groups = 0, n_items1 = 0, n_items2 = 0;
    bool built = false;
};

struct gs_streamer;   // pinned-host record stream of a graph (gs_stream.cu)
struct gs_seglists;   // double-buffered entry lists of segment sweeps (gs_stream.cu)

struct KernelTimes {
    uint64_t launches = 0;
    double ms = 0.0;
    uint64_t bytes = 0;
};

struct gs_ctx {
    int device = 0;
    int directed = 0;
    uint64_t budget = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;
    bool profile = false;
    KernelTimes ktime[8];
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    uint64_t* d_scalars = nullptr;   // small device scratch for counters/flags
    // run tickets of the persistent sweeps on `stream` ([0..1] generic sweep,
    // [2..3] PageRank row-slice sweep, [4..5] and [6..7] the two passes of the
    // propagation-blocked PageRank sweep): zero at launch, zeroed again by the
    // last CTA
    unsigned int* d_ticket = nullptr;
    uint64_t* h_scalars = nullptr;   // pinned mirror
    int num_sms = 148;
    uint64_t launches = 0;           // kernels launched on this context
    // device blocks returned by finished batches, by exact size (reused by
    // the next batch instead of cudaMalloc / cudaFree)
    std::multimap<size_t, void*> pool_free;
    uint64_t pool_bytes = 0;
};

struct gs_graph {
    gs_ctx* ctx = nullptr;
    int directed = 0;
    uint64_t V = 0;      // vertex count given by the caller
    uint64_t N = 0;      // padded vertex count: nw * 2^16
    uint32_t p = 0, p_s = 0, nw = 0;
    uint64_t T_all = 0;  // stored tiles (.start entries - 1)
    uint64_t E = 0;      // records
    uint64_t T = 0;      // non-empty tiles
    uint64_t I = 0;      // work items
    uint64_t R = 0;      // runs
    uint64_t U = 0;      // units
    uint32_t* d_rec = nullptr;
    gs_item* d_items = nullptr;
    gs_tile_run* d_runs = nullptr;
    gs_unit* d_units = nullptr;
    gs_tile_run* d_runs_lpt = nullptr; // BFS sweep: runs (maybe cut into pieces), longest first (resident)
    uint64_t R_lpt = 0;
    bool blocked_built = false;       // the two blocked orders below exist (gs_ensure_blocked)
    uint64_t R_blk = 0;               // runs of the L2-blocked order (resident graphs)
    gs_tile_run* d_runs_blk = nullptr;
    gs_unit* d_units_blk = nullptr;
    uint64_t R_blk2 = 0;              // the same with kBlockWindowsSmall blocks
    gs_tile_run* d_runs_blk2 = nullptr;
    gs_unit* d_units_blk2 = nullptr;
    uint64_t* d_tile_off = nullptr;   // T + 1 record offsets of non-empty tiles
    uint32_t* d_tile_rc = nullptr;    // T packed (row << 16 | col)
    int32_t* d_degree = nullptr;      // N
    uint64_t nonisolated = 0;         // vertices with degree > 0 (counted at the first BFS)
    bool nonisolated_known = false;
    SegView seg;                      // set during segment sweeps
    gs_pr_layout pr;                  // row-slice PageRank layout (serving, batches, smaller graphs)
    gs_pb_layout pb;                  // propagation-blocked PageRank layout (gs_run on large graphs)
    gs_streamer* stream = nullptr;    // non-null: records stay in host memory
    gs_seglists* lists = nullptr;     // segment entry lists of segment sweeps
    std::vector<gs_tile_run> h_runs;  // host copies of the run and unit tables
    std::vector<gs_unit> h_units;
    bool degree_from_records = false;
    std::vector<uint64_t> h_start;    // full .start copy (host), for planners
    std::vector<uint64_t> h_tile_off; // host copy of d_tile_off
    std::vector<uint32_t> h_tile_rc;  // host copy of d_tile_rc
    // device buffers above taken from the context's pool (gs_graph_alloc),
    // with their sizes: returned to the pool when the graph is freed
    std::vector<std::pair<void*, size_t>> pooled;
};

struct gs_state {
    gs_graph* g = nullptr;
    gs_algo algo = GS_ALGO_BFS;
    int64_t arg = 0;
    int step = 0;          // sweeps done (counted at finalize)
    bool swept = false;    // a sweep happened since the last finalize
    bool done = false;
    bool compat = false;   // PageRank int32 inverse-degree truncation
    // BFS
    uint8_t level = 1;
    uint8_t* d_depth = nullptr;      // N
    uint32_t* d_front = nullptr;     // N/32 frontier words
    uint32_t* d_visited = nullptr;   // N/32 words: discovered-this-sweep bitmap
    uint64_t* d_error = nullptr;     // bounded-wait failure flag
    uint32_t* d_ticket = nullptr;    // BFS sweep: run ticket, finished CTAs
    uint8_t* d_dead = nullptr;       // BFS: per unit, chunks with no record left to discover anything
    bool marking = false;            // BFS: dead chunks are being marked (and skipped)
    bool sweep_mark = false, sweep_skip = false;   // BFS: this level's mode (set per sweep)
    std::vector<uint8_t> level_skip; // BFS: per level, dead chunks were skipped (records read counted)
    unsigned long long* d_read = nullptr;   // BFS: records read per level (256)
    uint8_t* d_act = nullptr;        // nw window flags (current)
    uint8_t* d_act_next = nullptr;   // nw
    std::vector<uint64_t> level_counts;
    uint8_t* d_act_hist = nullptr;   // 256 x nw: each level's window flags (swept-record statistics)
    int n_act_hist = 0;              // levels recorded in d_act_hist
    // PageRank
    float* d_x = nullptr;            // N
    float* d_y = nullptr;            // N
    float* d_r = nullptr;            // N
    // WCC
    uint32_t* d_parent = nullptr;    // N
    uint8_t* d_touched = nullptr;    // N
    uint32_t* d_giant = nullptr;     // N/32 + 2 words: largest sampled tree's bitmap, then its root
    bool wcc_giant = false;          // d_giant was built by this run's first sweep
    // k-core
    int32_t* d_deg = nullptr;        // N
    uint32_t* d_kactive = nullptr;   // N/32
    // bfs2 / traverse
    uint32_t* d_lab = nullptr;       // N: depth (bfs2) or colour (traverse)
    int64_t last_count = 0;
    uint32_t* d_out = nullptr;       // N x 4 B: staging of derived results (WCC labels, bfs2 depth)
    // every device buffer above, taken from the context's pool (gs_state_alloc)
    // and returned to it by gs_state_free
    std::vector<std::pair<void*, size_t>> allocs;
};

// ---------------------------------------------------------------- errors --
gs_status gs_fail(gs_ctx* ctx, gs_status code, const std::string& msg);
gs_status gs_cuda_fail(gs_ctx* ctx, cudaError_t e, const char* what);

#define GS_CHECK_CUDA(ctx, call)                                  \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return gs_cuda_fail((ctx), e_, #call); \
    } while (0)

#define GS_TRY(call)                          \
    do {                                      \
        gs_status s_ = (call);                \
        if (s_ != GS_OK) return s_;           \
    } while (0)

// --------------------------------------------------------------- geometry --
inline uint64_t gs_calc_index_half(uint64_t i, uint64_t j, uint64_t pc) {
    return ((i * ((pc << 1) - i - 1)) >> 1) + j;   // calc_index, gstore.h:109-113
}
// First .start index of group (gi, gj): beg_edge_offset1/2 (gstore.h:128-178).
inline uint64_t gs_group_base(uint64_t gi, uint64_t gj, uint64_t p, int directed) {
    if (directed) return (gi * p + gj) << 16;
    if (gi == gj) return ((gs_calc_index_half(gi, gi, p) - gi) << 16) + ((gi * 257) << 7);
    return ((gs_calc_index_half(gi, gj, p) - gi - 1) << 16) + (((gi + 1) * 257) << 7);
}
void gs_geometry_of(uint64_t V, int directed, uint32_t* p, uint32_t* p_s, uint64_t* n_tiles);

// ------------------------------------------------------- device launchers --
gs_status gs_dev_alloc(gs_ctx* ctx, void** ptr, size_t bytes);
gs_status gs_alloc_records(gs_ctx* ctx, uint32_t** ptr, uint64_t n_records);
void gs_dev_free(void* ptr);
// Context pool: a cached block of exactly `bytes` (rounded to 256), or a new
// one; gs_pool_put returns it (blocks beyond kPoolMaxBytes are freed).
gs_status gs_pool_get(gs_ctx* ctx, size_t bytes, void** out);
// A buffer of a query state from the context's pool, recorded in s->allocs.
gs_status gs_state_alloc(gs_state* s, void** ptr, size_t bytes);
// Builds the L2-blocked run orders of a resident graph on first use.
gs_status gs_ensure_blocked(gs_graph* g);
void gs_pool_put(gs_ctx* ctx, void* ptr, size_t bytes);
void gs_pool_clear(gs_ctx* ctx);
// A buffer of a graph from the context's pool, recorded in g->pooled; and
// the same for a record buffer (n_records + kRecPad zero-padded entries).
gs_status gs_graph_alloc(gs_graph* g, void** ptr, size_t bytes);
gs_status gs_graph_alloc_records(gs_graph* g, uint32_t** ptr, uint64_t n_records);
// Returns a graph buffer: to the pool when it came from there, else cudaFree.
void gs_graph_release(gs_graph* g, void* ptr);

gs_status launch_validate_records(gs_graph* g, int* d_flag);
gs_status launch_degree_from_records(gs_graph* g);

// Per algorithm: init, sweep_begin (once per sweep, before its launches),
// sweep_launch (once per segment in g->seg, or once over the resident
// graph), finalize.
// Counts the graph's vertices with degree > 0 into g->nonisolated (once).
gs_status gs_graph_nonisolated(gs_graph* g);
gs_status bfs_init(gs_state* s);
gs_status bfs_sweep_begin(gs_state* s);
gs_status bfs_sweep_launch(gs_state* s);
gs_status bfs_finalize(gs_state* s, int64_t* frontier, int* done);

gs_status pr_init(gs_state* s);
gs_status pr_layout_build(gs_graph* g);
void pr_layout_free(gs_graph* g);
gs_status pr_slice_launch(gs_state* s);
gs_status pr_slice_sweep(gs_graph* g, cudaStream_t stream, const float* x, float* y, int* error,
                         bool item_ctas = false);
gs_status pr_finalize_launch(gs_ctx* ctx, cudaStream_t stream, float* x, float* y, float* r, const int32_t* deg,
                             uint64_t N, uint64_t V, int compat);
gs_status pr_sweep_launch(gs_state* s);
// Propagation-blocked PageRank (gs_pr_blocked.cu): whether the layout is worth
// building for this graph (and fits), building and freeing it, one sweep.
bool pb_layout_wanted(const gs_graph* g);
gs_status pb_layout_build(gs_graph* g);
void pb_layout_free(gs_graph* g);
gs_status pb_launch(gs_state* s);
// One sweep on `stream` into `y`, with the caller's value stream `val`
// (n_entries floats): one CTA per item, no ticket (the serving loop's side
// streams).
gs_status pb_sweep_on(gs_graph* g, cudaStream_t stream, const float* x, float* y, int* error, float* val);
gs_status pr_finalize(gs_state* s, int64_t* frontier, int* done);

gs_status wcc_init(gs_state* s);
gs_status wcc_sweep_begin(gs_state* s);
gs_status wcc_sweep_launch(gs_state* s);
// Sample of the first WCC sweep on graph g (one 16-byte record group in
// 2^shift hooked before the full pass); 0 = the plain one-sweep form
// (streamed graphs, graphs under 2^22 records, or GS_WCC_SAMPLE_SHIFT=0).
uint32_t gs_wcc_sample_shift(const gs_graph* g);
gs_status wcc_finalize(gs_state* s, int64_t* frontier, int* done);

gs_status kcore_init(gs_state* s);
gs_status kcore_sweep_launch(gs_state* s);
gs_status kcore_finalize(gs_state* s, int64_t* frontier, int* done);

// ------------------------------------------------------- segment sweeps --
// Which units a planned sweep needs (the algorithms' tile-skip rules).
struct gs_need {
    const uint8_t* act = nullptr;   // host window flags; null = every unit
    bool by_col = true;             // a unit is needed when its row or column window is active
    const uint8_t* dead_units = nullptr;   // host, per unit: non-zero = no live chunk left (BFS); null = none
};
// Calls `launch` once per segment with g->seg set: for a streamed graph the
// segments are planned from `need` and their records copied from pinned host
// memory on a side stream, overlapped with the launches; for a resident
// graph `launch` runs once over every run.  direction != 0 walks the
// segments last to first (a streamed graph then reuses the segment that
// the previous sweep left in HBM).
gs_status gs_each_segment_fn(gs_graph* g, const gs_need& need, int direction,
                             gs_status (*fn)(void*), void* arg);
template <class F>
gs_status gs_each_segment(gs_graph* g, const gs_need& need, int direction, F launch) {
    return gs_each_segment_fn(g, need, direction,
                              [](void* a) -> gs_status { return (*static_cast<F*>(a))(); }, &launch);
}
// The same for the tiles of reference part ranges (gs_segment list).
gs_status gs_each_part_fn(gs_graph* g, const gs_segment* segs, int n_segs, gs_status (*fn)(void*), void* arg);
template <class F>
gs_status gs_each_part(gs_graph* g, const gs_segment* segs, int n_segs, F launch) {
    return gs_each_part_fn(g, segs, n_segs,
                           [](void* a) -> gs_status { return (*static_cast<F*>(a))(); }, &launch);
}
gs_status gs_stream_open(gs_graph* g, const uint32_t* host_grid, uint64_t segment_bytes);
// Where a graph's records lie on disk: records [rec_beg, rec_beg + n) of the
// file order (the order of one .grid file) sit contiguously at record
// offset file_rec of file `file`.  One piece for a .grid file; one per
// (file, group row) for the multi-file layout of "-c 3".
struct gs_grid_piece {
    uint64_t rec_beg, n, file_rec;
    uint32_t file, pad;
};
struct gs_tile_layout {
    std::vector<uint64_t> start;          // the .start of the single-file layout
    std::vector<std::string> files;
    std::vector<gs_grid_piece> pieces;    // ascending rec_beg, covering [0, start.back())
};
// Reads <prefix>.start / .grid (the single-file layout) or the per-file
// <prefix>.start.N / .grid.N of "-c 3" (gs_files.cpp).
gs_status gs_read_layout(gs_ctx* ctx, const std::string& prefix, uint64_t V, int directed, gs_tile_layout* L);
// Reads `degree` entries (<= V) of <prefix>.degree; missing entries stay 0.
gs_status gs_read_degree(gs_ctx* ctx, const std::string& prefix, uint64_t V, int32_t* degree);
// Records [rec, rec + n) of a layout's files into dst.
bool gs_read_pieces(const std::vector<int>& fds, const std::vector<gs_grid_piece>& pieces, uint32_t* dst,
                    uint64_t rec, uint64_t n);
// A graph whose records stay in the files of `L`.
gs_status gs_stream_open_layout(gs_graph* g, const gs_tile_layout& L, uint64_t segment_bytes);
void gs_stream_close(gs_graph* g);
const uint32_t* gs_stream_records(const gs_graph* g);   // host records of a streamed graph (null: file-backed)
// A graph whose records stream from the .grid file at `path` (from byte 0).
gs_status gs_stream_open_file(gs_graph* g, const char* path, uint64_t segment_bytes);
// Copies a streamed graph's records (from memory or the file) to dst.
bool gs_stream_read_records(const gs_graph* g, uint32_t* dst);

// bfs2 (-j 30) and traverse (-j 4): one u32 label per vertex in d_lab
gs_status lab_init(gs_state* s);
gs_status lab_sweep_begin(gs_state* s);
gs_status lab_sweep_launch(gs_state* s);
gs_status lab_finalize(gs_state* s, int64_t* frontier, int* done);
gs_status lab_result(gs_state* s, uint8_t* d_out, uint64_t* count);

gs_status gs_count_reached(gs_state* s, uint64_t* reached, uint64_t* edges_in_component);
gs_status gs_count_kcore(gs_state* s, uint64_t* members);
gs_status gs_wcc_labels(gs_state* s, uint32_t* d_out, uint64_t* count);
gs_status gs_swept_records(gs_state* s, const uint8_t* h_act, uint64_t* swept);

gs_status gs_kron_gen_launch(gs_ctx* ctx, int scale, int64_t ef, uint64_t s1, uint64_t s2,
                             uint32_t* d_pairs);
gs_status gs_convert_launch(gs_ctx* ctx, const uint32_t* d_pairs, uint64_t n_pairs, uint64_t V,
                            int directed, uint64_t** d_start_out, uint32_t** d_grid_out,
                            int32_t** d_degree_out, uint64_t* n_start, uint64_t* n_rec);

gs_status gs_sort_tiles(gs_ctx* ctx, const uint64_t* d_start, uint64_t n_tiles, uint32_t* d_rec, uint64_t n_rec);
// A resident graph whose tiles hold their records out of ascending order
// (the reference converter leaves them in its threads' order) gets every
// tile sorted: the sweeps' column-side state lookups then walk neighbouring
// words.  Results do not depend on the in-tile order.
gs_status gs_order_tiles(gs_graph* g, bool* sorted_now);
gs_status gs_graph_adopt(gs_ctx* ctx, uint64_t V, const uint64_t* d_start, uint64_t n_start, uint32_t* d_rec,
                         uint64_t n_edges, const int32_t* d_degree, gs_graph** out);

gs_status bfs_seed_into(gs_ctx* ctx, uint8_t* depth, uint32_t* st, uint8_t* act, uint64_t root);
gs_status bfs_level_into(gs_ctx* ctx, const gs_graph* g, uint8_t* depth, uint32_t* st, uint32_t* next,
                         uint8_t* act, uint8_t* act_next, unsigned long long* count, int* error,
                         unsigned int* ticket, uint8_t next_level);

// Timing helpers around the main sweep kernel of an algorithm.
void gs_timer_begin(gs_ctx* ctx);
void gs_timer_end(gs_ctx* ctx, int algo, uint64_t bytes);

inline uint32_t gs_grid_size(const gs_ctx* ctx, int per_sm) { return (uint32_t)ctx->num_sms * per_sm; }

// Raises Kernel's dynamic shared-memory limit to `bytes` once per device (the
// device must be current).  Host threads that drive contexts on different
// devices may call it concurrently: each device's attempt runs exactly once
// and every caller sees its result.
template <auto Kernel>
inline cudaError_t gs_smem_limit_once(int device, int bytes) {
    static std::once_flag once[64];
    static cudaError_t result[64];
    const int d = device & 63;
    std::call_once(once[d], [&] {
        result[d] = cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    });
    return result[d];
}
