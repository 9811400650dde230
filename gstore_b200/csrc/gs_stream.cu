// Segment sweeps: the semi-external (streamed) sweep and sweeps over
// reference part ranges.
//
// The reference keeps a graph larger than its memory budget on disk and
// sweeps it through two IO segments: fetch_mem_part (gstore.cpp:3867-3918)
// plans contiguous runs of tiles whose row or column window is active into a
// segment, libaio reads the next segment while algo_mem_part processes the
// current one, and part_meta_t{offset, start, end} (gstore.h:563-568) records
// where each run landed.  Here the records stay in pinned host memory and two
// HBM segment buffers take their place:
//
//   * the planner walks the run table (consecutive tiles of one tile row in a
//     group, file order) and keeps the units the algorithm's skip rule needs:
//     every unit of a run whose row window is active, else (half grid) the
//     units whose column window is active; gaps of at most kGapRecords
//     records are copied rather than split;
//   * entries are packed into segments of segment_bytes; each segment is a
//     handful of cudaMemcpyAsync copies on a side stream (one per contiguous
//     file range), rounded down to a 16-byte boundary so the sweep kernels'
//     128-bit loads stay aligned (entry delta is a multiple of 4 records);
//   * segment k+1 copies while segment k sweeps; an event per buffer orders
//     the copy into a buffer after the sweep that last read it;
//   * sweeps alternate direction, so the segment the previous sweep ended
//     on is already in HBM when the next one starts (the reference's cache
//     of segments already in memory, gstore.cpp:1494-1768).
//
// A file-backed graph (gs_upload_graph_file) keeps its records in the .grid
// file instead, as the reference does: a segment's ranges are read with
// pread into one of two pinned staging buffers (a staging buffer is reused
// once its previous copy to HBM is done) and copied to HBM in one piece.
// The host reads segment k+1 while the GPU sweeps segment k.
#include "gs_internal.cuh"

#include <algorithm>
#include <cerrno>
#include <cstring>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

namespace {

// Records of a gap between two needed ranges that are copied instead of
// starting a new copy (64 KB: about a microsecond of PCIe, less than the
// cost of another copy).
constexpr uint64_t kGapRecords = 16384;

// File records [src, src + n) go to segment-buffer records [dst, dst + n).
struct CopyOp {
    uint64_t src, dst, n;
    bool operator==(const CopyOp& o) const { return src == o.src && dst == o.dst && n == o.n; }
};

struct SegPlan {
    uint64_t list_beg = 0, list_n = 0;
    std::vector<CopyOp> copies;
};

inline uint64_t round4(uint64_t x) { return (x + 3) & ~3ull; }

}  // namespace

struct gs_streamer {
    const uint32_t* h_rec = nullptr;
    bool registered = false;       // cudaHostRegister'ed by the library
    std::vector<int> fds;          // file-backed: the layout's files
    std::vector<gs_grid_piece> pieces;   // file-backed: where each record range lies
    uint32_t* h_stage[2] = {nullptr, nullptr};   // file-backed: pinned staging, one per buffer
    bool staged[2] = {false, false};             // a copy from the staging buffer was queued
    uint64_t seg_records = 0;      // capacity of one segment buffer
    uint32_t* d_buf[2] = {nullptr, nullptr};
    bool used[2] = {false, false};
    std::vector<CopyOp> content[2];
    cudaEvent_t ready[2] = {nullptr, nullptr};   // copies into the buffer done
    cudaEvent_t freed[2] = {nullptr, nullptr};   // last sweep reading the buffer done
    cudaStream_t copy = nullptr;
    int last = 1;                  // buffer of the last segment swept
    uint64_t bytes = 0, copies = 0, segments = 0, reused = 0;
};

// Entry lists of consecutive segment sweeps alternate between two slots, so
// the list of the next sweep uploads while the current one still runs.
struct gs_seglists {
    gs_seg_run* d[2] = {nullptr, nullptr};
    gs_seg_run* h[2] = {nullptr, nullptr};      // pinned
    uint64_t cap = 0;
    cudaEvent_t uploaded[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};    // last sweep reading the slot
    bool upload_pending[2] = {false, false};
    bool done_recorded[2] = {false, false};
    int slot = 0;
};

namespace {

void free_lists(gs_seglists* L) {
    for (int k = 0; k < 2; ++k) {
        gs_dev_free(L->d[k]);
        if (L->h[k]) cudaFreeHost(L->h[k]);
        L->d[k] = nullptr;
        L->h[k] = nullptr;
    }
    L->cap = 0;
}

// Uploads the entries of the next sweep on `stream` into the next slot and
// makes the compute stream wait for them; returns the slot.
gs_status upload_list(gs_graph* g, const std::vector<gs_seg_run>& ent, cudaStream_t stream, int* slot_out) {
    gs_ctx* ctx = g->ctx;
    if (!g->lists) {
        g->lists = new (std::nothrow) gs_seglists();
        if (!g->lists) return GS_ERR_OOM;
        for (int k = 0; k < 2; ++k) {
            GS_CHECK_CUDA(ctx, cudaEventCreateWithFlags(&g->lists->uploaded[k], cudaEventDisableTiming));
            GS_CHECK_CUDA(ctx, cudaEventCreateWithFlags(&g->lists->done[k], cudaEventDisableTiming));
        }
    }
    gs_seglists* L = g->lists;
    if (ent.size() > L->cap) {
        // queued sweeps may still read the old lists
        GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        if (g->stream) GS_CHECK_CUDA(ctx, cudaStreamSynchronize(g->stream->copy));
        free_lists(L);
        const uint64_t cap = std::max<uint64_t>(ent.size(), 1024);
        for (int k = 0; k < 2; ++k) {
            GS_TRY(gs_dev_alloc(ctx, (void**)&L->d[k], cap * sizeof(gs_seg_run)));
            GS_CHECK_CUDA(ctx, cudaHostAlloc((void**)&L->h[k], cap * sizeof(gs_seg_run), cudaHostAllocDefault));
        }
        L->cap = cap;
        L->upload_pending[0] = L->upload_pending[1] = false;
    }
    const int k = L->slot;
    L->slot ^= 1;
    if (L->upload_pending[k]) {      // the host slot is free once its last upload finished
        GS_CHECK_CUDA(ctx, cudaEventSynchronize(L->uploaded[k]));
        L->upload_pending[k] = false;
    }
    std::memcpy(L->h[k], ent.data(), ent.size() * sizeof(gs_seg_run));
    if (L->done_recorded[k]) GS_CHECK_CUDA(ctx, cudaStreamWaitEvent(stream, L->done[k], 0));
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(L->d[k], L->h[k], ent.size() * sizeof(gs_seg_run), cudaMemcpyHostToDevice,
                                       stream));
    GS_CHECK_CUDA(ctx, cudaEventRecord(L->uploaded[k], stream));
    L->upload_pending[k] = true;
    if (stream != ctx->stream) GS_CHECK_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, L->uploaded[k], 0));
    *slot_out = k;
    return GS_OK;
}

// Marks the end of the sweep that reads list slot k.
gs_status list_done(gs_graph* g, int k) {
    GS_CHECK_CUDA(g->ctx, cudaEventRecord(g->lists->done[k], g->ctx->stream));
    g->lists->done_recorded[k] = true;
    return GS_OK;
}

inline uint64_t unit_end_rec(const gs_unit& u) { return u.rec_beg + u.n; }

// Entries (run, unit range) a sweep needs under `need`, in file order.
// Units with no live chunk left (need.dead_units) are left out.
void plan_entries(const gs_graph* g, const gs_need& need, std::vector<gs_seg_run>& out) {
    out.clear();
    const std::vector<gs_unit>& units = g->h_units;
    for (uint32_t r = 0; r < (uint32_t)g->R; ++r) {
        const gs_tile_run& run = g->h_runs[r];
        const uint32_t row = units[run.unit_beg].rc >> 16;
        const bool row_on = !need.act || need.act[row];
        if (row_on && !need.dead_units) {
            out.push_back(gs_seg_run{r, run.unit_beg, run.unit_end, 0, 0});
            continue;
        }
        if (!row_on && !need.by_col) continue;
        bool open = false;
        gs_seg_run cur{r, 0, 0, 0, 0};
        uint64_t cur_hi = 0;
        for (uint32_t u = run.unit_beg; u < run.unit_end; ++u) {
            if (!row_on && !need.act[units[u].rc & 0xFFFFu]) continue;
            if (need.dead_units && need.dead_units[u]) continue;
            if (open && units[u].rec_beg - cur_hi <= kGapRecords) {
                cur.unit_end = u + 1;
            } else {
                if (open) out.push_back(cur);
                cur.unit_beg = u;
                cur.unit_end = u + 1;
                open = true;
            }
            cur_hi = unit_end_rec(units[u]);
        }
        if (open) out.push_back(cur);
    }
}

// Assigns every entry its place in a segment buffer of `cap` records and
// cuts the entry list into segments.
void pack(const gs_graph* g, std::vector<gs_seg_run>& ent, uint64_t cap, std::vector<SegPlan>& segs) {
    segs.clear();
    SegPlan cur;
    uint64_t pos = 0;
    for (uint64_t i = 0; i < ent.size(); ++i) {
        gs_seg_run& e = ent[i];
        const uint64_t lo = g->h_units[e.unit_beg].rec_beg;
        const uint64_t hi = unit_end_rec(g->h_units[e.unit_end - 1]);
        if (!cur.copies.empty()) {
            CopyOp& c = cur.copies.back();
            const uint64_t c_end = c.src + c.n;
            if (lo >= c_end && lo - c_end <= kGapRecords && c.dst + (hi - c.src) <= cap) {
                c.n = hi - c.src;
                e.delta = (int64_t)c.dst - (int64_t)c.src;
                pos = c.dst + round4(c.n);
                continue;
            }
        }
        const uint64_t lo4 = lo & ~3ull;
        if (pos + (hi - lo4) > cap) {
            cur.list_n = i - cur.list_beg;
            segs.push_back(cur);
            cur = SegPlan();
            cur.list_beg = i;
            pos = 0;
        }
        cur.copies.push_back(CopyOp{lo4, pos, hi - lo4});
        e.delta = (int64_t)pos - (int64_t)lo4;
        pos += round4(hi - lo4);
    }
    cur.list_n = ent.size() - cur.list_beg;
    if (cur.list_n) segs.push_back(cur);
}

// Reads `bytes` at file offset `off` into dst (pread may return short counts).
bool pread_full(int fd, void* dst, uint64_t bytes, uint64_t off) {
    char* p = static_cast<char*>(dst);
    while (bytes) {
        const size_t chunk = (size_t)std::min<uint64_t>(bytes, 1ull << 30);
        const ssize_t r = pread(fd, p, chunk, (off_t)off);
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) return false;
        p += r;
        off += (uint64_t)r;
        bytes -= (uint64_t)r;
    }
    return true;
}

// Queues the copies of segment `sp` into a buffer and returns the buffer.
gs_status stage(gs_graph* g, const SegPlan& sp, bool first, int prev, int* out) {
    gs_ctx* ctx = g->ctx;
    gs_streamer* st = g->stream;
    int b = prev ^ 1;
    if (first) {
        for (int x = 0; x < 2; ++x) {
            if (st->used[x] && st->content[x] == sp.copies) {
                st->reused += 1;
                *out = x;
                return GS_OK;
            }
        }
    }
    if (st->used[b]) GS_CHECK_CUDA(ctx, cudaStreamWaitEvent(st->copy, st->freed[b], 0));
    st->content[b].clear();
    if (!st->fds.empty()) {
        // the staging buffer's previous copy to HBM must be done before the
        // files are read into it
        if (st->staged[b]) GS_CHECK_CUDA(ctx, cudaEventSynchronize(st->ready[b]));
        uint64_t extent = 0;
        for (const CopyOp& c : sp.copies) {
            if (!gs_read_pieces(st->fds, st->pieces, st->h_stage[b] + c.dst, c.src, c.n))
                return gs_fail(ctx, GS_ERR_FORMAT, "reading the grid files failed at record " + std::to_string(c.src));
            extent = std::max(extent, c.dst + c.n);
            st->bytes += c.n * 4;
        }
        if (extent) {
            GS_CHECK_CUDA(ctx, cudaMemcpyAsync(st->d_buf[b], st->h_stage[b], extent * 4, cudaMemcpyHostToDevice,
                                               st->copy));
            st->copies += 1;
        }
        st->staged[b] = true;
    } else {
        for (const CopyOp& c : sp.copies) {
            GS_CHECK_CUDA(ctx, cudaMemcpyAsync(st->d_buf[b] + c.dst, st->h_rec + c.src, c.n * 4,
                                               cudaMemcpyHostToDevice, st->copy));
            st->bytes += c.n * 4;
            st->copies += 1;
        }
    }
    st->content[b] = sp.copies;
    GS_CHECK_CUDA(ctx, cudaEventRecord(st->ready[b], st->copy));
    *out = b;
    return GS_OK;
}

// Runs the planned segments through the two buffers.
gs_status run_streamed(gs_graph* g, std::vector<gs_seg_run>& ent, int direction, gs_status (*fn)(void*),
                       void* arg) {
    gs_ctx* ctx = g->ctx;
    gs_streamer* st = g->stream;
    std::vector<SegPlan> segs;
    pack(g, ent, st->seg_records, segs);
    if (segs.empty()) return GS_OK;
    if (direction) std::reverse(segs.begin(), segs.end());
    int slot = 0;
    GS_TRY(upload_list(g, ent, st->copy, &slot));
    const gs_seg_run* list = g->lists->d[slot];
    int b = 0;
    GS_TRY(stage(g, segs[0], true, st->last, &b));
    gs_status status = GS_OK;
    // the sweep of segment k is queued before segment k+1 is staged, so a
    // file-backed segment is read while the previous one sweeps
    for (size_t k = 0; k < segs.size(); ++k) {
        cudaError_t e = cudaStreamWaitEvent(ctx->stream, st->ready[b], 0);
        if (e != cudaSuccess) {
            status = gs_cuda_fail(ctx, e, "cudaStreamWaitEvent(ready)");
            break;
        }
        g->seg.list = list + segs[k].list_beg;
        g->seg.n = (uint32_t)segs[k].list_n;
        g->seg.buf = st->d_buf[b];
        status = fn(arg);
        if (status == GS_OK) {
            e = cudaEventRecord(st->freed[b], ctx->stream);
            if (e != cudaSuccess) status = gs_cuda_fail(ctx, e, "cudaEventRecord(freed)");
        }
        st->used[b] = true;
        st->last = b;
        st->segments += 1;
        if (status != GS_OK) break;
        if (k + 1 < segs.size()) {
            int nb = b;
            status = stage(g, segs[k + 1], false, b, &nb);
            if (status != GS_OK) break;
            b = nb;
        }
    }
    g->seg = SegView();
    gs_status st2 = list_done(g, slot);
    return status != GS_OK ? status : st2;
}

// Part id (group_full_index << 16 | i << 8 | j, get_ij in gstore.h:199-220)
// to its .start index; false when the id names no stored tile.
bool part_to_tile(const gs_graph* g, uint64_t part, uint64_t* t) {
    const uint64_t gfi = part >> 16;
    const uint64_t bi = gfi / g->p, bj = gfi % g->p;
    const uint64_t si = (part >> 8) & 0xFF, sj = part & 0xFF;
    if (bi >= g->p) return false;
    if (!g->directed && bi > bj) return false;
    uint64_t within;
    if (!g->directed && bi == bj) {
        if (si > sj) return false;
        within = gs_calc_index_half(si, sj, kGroupTiles);
    } else {
        within = si * kGroupTiles + sj;
    }
    *t = gs_group_base(bi, bj, g->p, g->directed) + within;
    return *t < g->T_all;
}

}  // namespace

gs_status gs_each_segment_fn(gs_graph* g, const gs_need& need, int direction, gs_status (*fn)(void*),
                             void* arg) {
    if (!g->stream) {
        g->seg = SegView();
        return fn(arg);
    }
    std::vector<gs_seg_run> ent;
    plan_entries(g, need, ent);
    return run_streamed(g, ent, direction, fn, arg);
}

gs_status gs_each_part_fn(gs_graph* g, const gs_segment* segs, int n_segs, gs_status (*fn)(void*), void* arg) {
    gs_ctx* ctx = g->ctx;
    const std::vector<gs_unit>& units = g->h_units;
    std::vector<gs_seg_run> ent;
    for (int k = 0; k < n_segs; ++k) {
        uint64_t t0, t1;
        if (!part_to_tile(g, segs[k].part_start, &t0) || !part_to_tile(g, segs[k].part_end, &t1) || t1 < t0)
            return gs_fail(ctx, GS_ERR_ARG, "segment " + std::to_string(k) + " names no tile range");
        const uint64_t lo = g->h_start[t0], hi = g->h_start[t1 + 1];
        // units whose records lie in [lo, hi) (units follow the file order)
        auto ub = std::lower_bound(units.begin(), units.end(), lo,
                                   [](const gs_unit& u, uint64_t x) { return u.rec_beg < x; });
        uint32_t u = (uint32_t)(ub - units.begin());
        uint32_t u_hi = u;
        while (u_hi < units.size() && units[u_hi].rec_beg < hi) ++u_hi;
        while (u < u_hi) {
            auto rit = std::upper_bound(g->h_runs.begin(), g->h_runs.end(), u,
                                        [](uint32_t x, const gs_tile_run& r) { return x < r.unit_end; });
            const uint32_t r = (uint32_t)(rit - g->h_runs.begin());
            const uint32_t e = std::min<uint32_t>(u_hi, rit->unit_end);
            ent.push_back(gs_seg_run{r, u, e, 0, 0});
            u = e;
        }
    }
    if (ent.empty()) return GS_OK;
    if (g->stream) return run_streamed(g, ent, 0, fn, arg);
    int slot = 0;
    GS_TRY(upload_list(g, ent, ctx->stream, &slot));
    g->seg.list = g->lists->d[slot];
    g->seg.n = (uint32_t)ent.size();
    g->seg.buf = g->d_rec;
    gs_status status = fn(arg);
    g->seg = SegView();
    gs_status st2 = list_done(g, slot);
    return status != GS_OK ? status : st2;
}

namespace {

// The segment buffers, their events and the copy stream of a streamer.
gs_status open_buffers(gs_graph* g, gs_streamer* st) {
    gs_ctx* ctx = g->ctx;
    GS_CHECK_CUDA(ctx, cudaStreamCreateWithFlags(&st->copy, cudaStreamNonBlocking));
    for (int b = 0; b < 2; ++b) {
        GS_TRY(gs_dev_alloc(ctx, (void**)&st->d_buf[b], st->seg_records * 4 + 16));
        GS_CHECK_CUDA(ctx, cudaEventCreateWithFlags(&st->ready[b], cudaEventDisableTiming));
        GS_CHECK_CUDA(ctx, cudaEventCreateWithFlags(&st->freed[b], cudaEventDisableTiming));
    }
    return GS_OK;
}

}  // namespace

bool gs_read_pieces(const std::vector<int>& fds, const std::vector<gs_grid_piece>& pieces, uint32_t* dst,
                    uint64_t rec, uint64_t n) {
    // the first piece holding `rec` (pieces are sorted by rec_beg)
    size_t lo = 0, hi = pieces.size();
    while (lo < hi) {
        const size_t mid = (lo + hi) / 2;
        if (pieces[mid].rec_beg + pieces[mid].n <= rec) lo = mid + 1;
        else hi = mid;
    }
    for (size_t i = lo; n > 0; ++i) {
        if (i >= pieces.size() || pieces[i].rec_beg > rec) return false;
        const gs_grid_piece& p = pieces[i];
        const uint64_t k = std::min<uint64_t>(n, p.rec_beg + p.n - rec);
        if (!pread_full(fds[p.file], dst, k * 4, (p.file_rec + (rec - p.rec_beg)) * 4)) return false;
        dst += k;
        rec += k;
        n -= k;
    }
    return true;
}

gs_status gs_stream_open_layout(gs_graph* g, const gs_tile_layout& L, uint64_t segment_bytes) {
    gs_ctx* ctx = g->ctx;
    const uint64_t min_bytes = 2 * (kRunRecords + 8) * 4;
    if (segment_bytes < min_bytes)
        return gs_fail(ctx, GS_ERR_ARG, "segment_bytes must be at least " + std::to_string(min_bytes));
    gs_streamer* st = new (std::nothrow) gs_streamer();
    if (!st) return GS_ERR_OOM;
    g->stream = st;
    st->seg_records = (segment_bytes / 4) & ~3ull;
    st->pieces = L.pieces;
    for (const std::string& path : L.files) {
        const int fd = open(path.c_str(), O_RDONLY);
        if (fd < 0) return gs_fail(ctx, GS_ERR_ARG, "cannot open " + path);
        st->fds.push_back(fd);
    }
    for (const gs_grid_piece& p : L.pieces) {
        struct stat sb;
        if (fstat(st->fds[p.file], &sb) != 0 || (uint64_t)sb.st_size < (p.file_rec + p.n) * 4)
            return gs_fail(ctx, GS_ERR_FORMAT, L.files[p.file] + " holds fewer than the records .start counts");
    }
    for (int b = 0; b < 2; ++b)
        GS_CHECK_CUDA(ctx, cudaHostAlloc((void**)&st->h_stage[b], st->seg_records * 4 + 16, cudaHostAllocDefault));
    return open_buffers(g, st);
}

gs_status gs_stream_open_file(gs_graph* g, const char* path, uint64_t segment_bytes) {
    gs_tile_layout L;
    L.files.push_back(path);
    if (g->E) L.pieces.push_back(gs_grid_piece{0, g->E, 0, 0, 0});
    return gs_stream_open_layout(g, L, segment_bytes);
}

bool gs_stream_read_records(const gs_graph* g, uint32_t* dst) {
    const gs_streamer* st = g->stream;
    if (!st) return false;
    if (!st->fds.empty()) return g->E == 0 || gs_read_pieces(st->fds, st->pieces, dst, 0, g->E);
    std::memcpy(dst, st->h_rec, g->E * 4);
    return true;
}

gs_status gs_stream_open(gs_graph* g, const uint32_t* host_grid, uint64_t segment_bytes) {
    gs_ctx* ctx = g->ctx;
    const uint64_t min_bytes = 2 * (kRunRecords + 8) * 4;
    if (segment_bytes < min_bytes)
        return gs_fail(ctx, GS_ERR_ARG, "segment_bytes must be at least " + std::to_string(min_bytes));
    gs_streamer* st = new (std::nothrow) gs_streamer();
    if (!st) return GS_ERR_OOM;
    g->stream = st;
    st->h_rec = host_grid;
    st->seg_records = (segment_bytes / 4) & ~3ull;
    if (g->E) {
        // DMA straight from the caller's array: pin it unless it already is
        cudaPointerAttributes attr;
        cudaError_t e = cudaPointerGetAttributes(&attr, host_grid);
        if (e != cudaSuccess || attr.type != cudaMemoryTypeHost) {
            cudaGetLastError();
            e = cudaHostRegister((void*)host_grid, g->E * 4, cudaHostRegisterDefault);
            if (e == cudaErrorHostMemoryAlreadyRegistered) {
                cudaGetLastError();       // pinned by its owner
            } else if (e != cudaSuccess) {
                return gs_cuda_fail(ctx, e, "cudaHostRegister(grid)");
            } else {
                st->registered = true;
            }
        }
    }
    return open_buffers(g, st);
}

void gs_stream_close(gs_graph* g) {
    gs_streamer* st = g->stream;
    if (st || g->lists) cudaStreamSynchronize(g->ctx->stream);   // sweeps reading buffers or lists
    if (st) {
        if (st->copy) cudaStreamSynchronize(st->copy);
        for (int b = 0; b < 2; ++b) {
            gs_dev_free(st->d_buf[b]);
            if (st->ready[b]) cudaEventDestroy(st->ready[b]);
            if (st->freed[b]) cudaEventDestroy(st->freed[b]);
        }
        if (st->copy) cudaStreamDestroy(st->copy);
        if (st->registered) cudaHostUnregister((void*)st->h_rec);
        for (int b = 0; b < 2; ++b)
            if (st->h_stage[b]) cudaFreeHost(st->h_stage[b]);
        for (int fd : st->fds) close(fd);
        delete st;
        g->stream = nullptr;
    }
    if (g->lists) {
        gs_seglists* L = g->lists;
        free_lists(L);
        for (int k = 0; k < 2; ++k) {
            if (L->uploaded[k]) cudaEventDestroy(L->uploaded[k]);
            if (L->done[k]) cudaEventDestroy(L->done[k]);
        }
        delete L;
        g->lists = nullptr;
    }
}

extern "C" gs_status gs_stream_stats(const gs_graph* g, uint64_t* bytes_copied, uint64_t* copies,
                                     uint64_t* segments, uint64_t* segments_reused) {
    if (!g) return GS_ERR_ARG;
    const gs_streamer* st = g->stream;
    if (bytes_copied) *bytes_copied = st ? st->bytes : 0;
    if (copies) *copies = st ? st->copies : 0;
    if (segments) *segments = st ? st->segments : 0;
    if (segments_reused) *segments_reused = st ? st->reused : 0;
    return GS_OK;
}

const uint32_t* gs_stream_records(const gs_graph* g) { return g->stream ? g->stream->h_rec : nullptr; }
