// C-ABI entry points of libgstore_cuda.so: contexts, resident graphs and the
// algo_t-style state machine (init / sweep / finalize / download).
#include "gs_internal.cuh"

#include <sys/stat.h>

#include <algorithm>
#include <cstring>
#include <new>

// ------------------------------------------------------------------ errors --
gs_status gs_fail(gs_ctx* ctx, gs_status code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

gs_status gs_cuda_fail(gs_ctx* ctx, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return gs_fail(ctx, GS_ERR_OOM, m);
    }
    return gs_fail(ctx, GS_ERR_CUDA, m);
}

gs_status gs_dev_alloc(gs_ctx* ctx, void** ptr, size_t bytes) {
    *ptr = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e == cudaErrorMemoryAllocation && ctx && !ctx->pool_free.empty()) {
        // the pool's idle blocks hold the memory: release them, try once more
        cudaGetLastError();
        gs_pool_clear(ctx);
        e = cudaMalloc(ptr, bytes);
    }
    if (e != cudaSuccess) {
        *ptr = nullptr;
        return gs_cuda_fail(ctx, e, "cudaMalloc");
    }
    return GS_OK;
}

void gs_dev_free(void* ptr) {
    if (ptr) cudaFree(ptr);
}

constexpr uint64_t kPoolMaxBytes = 16ull << 30;

gs_status gs_pool_get(gs_ctx* ctx, size_t bytes, void** out) {
    bytes = (bytes + 255) & ~(size_t)255;
    auto it = ctx->pool_free.find(bytes);
    if (it != ctx->pool_free.end()) {
        *out = it->second;
        ctx->pool_free.erase(it);
        ctx->pool_bytes -= bytes;
        return GS_OK;
    }
    return gs_dev_alloc(ctx, out, bytes);
}

void gs_pool_put(gs_ctx* ctx, void* ptr, size_t bytes) {
    if (!ptr) return;
    bytes = (bytes + 255) & ~(size_t)255;
    if (ctx->pool_bytes + bytes > kPoolMaxBytes) {
        gs_dev_free(ptr);
        return;
    }
    ctx->pool_free.emplace(bytes, ptr);
    ctx->pool_bytes += bytes;
}

gs_status gs_state_alloc(gs_state* s, void** ptr, size_t bytes) {
    GS_TRY(gs_pool_get(s->g->ctx, bytes, ptr));
    s->allocs.emplace_back(*ptr, bytes);
    return GS_OK;
}

void gs_pool_clear(gs_ctx* ctx) {
    for (auto& kv : ctx->pool_free) gs_dev_free(kv.second);
    ctx->pool_free.clear();
    ctx->pool_bytes = 0;
}

gs_status gs_alloc_records(gs_ctx* ctx, uint32_t** ptr, uint64_t n_records) {
    GS_TRY(gs_dev_alloc(ctx, (void**)ptr, (n_records + kRecPad) * 4));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(*ptr + n_records, 0, kRecPad * 4, ctx->stream));
    return GS_OK;
}

gs_status gs_graph_alloc(gs_graph* g, void** ptr, size_t bytes) {
    GS_TRY(gs_pool_get(g->ctx, bytes, ptr));
    g->pooled.emplace_back(*ptr, bytes);
    return GS_OK;
}

gs_status gs_graph_alloc_records(gs_graph* g, uint32_t** ptr, uint64_t n_records) {
    GS_TRY(gs_graph_alloc(g, (void**)ptr, (n_records + kRecPad) * 4));
    GS_CHECK_CUDA(g->ctx, cudaMemsetAsync(*ptr + n_records, 0, kRecPad * 4, g->ctx->stream));
    return GS_OK;
}

void gs_graph_release(gs_graph* g, void* ptr) {
    if (!ptr) return;
    for (auto it = g->pooled.begin(); it != g->pooled.end(); ++it) {
        if (it->first == ptr) {
            gs_pool_put(g->ctx, ptr, it->second);
            g->pooled.erase(it);
            return;
        }
    }
    gs_dev_free(ptr);
}

void gs_geometry_of(uint64_t V, int directed, uint32_t* p, uint32_t* p_s, uint64_t* n_tiles) {
    // grid::init "-v" (gstore.cpp:152-161): p = ceil(V / 2^24), p_s = 256 p.
    uint64_t pp = (V >> kGroupBits) + ((V & ((1ull << kGroupBits) - 1)) != 0);
    if (pp == 0) pp = 1;
    uint64_t ps = pp * kGroupTiles;
    if (p) *p = (uint32_t)pp;
    if (p_s) *p_s = (uint32_t)ps;
    if (n_tiles) *n_tiles = directed ? ps * ps : ps * (ps + 1) / 2;  // calc_total_part
}

void gs_timer_begin(gs_ctx* ctx) {
    if (ctx->profile) cudaEventRecord(ctx->ev0, ctx->stream);
}

void gs_timer_end(gs_ctx* ctx, int algo, uint64_t bytes) {
    if (!ctx->profile) return;
    cudaEventRecord(ctx->ev1, ctx->stream);
    cudaEventSynchronize(ctx->ev1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    KernelTimes& k = ctx->ktime[algo & 7];
    k.launches += 1;
    k.ms += ms;
    k.bytes += bytes;
}

extern "C" {

const char* gs_last_error(const gs_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

gs_status gs_geometry(uint64_t V, int directed, uint32_t* p, uint32_t* p_s,
                      uint64_t* n_start_entries) {
    uint64_t T;
    gs_geometry_of(V, directed, p, p_s, &T);
    if (n_start_entries) *n_start_entries = T + 1;
    return GS_OK;
}

gs_status gs_create(gs_ctx** out, int device, uint64_t hbm_budget_bytes, int directed) {
    if (!out) return GS_ERR_ARG;
    *out = nullptr;
    gs_ctx* ctx = new (std::nothrow) gs_ctx();
    if (!ctx) return GS_ERR_OOM;
    ctx->device = device;
    ctx->budget = hbm_budget_bytes;
    ctx->directed = directed ? 1 : 0;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev1);
    if (e == cudaSuccess) e = cudaMalloc((void**)&ctx->d_scalars, 64 * sizeof(uint64_t));
    if (e == cudaSuccess) e = cudaMalloc((void**)&ctx->d_ticket, 8 * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemset(ctx->d_ticket, 0, 8 * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&ctx->h_scalars, 64 * sizeof(uint64_t));
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) {
        gs_status st = (e == cudaErrorMemoryAllocation) ? GS_ERR_OOM : GS_ERR_CUDA;
        gs_destroy(ctx);
        return st;
    }
    ctx->own_stream = true;
    *out = ctx;
    return GS_OK;
}

gs_status gs_destroy(gs_ctx* ctx) {
    if (!ctx) return GS_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    gs_pool_clear(ctx);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->d_scalars) cudaFree(ctx->d_scalars);
    if (ctx->d_ticket) cudaFree(ctx->d_ticket);
    if (ctx->h_scalars) cudaFreeHost(ctx->h_scalars);
    delete ctx;
    return GS_OK;
}

gs_status gs_set_stream(gs_ctx* ctx, void* cuda_stream) {
    if (!ctx) return GS_ERR_ARG;
    GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    if (cuda_stream) {
        ctx->stream = (cudaStream_t)cuda_stream;
        ctx->own_stream = false;
    } else {
        GS_CHECK_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        ctx->own_stream = true;
    }
    return GS_OK;
}

gs_status gs_profile(gs_ctx* ctx, int enable) {
    if (!ctx) return GS_ERR_ARG;
    ctx->profile = enable != 0;
    for (auto& k : ctx->ktime) k = KernelTimes();
    return GS_OK;
}

gs_status gs_launch_count(const gs_ctx* ctx, uint64_t* launches) {
    if (!ctx || !launches) return GS_ERR_ARG;
    *launches = ctx->launches;
    return GS_OK;
}

gs_status gs_kernel_time(gs_ctx* ctx, int algo, uint64_t* launches, double* total_ms,
                         uint64_t* bytes) {
    if (!ctx || algo < 0 || algo > 3) return GS_ERR_ARG;
    if (launches) *launches = ctx->ktime[algo].launches;
    if (total_ms) *total_ms = ctx->ktime[algo].ms;
    if (bytes) *bytes = ctx->ktime[algo].bytes;
    return GS_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ graph --
static void free_graph_arrays(gs_graph* g) {
    // pooled buffers are reused by the next request in stream order only:
    // no copy or kernel may still touch them when they go back to the pool
    cudaStreamSynchronize(g->ctx->stream);
    gs_stream_close(g);
    pr_layout_free(g);
    pb_layout_free(g);
    for (void* p : {(void*)g->d_rec, (void*)g->d_items, (void*)g->d_tile_off, (void*)g->d_tile_rc,
                    (void*)g->d_degree, (void*)g->d_runs, (void*)g->d_runs_lpt, (void*)g->d_units,
                    (void*)g->d_runs_blk, (void*)g->d_units_blk, (void*)g->d_runs_blk2, (void*)g->d_units_blk2})
        gs_graph_release(g, p);
    for (auto& pb : g->pooled) gs_pool_put(g->ctx, pb.first, pb.second);   // none expected
    g->pooled.clear();
    g->d_runs_blk2 = nullptr;
    g->d_units_blk2 = nullptr;
    g->d_runs = nullptr;
    g->d_runs_lpt = nullptr;
    g->d_units = nullptr;
    g->d_runs_blk = nullptr;
    g->d_units_blk = nullptr;
    g->d_rec = nullptr;
    g->d_items = nullptr;
    g->d_tile_off = nullptr;
    g->d_tile_rc = nullptr;
    g->d_degree = nullptr;
}

// An L2-blocked sweep order: tiles grouped into blocks of `block` x `block`
// windows (row-major inside a block), so the vertex state the tiles in
// flight touch (2 `block` windows) stays in L2.  Runs are short (one tile
// row, <= kBlockRunUnits units, one per warp of a CTA) so the CTAs in flight
// work inside one or two blocks.  Used by the sweeps whose per-record state
// is large (WCC, k-core, batches, serving: kBlockWindows; multi-source BFS
// with 16-byte vertex state may pick kBlockWindowsSmall); their results do
// not depend on the order.
static gs_status build_blocked_order(gs_graph* g, uint32_t block, uint64_t* R_out, gs_tile_run** d_runs_out,
                                     gs_unit** d_units_out) {
    gs_ctx* ctx = g->ctx;
    const uint64_t T = g->T;
    std::vector<uint32_t> tile_unit(T + 1, 0);
    {
        uint64_t k = 0;
        for (uint32_t u = 0; u < g->U; ++u) {
            while (g->h_tile_off[k + 1] <= g->h_units[u].rec_beg) tile_unit[++k] = u;
        }
        while (k < T) tile_unit[++k] = (uint32_t)g->U;
    }
    std::vector<uint32_t> order(T);
    for (uint32_t k = 0; k < T; ++k) order[k] = k;
    auto block_of = [&](uint32_t k) {
        const uint32_t rc = g->h_tile_rc[k];
        return ((uint64_t)((rc >> 16) / block) << 32) | ((rc & 0xFFFFu) / block);
    };
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return block_of(a) < block_of(b); });
    std::vector<gs_unit> units;
    std::vector<gs_tile_run> runs;
    units.reserve(g->U);
    uint64_t open_block = ~0ull;
    uint32_t open_row = ~0u;
    bool is_open = false;
    for (uint32_t k : order) {
        const uint32_t row = g->h_tile_rc[k] >> 16;
        const uint64_t blk = block_of(k);
        for (uint32_t u = tile_unit[k]; u < tile_unit[k + 1]; ++u) {
            const gs_unit& d = g->h_units[u];
            if (!is_open || row != open_row || blk != open_block || runs.back().unit_end - runs.back().unit_beg >= kBlockRunUnits) {
                runs.push_back(gs_tile_run{d.rec_beg, d.rec_beg, 0, 0, (uint32_t)units.size(), (uint32_t)units.size()});
                open_row = row;
                open_block = blk;
                is_open = true;
            }
            units.push_back(d);
            runs.back().rec_end = d.rec_beg + d.n;
            runs.back().unit_end = (uint32_t)units.size();
        }
    }
    *R_out = runs.size();
    GS_TRY(gs_graph_alloc(g, (void**)d_units_out, std::max<size_t>(1, units.size()) * sizeof(gs_unit)));
    GS_TRY(gs_graph_alloc(g, (void**)d_runs_out, std::max<size_t>(1, runs.size()) * sizeof(gs_tile_run)));
    if (!units.empty())
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(*d_units_out, units.data(), units.size() * sizeof(gs_unit),
                                           cudaMemcpyHostToDevice, ctx->stream));
    if (!runs.empty())
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(*d_runs_out, runs.data(), runs.size() * sizeof(gs_tile_run),
                                           cudaMemcpyHostToDevice, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return GS_OK;
}

// The L2-blocked orders of a resident graph, built at their first use (the
// BFS sweep and a plain upload do not need them).
gs_status gs_ensure_blocked(gs_graph* g) {
    if (g->stream || g->blocked_built) return GS_OK;
    GS_TRY(build_blocked_order(g, kBlockWindows, &g->R_blk, &g->d_runs_blk, &g->d_units_blk));
    GS_TRY(build_blocked_order(g, kBlockWindowsSmall, &g->R_blk2, &g->d_runs_blk2, &g->d_units_blk2));
    g->blocked_built = true;
    return GS_OK;
}

// Builds the non-empty tile table and the work items from the host .start
// array, walking the stored tiles in file order (the loops of grid::*_mmap,
// gstore.cpp:2520-2559), and uploads them.
static gs_status build_tables(gs_graph* g) {
    gs_ctx* ctx = g->ctx;
    const std::vector<uint64_t>& st = g->h_start;
    std::vector<uint64_t>& tile_off = g->h_tile_off;
    std::vector<uint32_t>& tile_rc = g->h_tile_rc;
    std::vector<gs_tile_run>& runs = g->h_runs;
    std::vector<gs_unit>& units = g->h_units;
    uint64_t n_items = 0;
    runs.clear();
    units.clear();
    tile_off.clear();
    tile_rc.clear();
    tile_off.reserve(1024);
    uint64_t t = 0;
    const uint64_t p = g->p;
    gs_tile_run open{0, 0, 0, 0, 0, 0};
    bool is_open = false;
    auto close_run = [&]() {
        if (is_open) runs.push_back(open);
        is_open = false;
    };
    for (uint64_t gi = 0; gi < p; ++gi) {
        for (uint64_t gj = g->directed ? 0 : gi; gj < p; ++gj) {
            for (uint64_t m = 0; m < kGroupTiles; ++m) {
                uint64_t n0 = (!g->directed && gi == gj) ? m : 0;
                close_run();  // a run never leaves the row segment of its group
                for (uint64_t n = n0; n < kGroupTiles; ++n, ++t) {
                    uint64_t b = st[t], e = st[t + 1];
                    if (e == b) continue;
                    uint32_t row = (uint32_t)(gi * kGroupTiles + m);
                    uint32_t col = (uint32_t)(gj * kGroupTiles + n);
                    if (row >= g->nw || col >= g->nw)
                        return gs_fail(ctx, GS_ERR_FORMAT,
                                       "tile (" + std::to_string(row) + "," + std::to_string(col) +
                                           ") holds records beyond the vertex count");
                    uint32_t rc = (row << 16) | col;
                    const uint32_t k = (uint32_t)tile_rc.size();
                    const uint32_t u0 = (uint32_t)units.size();
                    for (uint64_t x = b; x < e; x += kUnitRecords)
                        units.push_back(gs_unit{x, (uint32_t)std::min<uint64_t>(kUnitRecords, e - x), rc});
                    const uint32_t u1 = (uint32_t)units.size();
                    // kRunRecords is a multiple of kUnitRecords: units never straddle runs
                    if (e - b > kRunRecords) {
                        close_run();
                        for (uint64_t x = b; x < e; x += kRunRecords) {
                            const uint64_t xe = std::min<uint64_t>(e, x + kRunRecords);
                            runs.push_back(gs_tile_run{x, xe, k, k + 1, u0 + (uint32_t)((x - b) / kUnitRecords),
                                                       u0 + (uint32_t)((xe - b + kUnitRecords - 1) / kUnitRecords)});
                        }
                    } else if (is_open && e - open.rec_beg <= kRunRecords) {
                        open.rec_end = e;
                        open.tile_end = k + 1;
                        open.unit_end = u1;
                    } else {
                        close_run();
                        open = gs_tile_run{b, e, k, k + 1, u0, u1};
                        is_open = true;
                    }
                    tile_off.push_back(b);
                    tile_rc.push_back(rc);
                    n_items += (e - b + kItemRecords - 1) / kItemRecords;
                }
            }
        }
    }
    close_run();
    tile_off.push_back(st[t]);
    g->T = tile_rc.size();
    g->I = n_items;
    g->R = runs.size();
    g->U = units.size();
    GS_TRY(gs_graph_alloc(g, (void**)&g->d_units, std::max<size_t>(1, units.size()) * sizeof(gs_unit)));
    if (!units.empty())
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(g->d_units, units.data(), units.size() * sizeof(gs_unit),
                                           cudaMemcpyHostToDevice, ctx->stream));
    GS_TRY(gs_graph_alloc(g, (void**)&g->d_runs, std::max<size_t>(1, runs.size()) * sizeof(gs_tile_run)));
    if (!runs.empty())
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(g->d_runs, runs.data(), runs.size() * sizeof(gs_tile_run),
                                           cudaMemcpyHostToDevice, ctx->stream));
    // The BFS sweep's runs, longest first, so that the runs drawn last from
    // the sweep's ticket are the short ones.  A graph with fewer than
    // kBfsRunsPerCta runs per CTA of the sweep has its runs cut into pieces
    // of 32, 16 or 8 units (the largest cut that gives that many pieces):
    // pieces spread a small grid over the machine, while on a large grid
    // whole runs pay their per-run set-up (row state, flush) over more
    // records.
    std::vector<gs_tile_run> lpt;
    if (!g->stream && !runs.empty()) {
        const uint64_t want = kBfsRunsPerCta * gs_grid_size(ctx, kBfsCtasPerSm);
        uint32_t cut = 0;   // whole runs
        if (runs.size() < want)
            for (cut = 32; cut > kBfsMinRunUnits; cut /= 2) {
                uint64_t pieces = 0;
                for (const gs_tile_run& r : runs) pieces += (r.unit_end - r.unit_beg + cut - 1) / cut;
                if (pieces >= want) break;
            }
        if (cut == 0) cut = UINT32_MAX;
        for (const gs_tile_run& r : runs)
            for (uint32_t u = r.unit_beg; u < r.unit_end;) {
                const uint32_t ue = (uint32_t)std::min<uint64_t>(r.unit_end, (uint64_t)u + cut);
                lpt.push_back(gs_tile_run{units[u].rec_beg, units[ue - 1].rec_beg + units[ue - 1].n, r.tile_beg,
                                          r.tile_end, u, ue});
                u = ue;
            }
        std::stable_sort(lpt.begin(), lpt.end(), [](const gs_tile_run& x, const gs_tile_run& y) {
            return x.rec_end - x.rec_beg > y.rec_end - y.rec_beg;
        });
        g->R_lpt = lpt.size();
        GS_TRY(gs_graph_alloc(g, (void**)&g->d_runs_lpt, lpt.size() * sizeof(gs_tile_run)));
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(g->d_runs_lpt, lpt.data(), lpt.size() * sizeof(gs_tile_run),
                                           cudaMemcpyHostToDevice, ctx->stream));
    }
    GS_TRY(gs_graph_alloc(g, (void**)&g->d_tile_off, tile_off.size() * sizeof(uint64_t)));
    GS_TRY(gs_graph_alloc(g, (void**)&g->d_tile_rc, std::max<size_t>(1, tile_rc.size()) * sizeof(uint32_t)));
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(g->d_tile_off, tile_off.data(), tile_off.size() * sizeof(uint64_t),
                                       cudaMemcpyHostToDevice, ctx->stream));
    if (!tile_rc.empty())
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(g->d_tile_rc, tile_rc.data(), tile_rc.size() * sizeof(uint32_t),
                                           cudaMemcpyHostToDevice, ctx->stream));
    // The host vectors die at return: wait for the copies.
    GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return GS_OK;
}

static gs_status check_start(gs_graph* g, uint64_t n_start, uint64_t n_edges) {
    gs_ctx* ctx = g->ctx;
    if (n_start != g->T_all + 1)
        return gs_fail(ctx, GS_ERR_FORMAT,
                       "start has " + std::to_string(n_start) + " entries, geometry needs " +
                           std::to_string(g->T_all + 1));
    const std::vector<uint64_t>& st = g->h_start;
    if (st[0] != 0) return gs_fail(ctx, GS_ERR_FORMAT, "start[0] != 0");
    for (uint64_t t = 0; t < g->T_all; ++t)
        if (st[t + 1] < st[t])
            return gs_fail(ctx, GS_ERR_FORMAT, "start decreases at tile " + std::to_string(t));
    if (st[g->T_all] != n_edges)
        return gs_fail(ctx, GS_ERR_FORMAT,
                       "start[last] = " + std::to_string(st[g->T_all]) + " but grid holds " +
                           std::to_string(n_edges) + " records");
    return GS_OK;
}

static gs_status finish_upload(gs_graph* g, const int32_t* degree, bool degree_on_device) {
    gs_ctx* ctx = g->ctx;
    GS_TRY(gs_graph_alloc(g, (void**)&g->d_degree, g->N * sizeof(int32_t)));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(g->d_degree, 0, g->N * sizeof(int32_t), ctx->stream));
    if (degree) {
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(g->d_degree, degree, g->V * sizeof(int32_t),
                                           degree_on_device ? cudaMemcpyDeviceToDevice
                                                            : cudaMemcpyHostToDevice,
                                           ctx->stream));
    }
    GS_TRY(build_tables(g));
    if ((g->V & 0xFFFF) != 0 && g->E > 0) {
        int* d_flag = (int*)ctx->d_scalars;
        GS_CHECK_CUDA(ctx, cudaMemsetAsync(d_flag, 0, sizeof(int), ctx->stream));
        GS_TRY(launch_validate_records(g, d_flag));
        int h_flag = 0;
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(&h_flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        if (h_flag) return gs_fail(ctx, GS_ERR_FORMAT, "a record addresses a vertex >= V");
    }
    if (!degree) {
        GS_TRY(launch_degree_from_records(g));
        g->degree_from_records = true;
    }
    GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return GS_OK;
}

static gs_status new_graph(gs_ctx* ctx, uint64_t V, gs_graph** out) {
    if (!ctx || !out || V == 0 || V > (1ull << 32)) return gs_fail(ctx, GS_ERR_ARG, "bad vertex count");
    GS_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    gs_graph* g = new (std::nothrow) gs_graph();
    if (!g) return GS_ERR_OOM;
    g->ctx = ctx;
    g->directed = ctx->directed;
    g->V = V;
    gs_geometry_of(V, g->directed, &g->p, &g->p_s, &g->T_all);
    g->nw = (uint32_t)((V + 0xFFFF) >> kTileBits);
    g->N = (uint64_t)g->nw << kTileBits;
    *out = g;
    return GS_OK;
}

// Builds a resident graph around records already in device memory
// (d_rec is adopted; d_start and d_degree are copied and stay the caller's).
gs_status gs_graph_adopt(gs_ctx* ctx, uint64_t V, const uint64_t* d_start, uint64_t n_start, uint32_t* d_rec,
                         uint64_t n_edges, const int32_t* d_degree, gs_graph** out) {
    *out = nullptr;
    gs_graph* g = nullptr;
    gs_status st = new_graph(ctx, V, &g);
    if (st != GS_OK) {
        gs_dev_free(d_rec);
        return st;
    }
    g->d_rec = d_rec;
    g->E = n_edges;
    g->h_start.resize(n_start);
    cudaError_t e = cudaMemcpyAsync(g->h_start.data(), d_start, n_start * 8, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) st = gs_cuda_fail(ctx, e, "copy start");
    if (st == GS_OK) st = check_start(g, n_start, n_edges);
    if (st == GS_OK) st = finish_upload(g, d_degree, true);
    if (st != GS_OK) {
        free_graph_arrays(g);
        delete g;
        return st;
    }
    *out = g;
    return GS_OK;
}

extern "C" {

gs_status gs_upload_graph(gs_ctx* ctx, const uint64_t* start, uint64_t n_start,
                          const uint32_t* grid, uint64_t n_edges, const int32_t* degree,
                          uint64_t V, gs_graph** out) {
    if (!ctx || !start || !out || (n_edges && !grid)) return gs_fail(ctx, GS_ERR_ARG, "null argument");
    *out = nullptr;
    gs_graph* g = nullptr;
    GS_TRY(new_graph(ctx, V, &g));
    g->h_start.assign(start, start + std::min<uint64_t>(n_start, g->T_all + 1));
    gs_status st = check_start(g, n_start, n_edges);
    if (st == GS_OK && ctx->budget && n_edges * 4 > ctx->budget) {
        // over the tile budget: stream the grid through two segments of half
        // the budget each (the reference's -m semi-external mode)
        g->E = n_edges;
        st = gs_stream_open(g, grid, (ctx->budget / 2) & ~15ull);
        if (st == GS_OK) st = finish_upload(g, degree, false);
        if (st != GS_OK) {
            free_graph_arrays(g);
            delete g;
            return st;
        }
        *out = g;
        return GS_OK;
    }
    if (st == GS_OK) {
        g->E = n_edges;
        st = gs_graph_alloc_records(g, &g->d_rec, n_edges);
        if (st == GS_OK && n_edges) {
            cudaError_t e = cudaMemcpyAsync(g->d_rec, grid, n_edges * 4, cudaMemcpyHostToDevice, ctx->stream);
            if (e != cudaSuccess) st = gs_cuda_fail(ctx, e, "cudaMemcpyAsync(grid)");
        }
    }
    if (st == GS_OK) st = finish_upload(g, degree, false);
    bool sorted_now = false;
    if (st == GS_OK) st = gs_order_tiles(g, &sorted_now);
    if (st != GS_OK) {
        free_graph_arrays(g);
        delete g;
        return st;
    }
    *out = g;
    return GS_OK;
}

gs_status gs_upload_graph_streamed(gs_ctx* ctx, const uint64_t* start, uint64_t n_start,
                                   const uint32_t* grid, uint64_t n_edges, const int32_t* degree,
                                   uint64_t V, uint64_t segment_bytes, gs_graph** out) {
    if (!ctx || !start || !out || (n_edges && !grid)) return gs_fail(ctx, GS_ERR_ARG, "null argument");
    *out = nullptr;
    gs_graph* g = nullptr;
    GS_TRY(new_graph(ctx, V, &g));
    g->h_start.assign(start, start + std::min<uint64_t>(n_start, g->T_all + 1));
    gs_status st = check_start(g, n_start, n_edges);
    g->E = n_edges;
    if (st == GS_OK) st = gs_stream_open(g, grid, segment_bytes);
    if (st == GS_OK) st = finish_upload(g, degree, false);
    if (st != GS_OK) {
        free_graph_arrays(g);
        delete g;
        return st;
    }
    *out = g;
    return GS_OK;
}

gs_status gs_upload_graph_file(gs_ctx* ctx, const uint64_t* start, uint64_t n_start, const char* grid_path,
                               uint64_t n_edges, const int32_t* degree, uint64_t V, uint64_t segment_bytes,
                               gs_graph** out) {
    if (!ctx || !start || !grid_path || !out) return gs_fail(ctx, GS_ERR_ARG, "null argument");
    *out = nullptr;
    gs_graph* g = nullptr;
    GS_TRY(new_graph(ctx, V, &g));
    g->h_start.assign(start, start + std::min<uint64_t>(n_start, g->T_all + 1));
    gs_status st = check_start(g, n_start, n_edges);
    g->E = n_edges;
    if (st == GS_OK) st = gs_stream_open_file(g, grid_path, segment_bytes);
    if (st == GS_OK) st = finish_upload(g, degree, false);
    if (st != GS_OK) {
        free_graph_arrays(g);
        delete g;
        return st;
    }
    *out = g;
    return GS_OK;
}

gs_status gs_upload_graph_files(gs_ctx* ctx, const char* prefix, uint64_t V, uint64_t segment_bytes,
                                gs_graph** out) {
    if (!ctx || !prefix || !out) return gs_fail(ctx, GS_ERR_ARG, "null argument");
    *out = nullptr;
    gs_tile_layout L;
    GS_TRY(gs_read_layout(ctx, prefix, V, ctx->directed, &L));
    // .degree when present (the converters write it), else counted on the device
    std::vector<int32_t> degree;
    struct stat sb;
    if (stat((std::string(prefix) + ".degree").c_str(), &sb) == 0) {
        degree.resize(V);
        GS_TRY(gs_read_degree(ctx, prefix, V, degree.data()));
    }
    gs_graph* g = nullptr;
    GS_TRY(new_graph(ctx, V, &g));
    g->h_start = L.start;
    gs_status st = check_start(g, L.start.size(), L.start.back());
    g->E = L.start.back();
    if (st == GS_OK) st = gs_stream_open_layout(g, L, segment_bytes);
    if (st == GS_OK) st = finish_upload(g, degree.empty() ? nullptr : degree.data(), false);
    if (st != GS_OK) {
        free_graph_arrays(g);
        delete g;
        return st;
    }
    *out = g;
    return GS_OK;
}

gs_status gs_upload_graph_device(gs_ctx* ctx, const uint64_t* d_start, uint64_t n_start,
                                 const uint32_t* d_grid, uint64_t n_edges,
                                 const int32_t* d_degree, uint64_t V, gs_graph** out) {
    if (!ctx || !d_start || !out || (n_edges && !d_grid)) return gs_fail(ctx, GS_ERR_ARG, "null argument");
    *out = nullptr;
    gs_graph* g = nullptr;
    GS_TRY(new_graph(ctx, V, &g));
    gs_status st = GS_OK;
    if (n_start != g->T_all + 1) st = check_start(g, n_start, n_edges);
    if (st == GS_OK) {
        g->h_start.resize(n_start);
        cudaError_t e = cudaMemcpyAsync(g->h_start.data(), d_start, n_start * 8, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) st = gs_cuda_fail(ctx, e, "copy start");
    }
    if (st == GS_OK) st = check_start(g, n_start, n_edges);
    if (st == GS_OK) {
        g->E = n_edges;
        st = gs_graph_alloc_records(g, &g->d_rec, n_edges);
        if (st == GS_OK && n_edges) {
            cudaError_t e = cudaMemcpyAsync(g->d_rec, d_grid, n_edges * 4, cudaMemcpyDeviceToDevice, ctx->stream);
            if (e != cudaSuccess) st = gs_cuda_fail(ctx, e, "cudaMemcpyAsync(grid)");
        }
    }
    if (st == GS_OK) st = finish_upload(g, d_degree, true);
    bool sorted_now = false;
    if (st == GS_OK) st = gs_order_tiles(g, &sorted_now);
    if (st != GS_OK) {
        free_graph_arrays(g);
        delete g;
        return st;
    }
    *out = g;
    return GS_OK;
}

gs_status gs_graph_free(gs_graph* g) {
    if (!g) return GS_OK;
    cudaStreamSynchronize(g->ctx->stream);
    free_graph_arrays(g);
    delete g;
    return GS_OK;
}

gs_status gs_graph_info(const gs_graph* g, uint64_t* n_edges, uint64_t* n_tiles, uint64_t* n_items,
                        uint64_t* V) {
    if (!g) return GS_ERR_ARG;
    if (n_edges) *n_edges = g->E;
    if (n_tiles) *n_tiles = g->T;
    if (n_items) *n_items = g->I;
    if (V) *V = g->V;
    return GS_OK;
}

gs_status gs_graph_degree(const gs_graph* g, int32_t* host_degree) {
    if (!g || !host_degree) return GS_ERR_ARG;
    GS_CHECK_CUDA(g->ctx, cudaMemcpyAsync(host_degree, g->d_degree, g->V * 4, cudaMemcpyDeviceToHost,
                                          g->ctx->stream));
    GS_CHECK_CUDA(g->ctx, cudaStreamSynchronize(g->ctx->stream));
    return GS_OK;
}

gs_status gs_graph_download(const gs_graph* g, uint64_t* host_start, uint32_t* host_grid,
                            int32_t* host_degree) {
    if (!g) return GS_ERR_ARG;
    gs_ctx* ctx = g->ctx;
    if (host_start) std::memcpy(host_start, g->h_start.data(), g->h_start.size() * 8);
    if (host_grid && g->E) {
        if (g->stream) {
            if (!gs_stream_read_records(g, host_grid)) return gs_fail(ctx, GS_ERR_FORMAT, "reading the records failed");
        }
        else GS_CHECK_CUDA(ctx, cudaMemcpyAsync(host_grid, g->d_rec, g->E * 4, cudaMemcpyDeviceToHost, ctx->stream));
    }
    if (host_degree)
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(host_degree, g->d_degree, g->V * 4, cudaMemcpyDeviceToHost, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return GS_OK;
}

// ------------------------------------------------------------------ state --
gs_status gs_state_create(gs_graph* g, gs_algo algo, int64_t arg, gs_state** out) {
    if (!g || !out) return GS_ERR_ARG;
    *out = nullptr;
    gs_ctx* ctx = g->ctx;
    if (algo == GS_ALGO_KCORE && g->directed)
        return gs_fail(ctx, GS_ERR_UNSUPPORTED, "Kcore not applicable for directed graphs");
    if (algo == GS_ALGO_BFS && (arg < 0 || (uint64_t)arg >= g->V))
        return gs_fail(ctx, GS_ERR_ARG, "BFS root out of range");
    if (algo == GS_ALGO_PAGERANK && arg < 1) return gs_fail(ctx, GS_ERR_ARG, "iterations < 1");
    if ((algo == GS_ALGO_BFS2 || algo == GS_ALGO_TRAVERSE) && (arg < 0 || (uint64_t)arg >= g->V))
        return gs_fail(ctx, GS_ERR_ARG, "root out of range");
    gs_state* s = new (std::nothrow) gs_state();
    if (!s) return GS_ERR_OOM;
    s->g = g;
    s->algo = algo;
    s->arg = arg;
    gs_status st = GS_ERR_ARG;
    switch (algo) {
        case GS_ALGO_BFS: st = bfs_init(s); break;
        case GS_ALGO_PAGERANK: st = pr_init(s); break;
        case GS_ALGO_WCC: st = wcc_init(s); break;
        case GS_ALGO_KCORE: st = kcore_init(s); break;
        case GS_ALGO_BFS2:
        case GS_ALGO_TRAVERSE: st = lab_init(s); break;
    }
    if (st != GS_OK) {
        gs_state_free(s);
        return st;
    }
    *out = s;
    return GS_OK;
}

gs_status gs_state_reset(gs_state* s, int64_t arg) {
    if (!s) return GS_ERR_ARG;
    gs_graph* g = s->g;
    if ((s->algo == GS_ALGO_BFS || s->algo == GS_ALGO_BFS2 || s->algo == GS_ALGO_TRAVERSE) &&
        (arg < 0 || (uint64_t)arg >= g->V))
        return gs_fail(g->ctx, GS_ERR_ARG, "BFS root out of range");
    if (s->algo == GS_ALGO_PAGERANK && arg < 1) return gs_fail(g->ctx, GS_ERR_ARG, "iterations < 1");
    s->arg = arg;
    s->step = 0;
    s->swept = false;
    s->done = false;
    s->last_count = 0;
    switch (s->algo) {
        case GS_ALGO_BFS: return bfs_init(s);
        case GS_ALGO_PAGERANK: return pr_init(s);
        case GS_ALGO_WCC: return wcc_init(s);
        case GS_ALGO_KCORE: return kcore_init(s);
        case GS_ALGO_BFS2:
        case GS_ALGO_TRAVERSE: return lab_init(s);
    }
    return GS_ERR_ARG;
}

gs_status gs_state_free(gs_state* s) {
    if (!s) return GS_OK;
    // the state's kernels are done before its buffers go back to the pool
    cudaStreamSynchronize(s->g->ctx->stream);
    for (auto& pb : s->allocs) gs_pool_put(s->g->ctx, pb.first, pb.second);
    delete s;
    return GS_OK;
}

gs_status gs_pagerank_compat(gs_state* s, int enable) {
    if (!s || s->algo != GS_ALGO_PAGERANK) return GS_ERR_ARG;
    if (s->step != 0) return gs_fail(s->g->ctx, GS_ERR_STATE, "compat must precede the first sweep");
    s->compat = enable != 0;
    return GS_OK;
}

}  // extern "C"

static gs_status sweep_launch(gs_state* s) {
    switch (s->algo) {
        case GS_ALGO_BFS: return bfs_sweep_launch(s);
        case GS_ALGO_PAGERANK: return pr_sweep_launch(s);
        case GS_ALGO_WCC: return wcc_sweep_launch(s);
        case GS_ALGO_KCORE: return kcore_sweep_launch(s);
        case GS_ALGO_BFS2:
        case GS_ALGO_TRAVERSE: return lab_sweep_launch(s);
    }
    return GS_ERR_ARG;
}

extern "C" {

gs_status gs_sweep(gs_state* s, const gs_segment* segs, int n_segs) {
    if (!s) return GS_ERR_ARG;
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    if (n_segs < 0 || (n_segs > 0 && !segs)) return gs_fail(ctx, GS_ERR_ARG, "bad segment list");
    if (s->done) return gs_fail(ctx, GS_ERR_STATE, "algorithm already finished");
    if (!s->swept) {
        // once per sweep, however many segment calls make it up
        if (s->algo == GS_ALGO_BFS) GS_TRY(bfs_sweep_begin(s));
        if (s->algo == GS_ALGO_WCC) GS_TRY(wcc_sweep_begin(s));
        if (s->algo == GS_ALGO_BFS2 || s->algo == GS_ALGO_TRAVERSE) GS_TRY(lab_sweep_begin(s));
        s->swept = true;
    }
    auto launch = [s]() { return sweep_launch(s); };
    if (n_segs > 0) return gs_each_part(g, segs, n_segs, launch);
    gs_need need;
    std::vector<uint8_t> act;
    if (g->stream && s->algo != GS_ALGO_PAGERANK && s->algo != GS_ALGO_WCC) {
        // the window flags the skip rule reads: BFS frontier windows
        // (bfs.cpp:290-312), k-core windows of removed vertices
        // (gstore.cpp:2773-2782)
        act.resize(g->nw);
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(act.data(), s->d_act, g->nw, cudaMemcpyDeviceToHost, ctx->stream));
        GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        need.act = act.data();
        // traverse colours v1 from v0 only: its tiles follow their row window
        need.by_col = !g->directed && s->algo != GS_ALGO_TRAVERSE;
    }
    std::vector<uint8_t> dead_units;
    if (g->stream && s->algo == GS_ALGO_BFS && s->sweep_skip) {
        // units whose chunks are all dead need not cross PCIe at all
        dead_units.resize(g->U);
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(dead_units.data(), s->d_dead, g->U, cudaMemcpyDeviceToHost, ctx->stream));
        GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        for (uint64_t u = 0; u < g->U; ++u) {
            const gs_unit& d = g->h_units[u];
            const uint64_t b = d.rec_beg, e = d.rec_beg + d.n;
            const uint64_t ab = std::min<uint64_t>((b + 3) & ~3ull, e);
            const uint64_t ae = std::max<uint64_t>(e & ~3ull, ab);
            const uint64_t n4 = (ae - ab) >> 2;
            const uint32_t nch = n4 ? (uint32_t)((n4 + 63) >> 6) : 1u;   // the sweep kernel's chunks
            dead_units[u] = dead_units[u] == ((1u << nch) - 1u) ? 1 : 0;
        }
        need.dead_units = dead_units.data();
    }
    return gs_each_segment(g, need, s->step & 1, launch);
}

gs_status gs_finalize(gs_state* s, int64_t* frontier_out, int* done_out) {
    if (!s) return GS_ERR_ARG;
    if (s->swept) {
        s->step += 1;
        s->swept = false;
    }
    int64_t f = 0;
    int d = 0;
    gs_status st = GS_ERR_ARG;
    switch (s->algo) {
        case GS_ALGO_BFS: st = bfs_finalize(s, &f, &d); break;
        case GS_ALGO_PAGERANK: st = pr_finalize(s, &f, &d); break;
        case GS_ALGO_WCC: st = wcc_finalize(s, &f, &d); break;
        case GS_ALGO_KCORE: st = kcore_finalize(s, &f, &d); break;
        case GS_ALGO_BFS2:
        case GS_ALGO_TRAVERSE: st = lab_finalize(s, &f, &d); break;
    }
    if (st != GS_OK) return st;
    s->last_count = f;
    s->done = d != 0;
    if (frontier_out) *frontier_out = f;
    if (done_out) *done_out = d;
    return GS_OK;
}

gs_status gs_run(gs_state* s, int64_t* steps_out) {
    if (!s) return GS_ERR_ARG;
    int64_t steps = 0;
    if (s->algo == GS_ALGO_KCORE && s->step == 0 && !s->done) {
        // kcore_mmap runs one iteration_finalize before the first sweep
        // (gstore.cpp:2725-2726).
        int64_t f;
        int d;
        GS_TRY(gs_finalize(s, &f, &d));
    }
    while (!s->done) {
        GS_TRY(gs_sweep(s, nullptr, 0));
        ++steps;
        int64_t f;
        int d;
        GS_TRY(gs_finalize(s, &f, &d));
    }
    if (steps_out) *steps_out = steps;
    return GS_OK;
}

gs_status gs_download(gs_state* s, int what, void* host_dst, uint64_t bytes) {
    if (!s || !host_dst) return GS_ERR_ARG;
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    const void* src = nullptr;
    uint64_t need = 0;
    if ((s->algo == GS_ALGO_BFS2 || s->algo == GS_ALGO_WCC) && !s->d_out)
        GS_TRY(gs_state_alloc(s, (void**)&s->d_out, g->N * 4));
    switch (s->algo) {
        case GS_ALGO_BFS: src = s->d_depth; need = g->V; break;
        case GS_ALGO_PAGERANK: src = what == 1 ? s->d_x : s->d_r; need = g->V * 4; break;
        case GS_ALGO_KCORE: src = s->d_deg; need = g->V * 4; break;
        case GS_ALGO_TRAVERSE: src = s->d_lab; need = g->V * 4; break;
        case GS_ALGO_BFS2: {
            uint64_t cnt;
            GS_TRY(lab_result(s, (uint8_t*)s->d_out, &cnt));
            src = s->d_out;
            need = g->V;
            break;
        }
        case GS_ALGO_WCC: {
            uint64_t cnt;
            GS_TRY(gs_wcc_labels(s, s->d_out, &cnt));
            src = s->d_out;
            need = g->V * 4;
            break;
        }
    }
    if (bytes < need) return gs_fail(ctx, GS_ERR_ARG, "destination too small: need " + std::to_string(need));
    cudaError_t e = cudaMemcpyAsync(host_dst, src, need, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return gs_cuda_fail(ctx, e, "download");
    return GS_OK;
}

gs_status gs_result_count(gs_state* s, uint64_t* count) {
    if (!s || !count) return GS_ERR_ARG;
    switch (s->algo) {
        case GS_ALGO_BFS: {
            uint64_t e;
            return gs_count_reached(s, count, &e);
        }
        case GS_ALGO_KCORE: return gs_count_kcore(s, count);
        case GS_ALGO_WCC:
            if (!s->d_out) GS_TRY(gs_state_alloc(s, (void**)&s->d_out, s->g->N * 4));
            return gs_wcc_labels(s, s->d_out, count);
        case GS_ALGO_PAGERANK: *count = (uint64_t)s->step; return GS_OK;
        case GS_ALGO_BFS2:
        case GS_ALGO_TRAVERSE: return lab_result(s, nullptr, count);
    }
    return GS_ERR_ARG;
}

gs_status gs_bfs_stats(gs_state* s, uint64_t* edges_in_component, uint64_t* swept_records,
                       int max_levels, int* n_levels, uint64_t* level_counts) {
    if (!s || s->algo != GS_ALGO_BFS) return GS_ERR_ARG;
    if (edges_in_component) {
        uint64_t reached;
        GS_TRY(gs_count_reached(s, &reached, edges_in_component));
    }
    int nl = (int)s->level_counts.size();
    if (n_levels) *n_levels = nl;
    if (level_counts)
        for (int l = 0; l < nl && l < max_levels; ++l) level_counts[l] = s->level_counts[l];
    if (swept_records) {
        const int nh = std::min(std::min(nl, max_levels), std::min(s->n_act_hist, 256));
        if (nh > 0) {
            gs_ctx* ctx = s->g->ctx;
            const size_t nw = s->g->nw;
            std::vector<uint8_t> hist((size_t)nh * nw);
            GS_CHECK_CUDA(ctx, cudaMemcpyAsync(hist.data(), s->d_act_hist, hist.size(), cudaMemcpyDeviceToHost,
                                               ctx->stream));
            GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            for (int l = 0; l < nh; ++l) {
                uint64_t sw = 0;
                GS_TRY(gs_swept_records(s, hist.data() + (size_t)l * nw, &sw));
                swept_records[l] = sw;
            }
        }
    }
    return GS_OK;
}

gs_status gs_bfs_records_read(gs_state* s, uint64_t* read_records, int max_levels, int* n_levels) {
    if (!s || s->algo != GS_ALGO_BFS || max_levels < 0 || (max_levels && !read_records)) return GS_ERR_ARG;
    const int nl = std::min((int)s->level_counts.size(), 256);
    if (n_levels) *n_levels = nl;
    const int n = std::min(nl, max_levels);
    if (n <= 0) return GS_OK;
    // a level that skipped dead chunks counted what it read; any other read
    // every record of the tiles the reference rule sweeps
    GS_TRY(gs_bfs_stats(s, nullptr, read_records, n, nullptr, nullptr));
    std::vector<uint64_t> counted(n, 0);
    gs_ctx* ctx = s->g->ctx;
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(counted.data(), s->d_read, (size_t)n * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                                       ctx->stream));
    GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int l = 0; l < n; ++l)
        if (l < (int)s->level_skip.size() && s->level_skip[l]) read_records[l] = counted[l];
    return GS_OK;
}

}  // extern "C"
