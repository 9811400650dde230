// Tile-grid sweep kernels (sm_100a) and per-vertex finalize kernels for
// PageRank, WCC and k-core (BFS has its own sweep in gs_bfs.cu).
//
// Work decomposition: the non-empty tiles are cut into units (<= kUnitRecords
// records of one tile) and the units grouped into runs (units of one tile
// row).  A CTA takes a run at a time, a warp a unit; records stream with
// 128-bit evict-first loads and the per-vertex state (ranks, labels,
// degrees) is the reused working set.  PageRank, WCC and k-core walk the
// L2-blocked run order (tiles grouped by 64 x 64-window blocks), which keeps
// that working set in L2.
//
// Reference semantics per record (edge_t{v0, v1} in tile (i, j)):
//   BFS     bfs.cpp:138-185     discover the unvisited end of a frontier end
//   PR      pr.cpp:119-154      s[v1] += x[v0]; s[v0] += x[v1] (half grid)
//   WCC     wcc.cpp:177-278     hook the larger root onto the smaller one
//   k-core  kcore.cpp:63-177    --deg[other] for every removed endpoint
#include "gs_internal.cuh"
#include "gs_ops.cuh"

namespace {

constexpr int kThreads = 256;
using namespace gsops;

// Generic run sweep.  A CTA takes one run at a time (consecutive tiles of one
// tile row inside a group; the next from `ticket` when one is given, else
// every gridDim.x-th), its warps take the run's units (tile slices of at
// most kUnitRecords records) and stream their records with 128-bit
// evict-first loads.  When `seg` lists runs, only those are swept and their
// units are read from a segment buffer (file record r at rec[r + delta]).
// Op is one of the per-record operations of gs_ops.cuh.
template <class Op>
__global__ void __launch_bounds__(kThreads) sweep_runs(const gs_tile_run* __restrict__ runs, uint64_t n_runs,
                                                       const gs_unit* __restrict__ units,
                                                       const uint32_t* __restrict__ rec,
                                                       const gs_seg_run* __restrict__ seg, Op op,
                                                       unsigned int* ticket) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr uint32_t kWarps = kThreads / 32;
    __shared__ unsigned long long s_run;
    auto advance = [&](uint64_t i) -> uint64_t {
        if (!ticket) return i + gridDim.x;
        __syncthreads();   // every thread has read the previous draw
        if (threadIdx.x == 0) s_run = atomicAdd(ticket, 1u);
        __syncthreads();
        return s_run;
    };
    for (uint64_t i = ticket ? advance(0) : blockIdx.x; i < n_runs; i = advance(i)) {
        uint32_t ub, ue;
        const uint32_t* base = rec;
        if (seg) {
            const gs_seg_run e = seg[i];
            ub = e.unit_beg;
            ue = e.unit_end;
            base = rec + e.delta;
        } else {
            ub = runs[i].unit_beg;
            ue = runs[i].unit_end;
        }
        for (uint32_t ui = ub + warp; ui < ue; ui += kWarps) sweep_unit(units[ui], base, op, lane);
    }
    if (ticket && threadIdx.x == 0 && atomicAdd(ticket + 1, 1u) == gridDim.x - 1) {
        atomicExch(ticket, 0u);   // every CTA has drawn its last ticket
        atomicExch(ticket + 1, 0u);
    }
}

// Sweeps the whole resident graph, or, during a streamed sweep, the runs of
// the segment the graph points at.
template <class Op>
gs_status launch_sweep(gs_graph* g, const Op& op, int algo, uint64_t bytes, bool blocked = false) {
    gs_ctx* ctx = g->ctx;
    const gs_seg_run* seg = g->seg.list;
    if (blocked && !seg) GS_TRY(gs_ensure_blocked(g));
    blocked = blocked && !seg && g->d_runs_blk;
    const uint64_t n = seg ? g->seg.n : (blocked ? g->R_blk : g->R);
    const uint32_t* rec = seg ? g->seg.buf : g->d_rec;
    if (n == 0) return GS_OK;
    const uint32_t grid = (uint32_t)std::min<uint64_t>(n, gs_grid_size(ctx, 8));
    gs_timer_begin(ctx);
    sweep_runs<Op><<<grid, kThreads, 0, ctx->stream>>>(blocked ? g->d_runs_blk : g->d_runs, n,
                                                        blocked ? g->d_units_blk : g->d_units, rec, seg, op,
                                                        ctx->d_ticket);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    gs_timer_end(ctx, algo, seg ? 0 : bytes);
    return GS_OK;
}

inline uint32_t blocks_for(uint64_t n, const gs_ctx* ctx) {
    uint64_t b = (n + kThreads - 1) / kThreads;
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(b, gs_grid_size(ctx, 16)));
}

// ---------------------------------------------------------- validation --
// Flags a record of the last (ragged) window that addresses a vertex >= V.
struct ValidateOp {
    uint32_t last_window;
    uint64_t V;
    int* flag;
    struct Item {
        uint64_t rb, cb;
    };
    __device__ bool begin(uint32_t row, uint32_t col, Item& c) const {
        c.rb = (uint64_t)row << 16;
        c.cb = (uint64_t)col << 16;
        return row == last_window || col == last_window;
    }
    __device__ void record(uint32_t r, Item& c) const {
        if (c.rb + (r & 0xFFFFu) >= V || c.cb + (r >> 16) >= V) *flag = 1;
    }
    __device__ void end(uint32_t, uint32_t, Item&) const {}
};

struct DegreeOp {
    int32_t* deg;
    int directed;
    struct Item {
        uint32_t rb, cb;
    };
    __device__ bool begin(uint32_t row, uint32_t col, Item& c) const {
        c.rb = row << 16;
        c.cb = col << 16;
        return true;
    }
    __device__ void record(uint32_t r, Item& c) const {
        atomicAdd(deg + c.rb + (r & 0xFFFFu), 1);          // gstore.cpp:1308
        if (!directed) atomicAdd(deg + c.cb + (r >> 16), 1);  // gstore.cpp:1310
    }
    __device__ void end(uint32_t, uint32_t, Item&) const {}
};

// -------------------------------------------------------------------- BFS --
__global__ void count_reached_kernel(const uint8_t* __restrict__ depth, uint64_t n,
                                     unsigned long long* out) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    uint64_t local = 0;
    for (uint64_t v = tid; v < n; v += nth) local += depth[v] != 0;
    warp_add_u64(out, local);
}

struct ComponentEdgesOp {
    const uint8_t* depth;
    unsigned long long* out;
    struct Item {
        uint32_t rb, cb;
        uint32_t n;
    };
    __device__ bool begin(uint32_t row, uint32_t col, Item& c) const {
        c.rb = row << 16;
        c.cb = col << 16;
        c.n = 0;
        return true;
    }
    __device__ void record(uint32_t r, Item& c) const {
        c.n += (depth[c.rb + (r & 0xFFFFu)] != 0) && (depth[c.cb + (r >> 16)] != 0);
    }
    __device__ void end(uint32_t, uint32_t, Item& c) const { warp_add_u64(out, c.n); }
};

__global__ void pr_init_kernel(float* x, float* y, uint64_t N, uint64_t V) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    const float x0 = (float)(1.0 / (double)V);         // pr.cpp:105-110
    for (uint64_t v = tid; v < N; v += nth) {
        x[v] = v < V ? x0 : 0.f;
        y[v] = 0.f;
    }
}

// rank = 0.15 + 0.85 s; x = rank * inv_degree; s := 0 (pr.cpp:281-302).  The
// expression is evaluated in double as the reference does (double literals)
// and stored as float.
template <class Acc>
__global__ void pr_finalize_kernel(float* __restrict__ x, Acc* __restrict__ y, float* __restrict__ r_out,
                                   const int32_t* __restrict__ deg, uint64_t N, uint64_t V, int compat) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = tid; v < N; v += nth) {
        const double r = 0.15 + 0.85 * (double)y[v];
        const int32_t d = deg[v];
        double xn;
        if (d == 0 || v >= V) xn = 0.0;
        else if (compat) xn = r * (double)(int32_t)(1.0 / (double)d);   // pr.cpp:112-114
        else xn = r / (double)d;
        r_out[v] = v < V ? (float)r : 0.f;
        x[v] = (float)xn;
        y[v] = 0;
    }
}

__global__ void iota_kernel(uint32_t* parent, uint64_t N) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = tid; v < N; v += nth) parent[v] = (uint32_t)v;
}

// Pointer jumping (wcc.cpp:372-390): every vertex points at its root.
__global__ void compress_kernel(uint32_t* parent, uint64_t N) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = tid; v < N; v += nth) {
        const uint32_t r = find_root(parent, (uint32_t)v);
        if (r != v) parent[v] = r;
    }
}

__global__ void wcc_label_kernel(const uint32_t* parent, const uint8_t* touched, uint32_t* out, uint64_t N,
                                 unsigned long long* count) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    uint64_t local = 0;
    for (uint64_t v = tid; v < N; v += nth) {
        if (!touched[v]) {
            out[v] = 0xFFFFFFFFu;  // invalid_cid, wcc.cpp:54
            continue;
        }
        const uint32_t r = find_root(parent, (uint32_t)v);
        out[v] = r;
        local += (r == v);
    }
    warp_add_u64(count, local);
}

// One warp per 32-vertex word (kcore.cpp:186-209): remove 0 < (int16)deg < k.
__global__ void kcore_round_kernel(int32_t* __restrict__ deg, uint32_t* __restrict__ removed,
                                   uint8_t* __restrict__ act, uint64_t n_words, int k,
                                   unsigned long long* count) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    uint64_t local = 0;
    for (uint64_t w = warp; w < n_words; w += nwarps) {
        const uint64_t v = w * 32 + lane;
        const int16_t m = (int16_t)deg[v];
        const bool gone = m < k && m > 0;
        if (gone) deg[v] = 0;
        const uint32_t bits = __ballot_sync(kFull, gone);
        if (lane == 0) {
            removed[w] = bits;
            if (bits) act[w >> 11] = 1;
            local += __popc(bits);
        }
    }
    if (lane == 0 && local) atomicAdd(count, (unsigned long long)local);
}

__global__ void count_nonzero_kernel(const int32_t* __restrict__ deg, uint64_t n, unsigned long long* out) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    uint64_t local = 0;
    for (uint64_t v = tid; v < n; v += nth) local += deg[v] != 0;
    warp_add_u64(out, local);
}

// ------------------------------------------------------ bfs2, traverse --
constexpr uint32_t kInf = 0xFFFFFFFFu;

// bfs2_t::bfs_onepart (bfs2.cpp:102-117): a record lowers the depth of an end
// to the other end's depth + 1 (depth 1 = root, kInf = unreached).  A tile is
// swept when its row or column window changed in the previous sweep (all
// windows before the first); a change marks its window for the next one.
struct Bfs2Op {
    uint32_t* dist;
    const uint8_t* act;
    uint8_t* act_next;
    unsigned long long* changes;
    int* overflow;
    int directed;
    struct Item {
        uint32_t rb, cb, n;
        bool cr, cc;
    };
    __device__ bool begin(uint32_t row, uint32_t col, Item& c) const {
        c.rb = row << 16;
        c.cb = col << 16;
        c.n = 0;
        c.cr = c.cc = false;
        return act[row] || act[col];
    }
    __device__ void record(uint32_t r, Item& c) const {
        const uint32_t a = c.rb + (r & 0xFFFFu), b = c.cb + (r >> 16);
        const uint32_t da = __ldcg(dist + a), db = __ldcg(dist + b);
        if (da != kInf && (db == kInf || db > da + 1)) {
            if (da >= 255) { *overflow = 1; return; }        // u8 depth_t
            if (atomicMin(dist + b, da + 1) > da + 1) { ++c.n; c.cc = true; }
        } else if (!directed && db != kInf && (da == kInf || da > db + 1)) {
            if (db >= 255) { *overflow = 1; return; }
            if (atomicMin(dist + a, db + 1) > db + 1) { ++c.n; c.cr = true; }
        }
    }
    __device__ void end(uint32_t row, uint32_t col, Item& c) const {
        warp_add_u64(changes, c.n);
        const bool cr = __any_sync(kFull, c.cr), cc = __any_sync(kFull, c.cc);
        if ((threadIdx.x & 31) == 0) {
            if (cr) act_next[row] = 1;   // read_part_next->set_bit_atomic(i), bfs2.cpp:126-128
            if (cc) act_next[col] = 1;   // bfs2.cpp:120-123
        }
    }
};

// traverse_t::traverse_onepart (traverse.cpp:173-188): a record colours v1
// from v0 (one direction, also in the half grid).  A tile is swept when its
// row window gained colour in the previous sweep (the pivot's window first).
struct TraverseOp {
    uint32_t* cid;
    const uint8_t* act;
    uint8_t* act_next;
    unsigned long long* changes;
    struct Item {
        uint32_t rb, cb, n;
        bool cc;
    };
    __device__ bool begin(uint32_t row, uint32_t col, Item& c) const {
        c.rb = row << 16;
        c.cb = col << 16;
        c.n = 0;
        c.cc = false;
        return act[row] != 0;
    }
    __device__ void record(uint32_t r, Item& c) const {
        const uint32_t a = c.rb + (r & 0xFFFFu), b = c.cb + (r >> 16);
        if (__ldcg(cid + a) == 0 && __ldcg(cid + b) == kInf && atomicCAS(cid + b, kInf, 0u) == kInf) {
            ++c.n;
            c.cc = true;
        }
    }
    __device__ void end(uint32_t, uint32_t col, Item& c) const {
        warp_add_u64(changes, c.n);
        if (__any_sync(kFull, c.cc) && (threadIdx.x & 31) == 0) act_next[col] = 1;
    }
};

__global__ void lab_to_depth_kernel(const uint32_t* __restrict__ dist, uint8_t* __restrict__ depth, uint64_t V,
                                    unsigned long long* reached) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    uint64_t local = 0;
    for (uint64_t v = tid; v < V; v += nth) {
        const uint32_t d = dist[v];
        if (depth) depth[v] = d == kInf ? 0 : (uint8_t)d;
        local += d != kInf;
    }
    warp_add_u64(reached, local);
}

__global__ void count_value_kernel(const uint32_t* __restrict__ lab, uint64_t V, uint32_t value,
                                   unsigned long long* out) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    uint64_t local = 0;
    for (uint64_t v = tid; v < V; v += nth) local += lab[v] == value;
    warp_add_u64(out, local);
}

gs_status read_scalar(gs_ctx* ctx, uint64_t* value) {
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->h_scalars, ctx->d_scalars, sizeof(uint64_t),
                                       cudaMemcpyDeviceToHost, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *value = ctx->h_scalars[0];
    return GS_OK;
}

gs_status zero_scalar(gs_ctx* ctx) {
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_scalars, 0, sizeof(uint64_t), ctx->stream));
    return GS_OK;
}

}  // namespace

// ================================================================ launchers ==
gs_status launch_validate_records(gs_graph* g, int* d_flag) {
    ValidateOp op{g->nw - 1, g->V, d_flag};
    return gs_each_segment(g, gs_need{}, 0, [&]() { return launch_sweep(g, op, 0, 0); });
}

gs_status launch_degree_from_records(gs_graph* g) {
    DegreeOp op{g->d_degree, g->directed};
    return gs_each_segment(g, gs_need{}, 0, [&]() { return launch_sweep(g, op, 0, 0); });
}

// ------------------------------------------------------------------- BFS ----
gs_status gs_count_reached(gs_state* s, uint64_t* reached, uint64_t* edges_in_component) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    GS_TRY(zero_scalar(ctx));
    count_reached_kernel<<<blocks_for(g->V, ctx), kThreads, 0, ctx->stream>>>(
        s->d_depth, g->V, (unsigned long long*)ctx->d_scalars);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    GS_TRY(read_scalar(ctx, reached));
    GS_TRY(zero_scalar(ctx));
    ComponentEdgesOp op{s->d_depth, (unsigned long long*)ctx->d_scalars};
    GS_TRY(gs_each_segment(g, gs_need{}, 0, [&]() { return launch_sweep(g, op, 0, 0); }));
    GS_TRY(read_scalar(ctx, edges_in_component));
    return GS_OK;
}

gs_status gs_swept_records(gs_state* s, const uint8_t* act, uint64_t* swept) {
    gs_graph* g = s->g;
    uint64_t sum = 0;
    for (uint64_t t = 0; t < g->T; ++t) {
        const uint32_t rc = g->h_tile_rc[t];
        const uint32_t row = rc >> 16, col = rc & 0xFFFFu;
        if (act[row] || (!g->directed && act[col])) sum += g->h_tile_off[t + 1] - g->h_tile_off[t];
    }
    *swept = sum;
    return GS_OK;
}

// -------------------------------------------------------------- PageRank ----
gs_status pr_init(gs_state* s) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    if (!s->d_x) GS_TRY(gs_state_alloc(s, (void**)&s->d_x, g->N * 4));
    // the sums of a streamed graph's sweep are doubles (PrOp<double>)
    if (!s->d_y) GS_TRY(gs_state_alloc(s, (void**)&s->d_y, g->N * (g->stream ? 8 : 4)));
    if (!s->d_r) GS_TRY(gs_state_alloc(s, (void**)&s->d_r, g->N * 4));
    pr_init_kernel<<<blocks_for(g->N, ctx), kThreads, 0, ctx->stream>>>(s->d_x, s->d_y, g->N, g->V);
    if (g->stream) GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_y, 0, g->N * 8, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_r, 0, g->N * 4, ctx->stream));
    if (s->d_error) GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_error, 0, sizeof(uint64_t), ctx->stream));
    // resident graphs sweep the propagation-blocked layout when it is worth
    // building and fits, else the row-slice layout (each built once per graph)
    if (!g->stream && g->E && !g->pb.built && !g->pr.built) {
        if (pb_layout_wanted(g)) GS_TRY(pb_layout_build(g));
        else GS_TRY(pr_layout_build(g));
    }
    return GS_OK;
}

gs_status pr_sweep_launch(gs_state* s) {
    gs_graph* g = s->g;
    if (!g->seg.list && g->pb.built) return pb_launch(s);
    if (!g->seg.list && g->pr.built) return pr_slice_launch(s);
    if (g->stream) {
        PrOp<double> op{s->d_x, reinterpret_cast<double*>(s->d_y), g->directed};
        return launch_sweep(g, op, GS_ALGO_PAGERANK, 4 * g->E + 12 * g->V, true);
    }
    PrOp<float> op{s->d_x, s->d_y, g->directed};
    // algorithmic bytes per iteration: 4E + 12V (records, x, s, inv)
    return launch_sweep(g, op, GS_ALGO_PAGERANK, 4 * g->E + 12 * g->V, true);
}

gs_status pr_finalize_launch(gs_ctx* ctx, cudaStream_t stream, float* x, float* y, float* r, const int32_t* deg,
                             uint64_t N, uint64_t V, int compat) {
    pr_finalize_kernel<float><<<blocks_for(N, ctx), kThreads, 0, stream>>>(x, y, r, deg, N, V, compat);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    return GS_OK;
}

gs_status pr_finalize(gs_state* s, int64_t* frontier, int* done) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    if (g->stream)
        pr_finalize_kernel<double><<<blocks_for(g->N, ctx), kThreads, 0, ctx->stream>>>(
            s->d_x, reinterpret_cast<double*>(s->d_y), s->d_r, g->d_degree, g->N, g->V, s->compat ? 1 : 0);
    else
        pr_finalize_kernel<float><<<blocks_for(g->N, ctx), kThreads, 0, ctx->stream>>>(
            s->d_x, s->d_y, s->d_r, g->d_degree, g->N, g->V, s->compat ? 1 : 0);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    *frontier = s->step;
    *done = s->step >= s->arg;
    if (*done && s->d_error) {
        // the row-slice sweep's bounded waits report here, once per run
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->h_scalars, s->d_error, 8, cudaMemcpyDeviceToHost, ctx->stream));
        GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        if (ctx->h_scalars[0]) return gs_fail(ctx, GS_ERR_TIMEOUT, "PageRank sweep: a bounded wait gave up");
    } else if (*done) {
        GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return GS_OK;
}

// ------------------------------------------------------------------- WCC ----
gs_status wcc_init(gs_state* s) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    if (!s->d_parent) GS_TRY(gs_state_alloc(s, (void**)&s->d_parent, g->N * 4));
    if (!s->d_touched) GS_TRY(gs_state_alloc(s, (void**)&s->d_touched, g->N));
    iota_kernel<<<blocks_for(g->N, ctx), kThreads, 0, ctx->stream>>>(s->d_parent, g->N);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_touched, 0, g->N, ctx->stream));
    return GS_OK;
}

gs_status wcc_sweep_begin(gs_state* s) { return zero_scalar(s->g->ctx); }

gs_status wcc_sweep_launch(gs_state* s) {
    gs_graph* g = s->g;
    WccOp op{s->d_parent, s->step == 0 ? s->d_touched : nullptr,
             (unsigned long long*)g->ctx->d_scalars};
    return launch_sweep(g, op, GS_ALGO_WCC, 4 * g->E + 8 * g->V, true);
}

gs_status wcc_finalize(gs_state* s, int64_t* frontier, int* done) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    uint64_t changes = 0;
    GS_TRY(read_scalar(ctx, &changes));
    compress_kernel<<<blocks_for(g->N, ctx), kThreads, 0, ctx->stream>>>(s->d_parent, g->N);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    *frontier = (int64_t)changes;
    *done = changes == 0;
    return GS_OK;
}

gs_status gs_wcc_labels(gs_state* s, uint32_t* d_out, uint64_t* count) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    GS_TRY(zero_scalar(ctx));
    wcc_mark_touched<<<blocks_for(g->N, ctx), kThreads, 0, ctx->stream>>>(s->d_parent, s->d_touched, g->N);
    wcc_label_kernel<<<blocks_for(g->N, ctx), kThreads, 0, ctx->stream>>>(
        s->d_parent, s->d_touched, d_out, g->N, (unsigned long long*)ctx->d_scalars);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches += 2;
    return read_scalar(ctx, count);
}

// ---------------------------------------------------------------- k-core ----
gs_status kcore_init(gs_state* s) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    if (!s->d_deg) GS_TRY(gs_state_alloc(s, (void**)&s->d_deg, g->N * 4));
    if (!s->d_kactive) GS_TRY(gs_state_alloc(s, (void**)&s->d_kactive, g->N / 8));
    if (!s->d_act) GS_TRY(gs_state_alloc(s, (void**)&s->d_act, g->nw));
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(s->d_deg, g->d_degree, g->N * 4, cudaMemcpyDeviceToDevice, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_kactive, 0, g->N / 8, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_act, 0, g->nw, ctx->stream));
    return GS_OK;
}

gs_status kcore_sweep_launch(gs_state* s) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    // Algorithmic bytes of the round, counted only while kernel timing is on:
    // the records of the tiles whose row or column window holds a vertex
    // removed this round (the tiles kcore_mmap sweeps, gstore.cpp:2773-2782),
    // plus the degree and removed-bit reads and the degree writes (8 B/vertex).
    uint64_t bytes = 0;
    if (ctx->profile && !g->seg.list) {
        std::vector<uint8_t> act(g->nw);
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(act.data(), s->d_act, g->nw, cudaMemcpyDeviceToHost, ctx->stream));
        GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        uint64_t swept = 0;
        GS_TRY(gs_swept_records(s, act.data(), &swept));
        bytes = 4 * swept + 8 * g->V;
    }
    KcoreOp op{s->d_deg, s->d_kactive, s->d_act};
    return launch_sweep(g, op, GS_ALGO_KCORE, bytes, true);
}

gs_status kcore_finalize(gs_state* s, int64_t* frontier, int* done) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    GS_TRY(zero_scalar(ctx));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_act, 0, g->nw, ctx->stream));
    const uint64_t words = g->N / 32;
    kcore_round_kernel<<<blocks_for(words * 32, ctx), kThreads, 0, ctx->stream>>>(
        s->d_deg, s->d_kactive, s->d_act, words, (int)s->arg, (unsigned long long*)ctx->d_scalars);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    uint64_t removed = 0;
    GS_TRY(read_scalar(ctx, &removed));
    *frontier = (int64_t)removed;
    *done = removed == 0;
    return GS_OK;
}

gs_status gs_count_kcore(gs_state* s, uint64_t* members) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    GS_TRY(zero_scalar(ctx));
    count_nonzero_kernel<<<blocks_for(g->N, ctx), kThreads, 0, ctx->stream>>>(
        s->d_deg, g->N, (unsigned long long*)ctx->d_scalars);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    return read_scalar(ctx, members);
}

// ------------------------------------------------------- bfs2 / traverse ----
gs_status lab_init(gs_state* s) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    if (!s->d_lab) GS_TRY(gs_state_alloc(s, (void**)&s->d_lab, g->N * 4));
    if (!s->d_act) GS_TRY(gs_state_alloc(s, (void**)&s->d_act, g->nw));
    if (!s->d_act_next) GS_TRY(gs_state_alloc(s, (void**)&s->d_act_next, g->nw));
    if (!s->d_error) GS_TRY(gs_state_alloc(s, (void**)&s->d_error, sizeof(uint64_t)));
    const uint64_t v = (uint64_t)s->arg;
    const bool bfs2 = s->algo == GS_ALGO_BFS2;
    // bfs2: every vertex unreached, root depth 1, every window active
    // (bfs2.cpp:56-78); traverse: invalid colour, pivot colour 0, the
    // pivot's window active (traverse.cpp:56-72)
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_lab, 0xFF, g->N * 4, ctx->stream));
    const uint32_t first = bfs2 ? 1u : 0u;
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(s->d_lab + v, &first, 4, cudaMemcpyHostToDevice, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_act, bfs2 ? 1 : 0, g->nw, ctx->stream));
    if (!bfs2) GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_act + (v >> 16), 1, 1, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_act_next, 0, g->nw, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_error, 0, sizeof(uint64_t), ctx->stream));
    GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));   // `first` lives on this stack frame
    return GS_OK;
}

gs_status lab_sweep_begin(gs_state* s) { return zero_scalar(s->g->ctx); }

gs_status lab_sweep_launch(gs_state* s) {
    gs_graph* g = s->g;
    unsigned long long* changes = (unsigned long long*)g->ctx->d_scalars;
    if (s->algo == GS_ALGO_BFS2) {
        Bfs2Op op{s->d_lab, s->d_act, s->d_act_next, changes, (int*)s->d_error, g->directed};
        return launch_sweep(g, op, GS_ALGO_BFS2, 0, true);
    }
    TraverseOp op{s->d_lab, s->d_act, s->d_act_next, changes};
    return launch_sweep(g, op, GS_ALGO_TRAVERSE, 0, true);
}

// iteration_finalize of bfs2_t / traverse_t (bfs2.cpp:130-181,
// traverse.cpp:191-212): the sweep's changes; done when there were none.
gs_status lab_finalize(gs_state* s, int64_t* frontier, int* done) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    uint64_t changes = 0;
    GS_TRY(read_scalar(ctx, &changes));
    std::swap(s->d_act, s->d_act_next);
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_act_next, 0, g->nw, ctx->stream));
    *frontier = (int64_t)changes;
    *done = changes == 0;
    if (s->algo == GS_ALGO_BFS2) {
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->h_scalars, s->d_error, 8, cudaMemcpyDeviceToHost, ctx->stream));
        GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        if (ctx->h_scalars[0]) return gs_fail(ctx, GS_ERR_RANGE, "bfs2 exceeds 254 levels (u8 depth_t)");
    }
    return GS_OK;
}

// bfs2: u8 depth into d_out (may be null) and the reached count; traverse:
// the number of vertices with colour 0.
gs_status lab_result(gs_state* s, uint8_t* d_out, uint64_t* count) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    GS_TRY(zero_scalar(ctx));
    if (s->algo == GS_ALGO_BFS2)
        lab_to_depth_kernel<<<blocks_for(g->V, ctx), kThreads, 0, ctx->stream>>>(
            s->d_lab, d_out, g->V, (unsigned long long*)ctx->d_scalars);
    else
        count_value_kernel<<<blocks_for(g->V, ctx), kThreads, 0, ctx->stream>>>(
            s->d_lab, g->V, 0u, (unsigned long long*)ctx->d_scalars);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    return read_scalar(ctx, count);
}
