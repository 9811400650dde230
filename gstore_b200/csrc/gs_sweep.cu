// Tile-grid sweep kernels (sm_100a) and per-vertex finalize kernels for BFS,
// PageRank, WCC and k-core.
//
// Work decomposition: the records of every non-empty tile are cut into work
// items of at most kItemRecords records (one tile each); a warp owns an item
// at a time (grid-stride over items in file order, so the warps of one CTA
// mostly work along one tile row).  Records stream with 128-bit evict-first
// loads; the per-vertex state (bitmaps, depth, ranks, labels, degrees) is the
// reused working set that stays in L2.
//
// Reference semantics per record (edge_t{v0, v1} in tile (i, j)):
//   BFS     bfs.cpp:138-185     discover the unvisited end of a frontier end
//   PR      pr.cpp:119-154      s[v1] += x[v0]; s[v0] += x[v1] (half grid)
//   WCC     wcc.cpp:177-278     hook the larger root onto the smaller one
//   k-core  kcore.cpp:63-177    --deg[other] for every removed endpoint
#include "gs_internal.cuh"

namespace {

constexpr int kThreads = 256;
constexpr unsigned kFull = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t bit_of(const uint32_t* __restrict__ bm, uint32_t v) {
    return (__ldg(bm + (v >> 5)) >> (v & 31)) & 1u;
}

__device__ __forceinline__ uint4 load_stream(const uint4* p) { return __ldcs(p); }

// Generic run sweep.  A CTA takes one run at a time (consecutive tiles of one
// tile row inside a group), its warps take the run's units (tile slices of at
// most kUnitRecords records) and stream their records with 128-bit
// evict-first loads.  When `seg` lists runs, only those are swept and their
// units are read from a segment buffer (file record r at rec[r + delta]).
// Op provides:
//   struct Item;                                    per-unit warp-uniform context
//   bool begin(uint32_t row, uint32_t col, Item&)   false = skip the unit
//   void record(uint32_t rec, Item&)                one record, any lane
//   void end(uint32_t row, uint32_t col, Item&)     warp-collective epilogue
template <class Op>
__global__ void __launch_bounds__(kThreads) sweep_runs(const gs_tile_run* __restrict__ runs, uint64_t n_runs,
                                                       const gs_unit* __restrict__ units,
                                                       const uint32_t* __restrict__ rec,
                                                       const gs_seg_run* __restrict__ seg, Op op) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr uint32_t kWarps = kThreads / 32;
    for (uint64_t i = blockIdx.x; i < n_runs; i += gridDim.x) {
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
        for (uint32_t ui = ub + warp; ui < ue; ui += kWarps) {
            const gs_unit d = units[ui];
            const uint32_t row = d.rc >> 16, col = d.rc & 0xFFFFu;
            typename Op::Item ic;
            if (!op.begin(row, col, ic)) continue;
            const uint64_t b = d.rec_beg, e = d.rec_beg + d.n;
            uint64_t ab = (b + 3) & ~3ull;
            if (ab > e) ab = e;
            uint64_t ae = e & ~3ull;
            if (ae < ab) ae = ab;
            if (b + lane < ab) op.record(__ldcs(base + b + lane), ic);
            if (ae + lane < e) op.record(__ldcs(base + ae + lane), ic);
            const uint4* r4 = reinterpret_cast<const uint4*>(base + ab);
            const uint32_t n4 = (uint32_t)((ae - ab) >> 2);
            for (uint32_t k = lane; k < n4; k += 2 * 32) {
                const uint4 q0 = load_stream(r4 + k);
                const bool two = k + 32 < n4;
                uint4 q1 = make_uint4(0, 0, 0, 0);
                if (two) q1 = load_stream(r4 + k + 32);
                op.record(q0.x, ic);
                op.record(q0.y, ic);
                op.record(q0.z, ic);
                op.record(q0.w, ic);
                if (two) {
                    op.record(q1.x, ic);
                    op.record(q1.y, ic);
                    op.record(q1.z, ic);
                    op.record(q1.w, ic);
                }
            }
            op.end(row, col, ic);
        }
    }
}

// Sweeps the whole resident graph, or, during a streamed sweep, the runs of
// the segment the graph points at.
template <class Op>
gs_status launch_sweep(gs_graph* g, const Op& op, int algo, uint64_t bytes, bool blocked = false) {
    gs_ctx* ctx = g->ctx;
    const gs_seg_run* seg = g->seg.list;
    blocked = blocked && !seg && g->d_runs_blk;
    const uint64_t n = seg ? g->seg.n : (blocked ? g->R_blk : g->R);
    const uint32_t* rec = seg ? g->seg.buf : g->d_rec;
    if (n == 0) return GS_OK;
    const uint32_t grid = (uint32_t)std::min<uint64_t>(n, gs_grid_size(ctx, 8));
    gs_timer_begin(ctx);
    sweep_runs<Op><<<grid, kThreads, 0, ctx->stream>>>(blocked ? g->d_runs_blk : g->d_runs, n,
                                                        blocked ? g->d_units_blk : g->d_units, rec, seg, op);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    gs_timer_end(ctx, algo, seg ? 0 : bytes);
    return GS_OK;
}

inline uint32_t blocks_for(uint64_t n, const gs_ctx* ctx) {
    uint64_t b = (n + kThreads - 1) / kThreads;
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(b, gs_grid_size(ctx, 16)));
}

__device__ __forceinline__ void warp_add_u64(unsigned long long* dst, uint64_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(dst, (unsigned long long)v);
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

// --------------------------------------------------------------- PageRank --
struct PrOp {
    const float* x;
    float* y;
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
        const uint32_t a = c.rb + (r & 0xFFFFu), b = c.cb + (r >> 16);
        atomicAdd(y + b, __ldg(x + a));                 // pr.cpp:145-146
        if (!directed) atomicAdd(y + a, __ldg(x + b));  // pr.cpp:147-150
    }
    __device__ void end(uint32_t, uint32_t, Item&) const {}
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
__global__ void pr_finalize_kernel(float* __restrict__ x, float* __restrict__ y, float* __restrict__ r_out,
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
        y[v] = 0.f;
    }
}

// -------------------------------------------------------------------- WCC --
__device__ __forceinline__ uint32_t find_root(const uint32_t* parent, uint32_t v) {
    uint32_t p = __ldcg(parent + v);
    while (p != v) {
        v = p;
        p = __ldcg(parent + v);
    }
    return v;
}

struct WccOp {
    uint32_t* parent;
    uint8_t* touched;  // non-null on the first sweep
    unsigned long long* changes;
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
        const uint32_t a = c.rb + (r & 0xFFFFu), b = c.cb + (r >> 16);
        if (touched) {          // wcc.cpp:203-217: every record's ends get a label
            touched[a] = 1;
            touched[b] = 1;
        }
        const uint32_t ra = find_root(parent, a), rb = find_root(parent, b);
        if (ra != rb) {         // wcc.cpp:218-231, 263-275: hook toward the smaller
            const uint32_t hi = ra > rb ? ra : rb, lo = ra > rb ? rb : ra;
            if (atomicMin(parent + hi, lo) > lo) c.n += 1;
        }
    }
    __device__ void end(uint32_t, uint32_t, Item& c) const { warp_add_u64(changes, c.n); }
};

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

// ----------------------------------------------------------------- k-core --
struct KcoreOp {
    int32_t* deg;
    const uint32_t* removed;
    const uint8_t* act;
    struct Item {
        uint32_t rb, cb;
        bool fr, fc;
    };
    __device__ bool begin(uint32_t row, uint32_t col, Item& c) const {
        // kcore_mmap dispatch (gstore.cpp:2773-2782)
        c.fr = act[row] != 0;
        c.fc = act[col] != 0;
        c.rb = row << 16;
        c.cb = col << 16;
        return c.fr || c.fc;
    }
    __device__ void record(uint32_t r, Item& c) const {
        const uint32_t a = c.rb + (r & 0xFFFFu), b = c.cb + (r >> 16);
        if (c.fr && bit_of(removed, a)) atomicSub(deg + b, 1);  // kcore.cpp:77-78
        if (c.fc && bit_of(removed, b)) atomicSub(deg + a, 1);  // kcore.cpp:90-91
    }
    __device__ void end(uint32_t, uint32_t, Item&) const {}
};

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
    if (!s->d_x) GS_TRY(gs_dev_alloc(ctx, (void**)&s->d_x, g->N * 4));
    if (!s->d_y) GS_TRY(gs_dev_alloc(ctx, (void**)&s->d_y, g->N * 4));
    if (!s->d_r) GS_TRY(gs_dev_alloc(ctx, (void**)&s->d_r, g->N * 4));
    pr_init_kernel<<<blocks_for(g->N, ctx), kThreads, 0, ctx->stream>>>(s->d_x, s->d_y, g->N, g->V);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_r, 0, g->N * 4, ctx->stream));
    return GS_OK;
}

gs_status pr_sweep_launch(gs_state* s) {
    gs_graph* g = s->g;
    PrOp op{s->d_x, s->d_y, g->directed};
    // algorithmic bytes per iteration: 4E + 12V (records, x, s, inv)
    return launch_sweep(g, op, GS_ALGO_PAGERANK, 4 * g->E + 12 * g->V, true);
}

gs_status pr_finalize(gs_state* s, int64_t* frontier, int* done) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    pr_finalize_kernel<<<blocks_for(g->N, ctx), kThreads, 0, ctx->stream>>>(
        s->d_x, s->d_y, s->d_r, g->d_degree, g->N, g->V, s->compat ? 1 : 0);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    *frontier = s->step;
    *done = s->step >= s->arg;
    if (*done) GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return GS_OK;
}

// ------------------------------------------------------------------- WCC ----
gs_status wcc_init(gs_state* s) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    if (!s->d_parent) GS_TRY(gs_dev_alloc(ctx, (void**)&s->d_parent, g->N * 4));
    if (!s->d_touched) GS_TRY(gs_dev_alloc(ctx, (void**)&s->d_touched, g->N));
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
    wcc_label_kernel<<<blocks_for(g->N, ctx), kThreads, 0, ctx->stream>>>(
        s->d_parent, s->d_touched, d_out, g->N, (unsigned long long*)ctx->d_scalars);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    return read_scalar(ctx, count);
}

// ---------------------------------------------------------------- k-core ----
gs_status kcore_init(gs_state* s) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    if (!s->d_deg) GS_TRY(gs_dev_alloc(ctx, (void**)&s->d_deg, g->N * 4));
    if (!s->d_kactive) GS_TRY(gs_dev_alloc(ctx, (void**)&s->d_kactive, g->N / 8));
    if (!s->d_act) GS_TRY(gs_dev_alloc(ctx, (void**)&s->d_act, g->nw));
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(s->d_deg, g->d_degree, g->N * 4, cudaMemcpyDeviceToDevice, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_kactive, 0, g->N / 8, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_act, 0, g->nw, ctx->stream));
    return GS_OK;
}

gs_status kcore_sweep_launch(gs_state* s) {
    gs_graph* g = s->g;
    KcoreOp op{s->d_deg, s->d_kactive, s->d_act};
    return launch_sweep(g, op, GS_ALGO_KCORE, 0, true);
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
