// Batched queries (sm_100a): many BFS, WCC and k-core queries per persistent
// launch.
//
// Multi-source BFS.  Up to 64 BFS roots on one graph run together with one
// bit per query in W-bit frontier words (W = 32 or 64): per vertex a pair
// {frontier, visited} and a `next` word.  A record (v0, v1) of a swept tile
// does, for all queries at once, what bfs_onepart does for one
// (bfs.cpp:138-185):
//     next[v1] |= frontier[v0] & ~visited[v1]
//     next[v0] |= frontier[v1] & ~visited[v0]     (half grid)
// and the finalize turns next into the new frontier and writes depth level+1
// for each new (vertex, query) bit (iteration_finalize, bfs.cpp:187-224)
// into the query's depth plane ([bits][N], so a warp's 32 consecutive
// vertices write one sector per query).  A
// tile is swept when its row or column window holds a frontier vertex of any
// query.  Per query the depths equal the single-root BFS bit for bit: a
// vertex's depth is its level distance, whichever query shares the sweep.
//
// Batched WCC / k-core.  Any mix of WCC and k-core queries over any set of
// resident graphs runs in one persistent launch: their runs and vertex
// words are concatenated into one work list per phase (so graphs of uneven
// size share the machine), each query keeping its own state.  The per-query
// steps are the plain ones: k-core rounds (kcore.cpp:179-217) and
// decrement sweeps (kcore.cpp:63-177), WCC hooking sweeps (wcc.cpp:177-278)
// and pointer jumping (wcc.cpp:372-390).
//
// Identical queries of one run (same graph, algorithm and argument) run
// once and share the result.
//
// Persistent launches are cooperative (every CTA resident); phases are
// separated by a grid barrier whose wait is bounded by kBarrierNs: a CTA that
// waits longer sets the error flag and every CTA returns.
//
// Autotuning.  For the BFS groups of a graph the tuner tries each candidate
// configuration once — frontier word width (32 or 64 queries per group) and
// run order (file order with 64-unit runs, or L2-blocked with 8-unit runs in
// blocks of 64 or 32 windows) — timing each launch with CUDA events per
// query, then keeps the fastest for that graph.
#include "gs_internal.cuh"
#include "gs_ops.cuh"

#include <algorithm>
#include <cstring>
#include <new>

namespace {

using namespace gsops;

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr uint64_t kBarrierNs = 4000000000ull;   // 4 s

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid-wide barrier of a cooperative launch.  bar[0] counts arrivals, bar[1]
// is the generation.  False when the wait gave up or another CTA failed.
__device__ bool grid_barrier(unsigned int* bar, int* err) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int* vgen = bar + 1;
        const unsigned int gen = *vgen;
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            const uint64_t t0 = global_ns();
            while (*vgen == gen) {
                if (*(volatile int*)err) break;
                if (global_ns() - t0 > kBarrierNs) {
                    atomicOr(err, 1);
                    break;
                }
                __nanosleep(100);
            }
        }
        __threadfence();
        ok = *(volatile int*)err == 0;
    }
    __syncthreads();
    return ok != 0;
}

// ------------------------------------------------------------ MS-BFS ----
template <class W>
struct MsArgs {
    const gs_tile_run* runs;
    const gs_unit* units;
    const uint32_t* rec;
    uint64_t R;
    uint64_t N;
    uint32_t nw;
    FvPair<W>* fv;
    W* next;
    uint8_t* depth;                  // [bits][N]: one plane per query
    uint8_t* act;                    // 2 x nw, by level parity
    unsigned long long* total;       // fresh (vertex, query) pairs per level, [256]
    W* overflow;                     // queries that reached a depth over 254
    unsigned int* bar;
    int* err;
    int* levels;
    int directed;
    const gs_pr_item* items;         // row-slice order: (row, slice, column block) items
    uint64_t n_items;
    unsigned int* tickets;           // [256]: next run of each level's sweep
    uint8_t* dead;                   // per unit: chunks with no record left to discover (ms_sweep_unit_live)
    W qmask;                         // the group's queries
    uint64_t live_pairs;             // (vertex with records, query) pairs: nonisolated x queries
};

template <class W>
__global__ void __launch_bounds__(kThreads) msbfs_kernel(MsArgs<W> a) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (int level = 1; level < 255; ++level) {
        const uint8_t* act = a.act + (level & 1) * a.nw;
        uint8_t* act_next = a.act + ((level + 1) & 1) * a.nw;
        // the flags of the next frontier start empty (last read one level ago)
        for (uint64_t w = tid; w < a.nw; w += nth) act_next[w] = 0;
        // sweep: a CTA per run (drawn from the level's ticket), a warp per
        // unit; a tile is swept when its row (or, half grid, column) window
        // holds a frontier vertex of any query (grid::bfs_mmap,
        // gstore.cpp:2671-2698)
        __shared__ unsigned long long s_run;
        auto draw = [&]() -> uint64_t {
            __syncthreads();   // every thread has read the previous draw
            if (threadIdx.x == 0) s_run = atomicAdd(a.tickets + level, 1u);
            __syncthreads();
            return s_run;
        };
        // chunks whose records all have both ends visited by every query
        // are marked, and the marked ones skipped, once at most 1/64 of the
        // (vertex with records, query) pairs are unvisited (after the peak)
        uint64_t visited = (uint64_t)popc_w(a.qmask);
        for (int l = 1; l < level; ++l) visited += __ldcg(a.total + l);
        const bool mark = a.dead && (a.live_pairs > visited ? a.live_pairs - visited : 0) * 64 <= a.live_pairs;
        for (uint64_t i = draw(); i < a.R; i = draw()) {
            const gs_tile_run run = a.runs[i];
            const uint32_t row = a.units[run.unit_beg].rc >> 16;
            const bool ar = __ldcg(act + row) != 0;
            for (uint32_t ui = run.unit_beg + warp; ui < run.unit_end; ui += kWarps) {
                const gs_unit d = a.units[ui];
                if (!ar && (a.directed || !__ldcg(act + (d.rc & 0xFFFFu)))) continue;
                if (mark) ms_sweep_unit_live<W>(d, ui, a.rec, a.fv, a.next, a.directed, lane, a.dead, true, a.qmask);
                else ms_sweep_unit<W>(d, a.rec, a.fv, a.next, a.directed, lane);
            }
        }
        if (!grid_barrier(a.bar, a.err)) return;
        // finalize: new = next & ~visited; frontier := new; visited |= new
        uint64_t local = 0;
        for (uint64_t v = tid; v < a.N; v += nth) {
            const W nx = __ldcg(a.next + v);
            const FvPair<W> s = load_fv(a.fv + v);
            W fresh = 0;
            if (nx != 0 || s.f != 0) {
                if (nx) __stcg(a.next + v, (W)0);
                fresh = nx & ~s.vis;
                store_fv(a.fv + v, fresh, s.vis | fresh);
            }
            // depth planes written per query for the warp's 32 consecutive
            // vertices at once (one sector per plane)
            const W any = warp_or(fresh);
            if (!any) continue;
            if (fresh) local += popc_w(fresh);
            if (lane == 0) {
                act_next[v >> 16] = 1;
                if (level == 254) atomicOr(a.overflow, any);
            }
            W x = any;
            while (x) {
                const int q = ffs_w(x) - 1;
                if (fresh >> q & 1) a.depth[(uint64_t)q * a.N + v] = (uint8_t)(level + 1);
                x &= x - 1;
            }
        }
        warp_add_u64(a.total + level, local);
        if (!grid_barrier(a.bar, a.err)) return;
        if (__ldcg(a.total + level) == 0) {
            if (tid == 0) *a.levels = level;
            return;
        }
    }
    if (tid == 0) *a.levels = 254;
}

// ------------------------------------------- MS-BFS over row slices ----
// The same level loop over the row-slice layout (a copy of the records with
// each tile grouped by row slice v0 >> 13 and sorted by v1 inside it; items
// are (row window, slice, 32-window column block)).  A CTA stages the
// {frontier, visited} words of its item's row slice (8,192 vertices) in
// shared memory with coalesced loads and collects the row ends' discoveries
// in a shared `next` slice, flushed once per item; only the column end
// reads global memory per record.
constexpr int kSliceThreads = 1024;
constexpr int kSliceWarps = kSliceThreads / 32;
constexpr uint32_t kSliceV = 1u << kPrSliceBits;

template <class W>
struct MsSliceOp {
    const FvPair<W>* fvs;   // shared: row slice
    W* nxs;                 // shared: row slice discoveries
    FvPair<W>* fv;
    W* next;
    int directed;
    struct Item {
        uint32_t cb;
    };
    __device__ bool begin(uint32_t, uint32_t col, Item& c) const {
        c.cb = col << 16;
        return true;
    }
    __device__ void record(uint32_t r, Item& c) const {
        const uint32_t a = r & (kSliceV - 1), b = c.cb + (r >> 16);
        const FvPair<W> sa = fvs[a], sb = load_fv(fv + b);
        const W nb = sa.f & ~sb.vis;
        if (nb) atomicOr(next + b, nb);
        if (!directed) {
            const W na = sb.f & ~sa.vis;
            if (na) atomicOr(nxs + a, na);
        }
    }
    __device__ void end(uint32_t, uint32_t, Item&) const {}
};

template <class W>
__global__ void __launch_bounds__(kSliceThreads) msbfs_slice_kernel(MsArgs<W> a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    FvPair<W>* fvs = reinterpret_cast<FvPair<W>*>(smem_raw);
    W* nxs = reinterpret_cast<W*>(smem_raw + kSliceV * sizeof(FvPair<W>));
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    const MsSliceOp<W> op{fvs, nxs, a.fv, a.next, a.directed};
    for (int level = 1; level < 255; ++level) {
        const uint8_t* act = a.act + (level & 1) * a.nw;
        uint8_t* act_next = a.act + ((level + 1) & 1) * a.nw;
        for (uint64_t w = gtid; w < a.nw; w += nth) act_next[w] = 0;
        for (uint64_t i = blockIdx.x; i < a.n_items; i += gridDim.x) {
            const gs_pr_item it = a.items[i];
            const bool ar = __ldcg(act + it.row) != 0;
            int any = ar ? 1 : 0;
            if (!ar && !a.directed)
                for (uint32_t ui = it.unit_beg + tid; ui < it.unit_end; ui += kSliceThreads)
                    any |= __ldcg(act + (a.units[ui].rc & 0xFFFFu)) != 0;
            if (!__syncthreads_or(any)) continue;
            const uint64_t base = ((uint64_t)it.row << kTileBits) + ((uint64_t)it.slice << kPrSliceBits);
            const uint4* src = reinterpret_cast<const uint4*>(a.fv + base);
            uint4* dst = reinterpret_cast<uint4*>(fvs);
            for (uint32_t k = tid; k < kSliceV * sizeof(FvPair<W>) / 16; k += kSliceThreads) dst[k] = __ldcg(src + k);
            if (!a.directed)
                for (uint32_t k = tid; k < kSliceV; k += kSliceThreads) nxs[k] = 0;
            __syncthreads();
            for (uint32_t ui = it.unit_beg + warp; ui < it.unit_end; ui += kSliceWarps) {
                const gs_unit d = a.units[ui];
                if (!ar && (a.directed || !__ldcg(act + (d.rc & 0xFFFFu)))) continue;
                sweep_unit(d, a.rec, op, lane);
            }
            __syncthreads();
            if (!a.directed)
                for (uint32_t k = tid; k < kSliceV; k += kSliceThreads)
                    if (nxs[k]) atomicOr(a.next + base + k, nxs[k]);
            __syncthreads();
        }
        if (!grid_barrier(a.bar, a.err)) return;
        uint64_t local = 0;
        for (uint64_t v = gtid; v < a.N; v += nth) {
            const W nx = __ldcg(a.next + v);
            const FvPair<W> s = load_fv(a.fv + v);
            W fresh = 0;
            if (nx != 0 || s.f != 0) {
                if (nx) __stcg(a.next + v, (W)0);
                fresh = nx & ~s.vis;
                store_fv(a.fv + v, fresh, s.vis | fresh);
            }
            // depth planes written per query for the warp's 32 consecutive
            // vertices at once (one sector per plane)
            const W any = warp_or(fresh);
            if (!any) continue;
            if (fresh) local += popc_w(fresh);
            if (lane == 0) {
                act_next[v >> 16] = 1;
                if (level == 254) atomicOr(a.overflow, any);
            }
            W x = any;
            while (x) {
                const int q = ffs_w(x) - 1;
                if (fresh >> q & 1) a.depth[(uint64_t)q * a.N + v] = (uint8_t)(level + 1);
                x &= x - 1;
            }
        }
        warp_add_u64(a.total + level, local);
        if (!grid_barrier(a.bar, a.err)) return;
        if (__ldcg(a.total + level) == 0) {
            if (gtid == 0) *a.levels = level;
            return;
        }
    }
    if (gtid == 0) *a.levels = 254;
}

// Root seeding: depth 1, frontier and visited bit of query q (bfs.cpp:70).
// (one thread: several queries may share a root)
template <class W>
__global__ void msbfs_seed_kernel(const uint64_t* roots, int n, FvPair<W>* fv, uint8_t* depth, uint64_t N,
                                  uint8_t* act1) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int q = 0; q < n; ++q) {
        const uint64_t r = roots[q];
        fv[r].f |= (W)1 << q;
        fv[r].vis |= (W)1 << q;
        depth[(uint64_t)q * N + r] = 1;
        act1[r >> 16] = 1;   // calc_part_needed (bfs.cpp:324-338); level 1 has parity 1
    }
}

// Per query and depth: vertex counts (the per-level frontier counts) of the
// planes [n_queries][N] (first V bytes of each).
__global__ void depth_histogram_kernel(const uint8_t* __restrict__ depth, uint64_t N, int n_queries, uint64_t V,
                                       unsigned long long* hist /* [n_queries][256] */) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = tid; i < V * (uint64_t)n_queries; i += nth) {
        const uint64_t q = i / V, v = i - q * V;
        const uint8_t d = depth[q * N + v];
        if (d) atomicAdd(hist + q * 256 + d, 1ull);
    }
}

// ----------------------------------------------------- WCC / k-core ----
struct BQuery {
    const gs_tile_run* runs;
    const gs_unit* units;
    const uint32_t* rec;
    uint64_t R;
    uint64_t words;              // N / 32
    uint32_t nw;
    int algo;
    int k;
    uint32_t* parent;            // WCC
    uint8_t* touched;
    int32_t* deg;                // k-core
    uint32_t* removed;
    uint8_t* act;                // 2 x nw, by iteration parity
    unsigned long long* cnt;     // [4]: changes (WCC) / removals (k-core) by iteration
    int* sweeps;
};

constexpr int kMaxBatch = 64;
constexpr int kMsCtasPerSm = 4;   // multi-source BFS launches
constexpr int kWkCtasPerSm = 8;   // WCC / k-core launches (their sweeps wait on dependent loads)

struct BatchArgs {
    BQuery* q;
    int nq;
    unsigned int* bar;
    int* err;
    unsigned int* tickets;       // [4], zero at launch
};

// Position of x among the prefix sums pre[0..n] (pre[0] = 0, x < pre[n]).
__device__ __forceinline__ int find_query(const uint64_t* pre, int n, uint64_t x) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= x) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Both phases walk only the queries still running: after each decision step
// every CTA rebuilds the same compact list (act_q) and its prefix sums of
// runs and words.  Phase B draws runs from tickets[it & 3]; phase A of
// iteration it zeroes tickets[(it + 2) & 3], last used two iterations before.
__global__ void __launch_bounds__(kThreads) wk_batch_kernel(BatchArgs a) {
    __shared__ uint64_t run_pre[kMaxBatch + 1], word_pre[kMaxBatch + 1];
    __shared__ int act_q[kMaxBatch];
    __shared__ int n_act;
    __shared__ unsigned long long done_mask, s_run;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t gwarp = (uint64_t)blockIdx.x * kWarps + warp;
    const uint64_t nwarps = (uint64_t)gridDim.x * kWarps;
    auto rebuild = [&]() {   // thread 0
        int n = 0;
        run_pre[0] = word_pre[0] = 0;
        for (int q = 0; q < a.nq; ++q) {
            if (done_mask >> q & 1) continue;
            act_q[n] = q;
            run_pre[n + 1] = run_pre[n] + a.q[q].R;
            word_pre[n + 1] = word_pre[n] + a.q[q].words;
            ++n;
        }
        n_act = n;
    };
    if (threadIdx.x == 0) {
        done_mask = 0;
        rebuild();
    }
    __syncthreads();
    for (int it = 0;; ++it) {
        const int p = it & 1;
        if (blockIdx.x == 0 && threadIdx.x == 0) a.tickets[(it + 2) & 3] = 0;
        // phase A: k-core round / WCC pointer jumping, per 32-vertex word
        for (uint64_t x = gwarp; x < word_pre[n_act]; x += nwarps) {
            const int ai = find_query(word_pre, n_act, x);
            const BQuery& q = a.q[act_q[ai]];
            const uint64_t w = x - word_pre[ai];
            const uint32_t v = (uint32_t)(w * 32 + lane);
            if (lane == 0 && w < 1) {
                q.cnt[(it + 2) & 3] = 0;
                for (uint32_t i = 0; i < q.nw; ++i) q.act[(p ^ 1) * q.nw + i] = 0;
            }
            if (q.algo == GS_ALGO_KCORE) {
                const int32_t dv = __ldcg(q.deg + v);
                const int16_t m = (int16_t)dv;           // kcore.cpp:189
                const bool gone = m < q.k && m > 0;
                if (gone) __stcg(q.deg + v, 0);
                const uint32_t bits = __ballot_sync(kFull, gone);
                if (lane == 0) {
                    __stcg(q.removed + w, bits);
                    if (bits) {
                        q.act[p * q.nw + (w >> 11)] = 1;
                        atomicAdd(q.cnt + (it & 3), (unsigned long long)__popc(bits));
                    }
                }
            } else if (it > 0) {
                const uint32_t r = find_root(q.parent, v);
                if (r != v) __stcg(q.parent + v, r);
            }
        }
        if (!grid_barrier(a.bar, a.err)) return;
        // decisions, identical in every CTA (counters are final here)
        if (threadIdx.x == 0) {
            for (int ai = 0; ai < n_act; ++ai) {
                const int qi = act_q[ai];
                const BQuery& q = a.q[qi];
                bool done;
                if (q.algo == GS_ALGO_KCORE) done = __ldcg(q.cnt + (it & 3)) == 0;
                else done = it > 0 && __ldcg(q.cnt + ((it - 1) & 3)) == 0;
                if (done) {
                    done_mask |= 1ull << qi;
                    if (blockIdx.x == 0) *q.sweeps = it;
                }
            }
            rebuild();
        }
        __syncthreads();
        if (n_act == 0) return;
        // phase B: one sweep of every query still running
        unsigned int* ticket = a.tickets + (it & 3);
        auto draw = [&]() -> uint64_t {
            __syncthreads();   // every thread has read the previous draw
            if (threadIdx.x == 0) s_run = atomicAdd(ticket, 1u);
            __syncthreads();
            return s_run;
        };
        for (uint64_t x = draw(); x < run_pre[n_act]; x = draw()) {
            const int ai = find_query(run_pre, n_act, x);
            const BQuery& q = a.q[act_q[ai]];
            const gs_tile_run run = q.runs[x - run_pre[ai]];
            if (q.algo == GS_ALGO_KCORE) {
                const KcoreOpL2 op{q.deg, q.removed, q.act + p * q.nw};
                for (uint32_t ui = run.unit_beg + warp; ui < run.unit_end; ui += kWarps)
                    sweep_unit(q.units[ui], q.rec, op, lane);
            } else {
                const WccOp op{q.parent, it == 0 ? q.touched : nullptr, q.cnt + (it & 3)};
                for (uint32_t ui = run.unit_beg + warp; ui < run.unit_end; ui += kWarps)
                    sweep_unit(q.units[ui], q.rec, op, lane);
            }
        }
        if (!grid_barrier(a.bar, a.err)) return;
    }
}

__global__ void wk_init_kernel(uint32_t* parent, uint64_t N) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = tid; v < N; v += nth) parent[v] = (uint32_t)v;
}

__global__ void wk_labels_kernel(const uint32_t* parent, const uint8_t* touched, uint32_t* out, uint64_t V,
                                 unsigned long long* count) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    uint64_t local = 0;
    for (uint64_t v = tid; v < V; v += nth) {
        if (!touched[v]) {
            out[v] = 0xFFFFFFFFu;     // invalid_cid, wcc.cpp:54
            continue;
        }
        uint32_t r = parent[v];
        while (parent[r] != r) r = parent[r];
        out[v] = r;
        local += r == v;
    }
    warp_add_u64(count, local);
}

__global__ void wk_count_nonzero_kernel(const int32_t* deg, uint64_t V, unsigned long long* out) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    uint64_t local = 0;
    for (uint64_t v = tid; v < V; v += nth) local += deg[v] != 0;
    warp_add_u64(out, local);
}

inline uint32_t blocks_for(uint64_t n, const gs_ctx* ctx) {
    const uint64_t b = (n + kThreads - 1) / kThreads;
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(b, gs_grid_size(ctx, 16)));
}

}  // namespace

// ================================================================ host ====
struct gs_batch_query {
    gs_graph* g = nullptr;
    gs_algo algo = GS_ALGO_BFS;
    int64_t arg = 0;
    gs_status status = GS_OK;
    bool ran = false;
    int group = -1;          // BFS: group index, bit = lane
    int lane = 0;
    int leader = -1;         // an identical query of the same run answers this one
    int64_t sweeps = 0;
    // WCC / k-core state
    uint32_t* parent = nullptr;
    uint8_t* touched = nullptr;
    int32_t* deg = nullptr;
    uint32_t* removed = nullptr;
    uint8_t* act = nullptr;
    unsigned long long* cnt = nullptr;
    // PageRank, and WCC on graphs whose plain WCC hooks a sample first: a
    // plain state (the query runs through gs_run)
    gs_state* pr = nullptr;
};

struct gs_bfs_group {
    gs_graph* g = nullptr;
    int bits = 64;
    int order = 1;                     // 0 file order, 1 / 2: 64- / 32-window blocks, 3 row slices
    std::vector<int> queries;
    uint8_t* depth = nullptr;          // [bits][N]: one plane per query
    int levels = 0;
    unsigned long long overflow = 0;
    std::vector<uint64_t> hist;        // [queries][256], filled on demand
};

struct gs_batch {
    gs_ctx* ctx = nullptr;
    std::vector<gs_batch_query> q;
    std::vector<gs_bfs_group> groups;
    size_t first_new = 0;              // queries before this index have run
    uint64_t launches = 0;
    double kernel_ms = 0.0;
    // scratch
    void* d_scratch = nullptr;
    size_t scratch_bytes = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
};

// Autotuner record of one graph: per candidate, time per query of its runs.
// (bits 32 / 64) x (file order / 64-window blocks / 32-window blocks / row slices)
constexpr int kOrders = 4;
constexpr int kCandidates = 2 * kOrders;
struct gs_tune {
    double ms_per_query[kCandidates] = {0, 0, 0, 0, 0, 0, 0, 0};
    int samples[kCandidates] = {0, 0, 0, 0, 0, 0, 0, 0};
};

namespace {

std::vector<std::pair<const gs_graph*, gs_tune>> g_tune;   // per graph (single-threaded contexts)

gs_tune& tune_of(const gs_graph* g) {
    for (auto& t : g_tune)
        if (t.first == g) return t.second;
    g_tune.emplace_back(g, gs_tune());
    return g_tune.back().second;
}

// Candidate c: word width 32 (c < kOrders) or 64 bits; order c % kOrders:
// file order (64-unit runs), 64-window or 32-window blocks (8-unit runs), or
// the row-slice layout (msbfs_slice_kernel).  Each is tried once, then the
// fastest per query is kept.
int pick_candidate(const gs_tune& t) {
    for (int c = kCandidates - 1; c >= 0; --c)
        if (t.samples[c] == 0) return c;
    int best = kCandidates - 1;
    for (int c = 0; c < kCandidates; ++c)
        if (t.ms_per_query[c] < t.ms_per_query[best]) best = c;
    return best;
}

gs_status scratch(gs_batch* b, size_t bytes, void** out) {
    if (bytes > b->scratch_bytes) {
        gs_pool_put(b->ctx, b->d_scratch, b->scratch_bytes);
        b->d_scratch = nullptr;
        b->scratch_bytes = 0;
        GS_TRY(gs_pool_get(b->ctx, bytes, &b->d_scratch));
        b->scratch_bytes = bytes;
    }
    *out = b->d_scratch;
    return GS_OK;
}

// Resident CTAs of a cooperative launch: every SM's share, at most `cap`
// per SM (fewer CTAs make the grid barriers cheaper; latency-bound sweeps
// want more warps).
int coop_grid(gs_ctx* ctx, const void* kernel, int cap) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return ctx->num_sms * std::min(per_sm, cap);
}

// One multi-source BFS launch over the queries of group `gi`.
template <class W>
gs_status run_bfs_group(gs_batch* b, gs_bfs_group& grp) {
    gs_ctx* ctx = b->ctx;
    gs_graph* g = grp.g;
    constexpr int kBits = sizeof(W) * 8;
    const int n = (int)grp.queries.size();
    const uint64_t N = g->N;
    // device scratch: fv (N pairs), next (N words), act (2 nw), totals, bar, err, levels, overflow, roots
    const size_t fv_b = N * sizeof(FvPair<W>), nx_b = N * sizeof(W);
    const size_t act_b = (2 * (size_t)g->nw + 255) & ~(size_t)255;
    const size_t small_b = 256 * 8 + 64 + 8 * kMaxBatch + 64 + 256 * 4;
    const size_t dead_b = (g->U + 4 + 255) & ~(size_t)255;   // a byte per unit, whole words
    void* base = nullptr;
    GS_TRY(scratch(b, fv_b + nx_b + act_b + small_b + dead_b, &base));
    char* p = (char*)base;
    FvPair<W>* fv = (FvPair<W>*)p;
    W* next = (W*)(p + fv_b);
    uint8_t* act = (uint8_t*)(p + fv_b + nx_b);
    char* small = p + fv_b + nx_b + act_b;
    unsigned long long* total = (unsigned long long*)small;
    unsigned int* bar = (unsigned int*)(small + 256 * 8);
    int* err = (int*)(small + 256 * 8 + 16);
    int* levels = (int*)(small + 256 * 8 + 32);
    W* overflow = (W*)(small + 256 * 8 + 48);
    uint64_t* roots = (uint64_t*)(small + 256 * 8 + 64);
    unsigned int* tickets = (unsigned int*)(small + 256 * 8 + 64 + 8 * kMaxBatch + 64);
    uint8_t* dead = (uint8_t*)(small + small_b);
    GS_TRY(gs_pool_get(ctx, N * kBits, (void**)&grp.depth));
    GS_TRY(gs_graph_nonisolated(g));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(base, 0, fv_b + nx_b + act_b + small_b + dead_b, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(grp.depth, 0, N * n, ctx->stream));   // the queries' planes
    std::vector<uint64_t> h_roots(n);
    for (int i = 0; i < n; ++i) h_roots[i] = (uint64_t)b->q[grp.queries[i]].arg;
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(roots, h_roots.data(), n * 8, cudaMemcpyHostToDevice, ctx->stream));
    msbfs_seed_kernel<W><<<1, 1, 0, ctx->stream>>>(roots, n, fv, grp.depth, N, act + g->nw);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    const gs_tile_run* runs = grp.order == 1 ? g->d_runs_blk : grp.order == 2 ? g->d_runs_blk2 : g->d_runs;
    const gs_unit* units = grp.order == 1 ? g->d_units_blk : grp.order == 2 ? g->d_units_blk2 : g->d_units;
    const uint64_t n_runs = grp.order == 1 ? g->R_blk : grp.order == 2 ? g->R_blk2 : g->R;
    MsArgs<W> a{runs,
                units,
                g->d_rec,
                n_runs,
                N,
                g->nw,
                fv,
                next,
                grp.depth,
                act,
                total,
                overflow,
                bar,
                err,
                levels,
                g->directed,
                nullptr,
                0,
                tickets,
                g->nonisolated_known ? dead : nullptr,
                n >= kBits ? (W)~(W)0 : (W)(((W)1 << n) - 1),
                g->nonisolated * (uint64_t)n};
    void* args[] = {&a};
    GS_CHECK_CUDA(ctx, cudaEventRecord(b->e0, ctx->stream));
    if (grp.order == 3) {
        a.units = g->pr.d_units;
        a.rec = g->pr.d_rec;
        a.items = g->pr.d_items;
        a.n_items = g->pr.n_items;
        const int smem = (int)(kSliceV * (sizeof(FvPair<W>) + sizeof(W)));
        GS_CHECK_CUDA(ctx, cudaFuncSetAttribute((const void*)msbfs_slice_kernel<W>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, msbfs_slice_kernel<W>, kSliceThreads, smem) !=
                cudaSuccess ||
            per_sm < 1)
            per_sm = 1;
        GS_CHECK_CUDA(ctx, cudaLaunchCooperativeKernel((const void*)msbfs_slice_kernel<W>,
                                                       dim3(ctx->num_sms * per_sm), dim3(kSliceThreads), args, smem,
                                                       ctx->stream));
    } else {
        const int grid = coop_grid(ctx, (const void*)msbfs_kernel<W>, kMsCtasPerSm);
        GS_CHECK_CUDA(ctx, cudaLaunchCooperativeKernel((const void*)msbfs_kernel<W>, dim3(grid), dim3(kThreads), args,
                                                       0, ctx->stream));
    }
    GS_CHECK_CUDA(ctx, cudaEventRecord(b->e1, ctx->stream));
    ctx->launches += 1;
    b->launches += 1;
    int h_err = 0, h_levels = 0;
    W h_over = 0;
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(&h_err, err, 4, cudaMemcpyDeviceToHost, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(&h_levels, levels, 4, cudaMemcpyDeviceToHost, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(&h_over, overflow, sizeof(W), cudaMemcpyDeviceToHost, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b->e0, b->e1);
    b->kernel_ms += ms;
    gs_tune& t = tune_of(g);
    const int c = (kBits == 64 ? kOrders : 0) + grp.order;
    t.ms_per_query[c] = (t.ms_per_query[c] * t.samples[c] + ms / n) / (t.samples[c] + 1);
    t.samples[c] += 1;
    if (h_err) return gs_fail(ctx, GS_ERR_TIMEOUT, "batched BFS: a grid barrier wait gave up");
    grp.levels = h_levels;
    grp.overflow = (unsigned long long)h_over;
    for (int i = 0; i < n; ++i) {
        gs_batch_query& q = b->q[grp.queries[i]];
        q.ran = true;
        q.sweeps = h_levels;
        if (grp.overflow >> i & 1) q.status = GS_ERR_RANGE;
    }
    return GS_OK;
}

gs_status run_bfs_queries(gs_batch* b, std::vector<int>& idx) {
    // group by graph, in order of first appearance
    std::vector<gs_graph*> graphs;
    for (int i : idx)
        if (std::find(graphs.begin(), graphs.end(), b->q[i].g) == graphs.end()) graphs.push_back(b->q[i].g);
    for (gs_graph* g : graphs) {
        std::vector<int> mine;
        for (int i : idx)
            if (b->q[i].g == g) mine.push_back(i);
        const int cand = pick_candidate(tune_of(g));
        const int bits = cand >= kOrders ? 64 : 32;
        GS_TRY(gs_ensure_blocked(g));
        const int order = g->d_runs_blk ? cand % kOrders : 0;
        if (order == 3 && !g->pr.built) GS_TRY(pr_layout_build(g));
        for (size_t s = 0; s < mine.size(); s += bits) {
            gs_bfs_group grp;
            grp.g = g;
            grp.bits = bits;
            grp.order = order;
            for (size_t k = s; k < std::min(mine.size(), s + bits); ++k) {
                grp.queries.push_back(mine[k]);
                b->q[mine[k]].group = (int)b->groups.size();
                b->q[mine[k]].lane = (int)(k - s);
            }
            b->groups.push_back(grp);
            gs_bfs_group& gg = b->groups.back();
            GS_TRY(bits == 64 ? run_bfs_group<unsigned long long>(b, gg) : run_bfs_group<uint32_t>(b, gg));
        }
    }
    return GS_OK;
}

gs_status run_wk_queries(gs_batch* b, std::vector<int>& idx) {
    gs_ctx* ctx = b->ctx;
    for (size_t s = 0; s < idx.size(); s += kMaxBatch) {
        const size_t e = std::min(idx.size(), s + kMaxBatch);
        std::vector<BQuery> dq;
        for (size_t k = s; k < e; ++k) {
            gs_batch_query& q = b->q[idx[k]];
            gs_graph* g = q.g;
            const uint64_t N = g->N;
            GS_TRY(gs_pool_get(ctx, 4 * sizeof(unsigned long long), (void**)&q.cnt));
            GS_CHECK_CUDA(ctx, cudaMemsetAsync(q.cnt, 0, 4 * sizeof(unsigned long long), ctx->stream));
            GS_TRY(gs_pool_get(ctx, 2 * (size_t)g->nw, (void**)&q.act));
            GS_CHECK_CUDA(ctx, cudaMemsetAsync(q.act, 0, 2 * (size_t)g->nw, ctx->stream));
            if (q.algo == GS_ALGO_WCC) {
                GS_TRY(gs_pool_get(ctx, N * 4, (void**)&q.parent));
                GS_TRY(gs_pool_get(ctx, N, (void**)&q.touched));
                wk_init_kernel<<<blocks_for(N, ctx), kThreads, 0, ctx->stream>>>(q.parent, N);
                ctx->launches++;
                GS_CHECK_CUDA(ctx, cudaMemsetAsync(q.touched, 0, N, ctx->stream));
            } else {
                GS_TRY(gs_pool_get(ctx, N * 4, (void**)&q.deg));
                GS_TRY(gs_pool_get(ctx, N / 8, (void**)&q.removed));
                GS_CHECK_CUDA(ctx, cudaMemcpyAsync(q.deg, g->d_degree, N * 4, cudaMemcpyDeviceToDevice, ctx->stream));
            }
            BQuery d;
            std::memset(&d, 0, sizeof(d));
            GS_TRY(gs_ensure_blocked(g));
            d.runs = g->d_runs_blk ? g->d_runs_blk : g->d_runs;
            d.units = g->d_runs_blk ? g->d_units_blk : g->d_units;
            d.rec = g->d_rec;
            d.R = g->d_runs_blk ? g->R_blk : g->R;
            d.words = N / 32;
            d.nw = g->nw;
            d.algo = (int)q.algo;
            d.k = (int)q.arg;
            d.parent = q.parent;
            d.touched = q.touched;
            d.deg = q.deg;
            d.removed = q.removed;
            d.act = q.act;
            d.cnt = q.cnt;
            dq.push_back(d);
        }
        const int nq = (int)dq.size();
        void* base = nullptr;
        const size_t qb = ((nq * sizeof(BQuery)) + 255) & ~(size_t)255;
        GS_TRY(scratch(b, qb + 256 + nq * sizeof(int), &base));
        BQuery* d_q = (BQuery*)base;
        unsigned int* bar = (unsigned int*)((char*)base + qb);
        int* err = (int*)((char*)base + qb + 16);
        unsigned int* tickets = (unsigned int*)((char*)base + qb + 32);   // 4, zeroed with bar and err
        int* sweeps = (int*)((char*)base + qb + 256);
        for (int k = 0; k < nq; ++k) dq[k].sweeps = sweeps + k;
        GS_CHECK_CUDA(ctx, cudaMemsetAsync((char*)base + qb, 0, 256 + nq * sizeof(int), ctx->stream));
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(d_q, dq.data(), nq * sizeof(BQuery), cudaMemcpyHostToDevice, ctx->stream));
        BatchArgs a{d_q, nq, bar, err, tickets};
        void* args[] = {&a};
        const int grid = coop_grid(ctx, (const void*)wk_batch_kernel, kWkCtasPerSm);
        GS_CHECK_CUDA(ctx, cudaEventRecord(b->e0, ctx->stream));
        GS_CHECK_CUDA(ctx, cudaLaunchCooperativeKernel((const void*)wk_batch_kernel, dim3(grid), dim3(kThreads), args,
                                                       0, ctx->stream));
        ctx->launches += 1;
        b->launches += 1;
        for (const BQuery& d : dq) {   // WCC post-processing, like the label kernels (not a batch launch)
            if (d.algo != GS_ALGO_WCC) continue;
            wcc_mark_touched<<<blocks_for(d.words * 32, ctx), kThreads, 0, ctx->stream>>>(d.parent, d.touched,
                                                                                         d.words * 32);
            ctx->launches += 1;
        }
        GS_CHECK_CUDA(ctx, cudaEventRecord(b->e1, ctx->stream));
        std::vector<int> h_sweeps(nq);
        int h_err = 0;
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(h_sweeps.data(), sweeps, nq * sizeof(int), cudaMemcpyDeviceToHost,
                                           ctx->stream));
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(&h_err, err, 4, cudaMemcpyDeviceToHost, ctx->stream));
        GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, b->e0, b->e1);
        b->kernel_ms += ms;
        if (h_err) return gs_fail(ctx, GS_ERR_TIMEOUT, "batched WCC/k-core: a grid barrier wait gave up");
        for (int k = 0; k < nq; ++k) {
            gs_batch_query& q = b->q[idx[s + k]];
            q.ran = true;
            q.sweeps = h_sweeps[k];
        }
    }
    return GS_OK;
}

void free_query(gs_ctx* ctx, gs_batch_query& q) {
    if (q.g) {
        const uint64_t N = q.g->N;
        gs_pool_put(ctx, q.parent, N * 4);
        gs_pool_put(ctx, q.touched, N);
        gs_pool_put(ctx, q.deg, N * 4);
        gs_pool_put(ctx, q.removed, N / 8);
        gs_pool_put(ctx, q.act, 2 * (size_t)q.g->nw);
        gs_pool_put(ctx, q.cnt, 4 * sizeof(unsigned long long));
    }
    q.parent = nullptr;
    q.touched = nullptr;
    q.deg = nullptr;
    q.removed = nullptr;
    q.act = nullptr;
    q.cnt = nullptr;
    if (q.pr) gs_state_free(q.pr);
    q.pr = nullptr;
}

gs_status query_of(gs_batch* b, int id, gs_batch_query** out) {
    if (!b || id < 0 || (size_t)id >= b->q.size()) return GS_ERR_ARG;
    if (b->q[id].leader >= 0) id = b->q[id].leader;
    gs_batch_query& q = b->q[id];
    if (!q.ran) return gs_fail(b->ctx, GS_ERR_STATE, "query has not run (call gs_batch_run)");
    if (q.status != GS_OK) return gs_fail(b->ctx, q.status, "query failed");
    *out = &q;
    return GS_OK;
}

}  // namespace

extern "C" {

gs_status gs_batch_create(gs_ctx* ctx, gs_batch** out) {
    if (!ctx || !out) return GS_ERR_ARG;
    gs_batch* b = new (std::nothrow) gs_batch();
    if (!b) return GS_ERR_OOM;
    b->ctx = ctx;
    if (cudaEventCreate(&b->e0) != cudaSuccess || cudaEventCreate(&b->e1) != cudaSuccess) {
        delete b;
        return gs_fail(ctx, GS_ERR_CUDA, "cudaEventCreate");
    }
    *out = b;
    return GS_OK;
}

gs_status gs_batch_add(gs_batch* b, gs_graph* g, gs_algo algo, int64_t arg, int* query_id) {
    if (!b || !g || !query_id) return GS_ERR_ARG;
    gs_ctx* ctx = b->ctx;
    if (g->ctx != ctx) return gs_fail(ctx, GS_ERR_ARG, "graph belongs to another context");
    if (g->stream) return gs_fail(ctx, GS_ERR_UNSUPPORTED, "batched queries need graphs resident in HBM");
    if (algo == GS_ALGO_BFS && (arg < 0 || (uint64_t)arg >= g->V)) return gs_fail(ctx, GS_ERR_ARG, "BFS root out of range");
    if (algo == GS_ALGO_KCORE && g->directed)
        return gs_fail(ctx, GS_ERR_UNSUPPORTED, "Kcore not applicable for directed graphs");
    if (algo == GS_ALGO_PAGERANK && arg < 1) return gs_fail(ctx, GS_ERR_ARG, "iterations < 1");
    if (algo != GS_ALGO_BFS && algo != GS_ALGO_WCC && algo != GS_ALGO_KCORE && algo != GS_ALGO_PAGERANK)
        return GS_ERR_ARG;
    gs_batch_query q;
    q.g = g;
    q.algo = algo;
    q.arg = arg;
    b->q.push_back(q);
    *query_id = (int)b->q.size() - 1;
    return GS_OK;
}

gs_status gs_batch_run(gs_batch* b) {
    if (!b) return GS_ERR_ARG;
    std::vector<int> bfs, wk, pr;
    for (size_t i = b->first_new; i < b->q.size(); ++i) {
        // identical queries (graph, algorithm, argument) run once
        gs_batch_query& qi = b->q[i];
        for (size_t j = b->first_new; j < i; ++j) {
            const gs_batch_query& qj = b->q[j];
            if (qj.leader < 0 && qj.g == qi.g && qj.algo == qi.algo && (qi.algo == GS_ALGO_WCC || qj.arg == qi.arg)) {
                qi.leader = (int)j;
                break;
            }
        }
        if (qi.leader >= 0) continue;
        switch (b->q[i].algo) {
            case GS_ALGO_BFS: bfs.push_back((int)i); break;
            case GS_ALGO_WCC:
                // the plain WCC's sampled pass (bitmap in shared memory, L1
                // reads) beats the persistent kernel's one hooking sweep
                if (gs_wcc_sample_shift(qi.g) > 0) pr.push_back((int)i);
                else wk.push_back((int)i);
                break;
            case GS_ALGO_KCORE: wk.push_back((int)i); break;
            default: pr.push_back((int)i); break;
        }
    }
    b->first_new = b->q.size();
    GS_TRY(run_bfs_queries(b, bfs));
    GS_TRY(run_wk_queries(b, wk));
    for (int i : pr) {
        gs_batch_query& q = b->q[i];
        GS_TRY(gs_state_create(q.g, q.algo, q.arg, &q.pr));
        int64_t steps = 0;
        GS_TRY(gs_run(q.pr, &steps));
        q.sweeps = steps;
        q.ran = true;
        b->launches += 1;   // one plain run (its sweeps and finalizes)
    }
    return GS_OK;
}

gs_status gs_batch_download(gs_batch* b, int query_id, int what, void* host_dst, uint64_t bytes) {
    gs_batch_query* q = nullptr;
    GS_TRY(query_of(b, query_id, &q));
    if (!host_dst) return GS_ERR_ARG;
    gs_ctx* ctx = b->ctx;
    gs_graph* g = q->g;
    if (q->pr) return gs_download(q->pr, what, host_dst, bytes);
    const uint64_t need = q->algo == GS_ALGO_BFS ? g->V : g->V * 4;
    if (bytes < need) return gs_fail(ctx, GS_ERR_ARG, "destination too small: need " + std::to_string(need));
    void* tmp = nullptr;
    GS_TRY(scratch(b, g->V * 4 + 16, &tmp));
    const void* src = nullptr;
    if (q->algo == GS_ALGO_BFS) {
        const gs_bfs_group& grp = b->groups[q->group];
        src = grp.depth + (size_t)q->lane * g->N;   // the query's depth plane
    } else if (q->algo == GS_ALGO_WCC) {
        wk_labels_kernel<<<blocks_for(g->V, ctx), kThreads, 0, ctx->stream>>>(q->parent, q->touched, (uint32_t*)tmp,
                                                                              g->V, (unsigned long long*)ctx->d_scalars);
        ctx->launches++;
        src = tmp;
    } else {
        src = q->deg;
    }
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(host_dst, src, need, cudaMemcpyDeviceToHost, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return GS_OK;
}

gs_status gs_batch_result_count(gs_batch* b, int query_id, uint64_t* count) {
    gs_batch_query* q = nullptr;
    GS_TRY(query_of(b, query_id, &q));
    if (!count) return GS_ERR_ARG;
    gs_ctx* ctx = b->ctx;
    gs_graph* g = q->g;
    if (q->pr) return gs_result_count(q->pr, count);
    if (q->algo == GS_ALGO_BFS) {
        GS_TRY(gs_batch_bfs_levels(b, query_id, nullptr, 0, nullptr));
        const uint64_t* h = b->groups[q->group].hist.data() + (size_t)q->lane * 256;
        uint64_t s = 0;
        for (int d = 1; d < 256; ++d) s += h[d];   // reached vertices (depth != 0)
        *count = s;
        return GS_OK;
    }
    unsigned long long* d = (unsigned long long*)ctx->d_scalars;
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(d, 0, 8, ctx->stream));
    if (q->algo == GS_ALGO_WCC) {
        void* tmp = nullptr;
        GS_TRY(scratch(b, g->V * 4 + 16, &tmp));
        wk_labels_kernel<<<blocks_for(g->V, ctx), kThreads, 0, ctx->stream>>>(q->parent, q->touched, (uint32_t*)tmp,
                                                                              g->V, d);
    } else {
        wk_count_nonzero_kernel<<<blocks_for(g->V, ctx), kThreads, 0, ctx->stream>>>(q->deg, g->V, d);
    }
    ctx->launches++;
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->h_scalars, d, 8, cudaMemcpyDeviceToHost, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *count = ctx->h_scalars[0];
    return GS_OK;
}

gs_status gs_batch_bfs_levels(gs_batch* b, int query_id, uint64_t* level_counts, int max_levels, int* n_levels) {
    gs_batch_query* q = nullptr;
    GS_TRY(query_of(b, query_id, &q));
    if (q->algo != GS_ALGO_BFS) return gs_fail(b->ctx, GS_ERR_ARG, "not a BFS query");
    gs_ctx* ctx = b->ctx;
    gs_bfs_group& grp = b->groups[q->group];
    if (grp.hist.empty()) {
        const int n = (int)grp.queries.size();
        void* tmp = nullptr;
        GS_TRY(scratch(b, (size_t)n * 256 * 8, &tmp));
        GS_CHECK_CUDA(ctx, cudaMemsetAsync(tmp, 0, (size_t)n * 256 * 8, ctx->stream));
        depth_histogram_kernel<<<blocks_for(grp.g->V * n, ctx), kThreads, 0, ctx->stream>>>(
            grp.depth, grp.g->N, n, grp.g->V, (unsigned long long*)tmp);
        ctx->launches++;
        GS_CHECK_CUDA(ctx, cudaGetLastError());
        grp.hist.resize((size_t)n * 256);
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(grp.hist.data(), tmp, (size_t)n * 256 * 8, cudaMemcpyDeviceToHost,
                                           ctx->stream));
        GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    // level L's count = vertices at depth L + 1 (iteration_finalize's frontier
    // count); the last level found nothing
    if (!level_counts && !n_levels) return GS_OK;
    const uint64_t* h = grp.hist.data() + (size_t)q->lane * 256;
    int last = 1;
    for (int d = 2; d < 256; ++d)
        if (h[d]) last = d;
    const int n = last;   // levels 1..last-1 found vertices, level `last` found none
    if (level_counts)
        for (int l = 0; l < n && l < max_levels; ++l) level_counts[l] = l + 2 < 256 ? h[l + 2] : 0;
    if (n_levels) *n_levels = n;
    return GS_OK;
}

gs_status gs_batch_stats(const gs_batch* b, uint64_t* launches, double* kernel_ms) {
    if (!b) return GS_ERR_ARG;
    if (launches) *launches = b->launches;
    if (kernel_ms) *kernel_ms = b->kernel_ms;
    return GS_OK;
}

gs_status gs_batch_free(gs_batch* b) {
    if (!b) return GS_OK;
    cudaStreamSynchronize(b->ctx->stream);
    for (auto& q : b->q) free_query(b->ctx, q);
    for (auto& grp : b->groups) gs_pool_put(b->ctx, grp.depth, grp.g->N * grp.bits);
    gs_pool_put(b->ctx, b->d_scratch, b->scratch_bytes);
    if (b->e0) cudaEventDestroy(b->e0);
    if (b->e1) cudaEventDestroy(b->e1);
    delete b;
    return GS_OK;
}

}  // extern "C"
