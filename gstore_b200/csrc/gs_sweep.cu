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
#include <cstdlib>

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

// WCC hooking sweep of a resident graph (wcc.cpp:177-278, the rule of
// WccOp) over a list of single-row runs, in two forms:
//   * sampled (shift > 0): a warp hooks only every 2^shift-th 16-byte group
//     (four records) of its unit, about 1/2^(shift-1) of the record sectors.
//     It only builds trees early; which records it picks changes no result.
//   * full (shift == 0): every record; with `giant` (the bitmap of the
//     largest tree after the sampled pass), a record whose two ends are both
//     in it joins nothing new and is skipped.  The run's row window of that
//     bitmap (8 KB) is staged in shared memory, since row ends are scattered
//     inside a tile; column ends come sorted and are read through L1.
// The records that need their parents looked at go to a per-warp queue in
// shared memory and are hooked 32 at a time, one per lane, so the few left
// after the bitmap test do not run their dependent loads on a lane or two
// of an otherwise idle warp.  The queue carries over units and runs and is
// emptied before the CTA leaves.
constexpr uint32_t kWindowWords = (1u << kTileBits) / 32;
constexpr int kWccHookCtasPerSm = 6;
__global__ void __launch_bounds__(kThreads, kWccHookCtasPerSm) wcc_hook_runs(const gs_tile_run* __restrict__ runs, uint64_t n_runs,
                                                          const gs_unit* __restrict__ units,
                                                          const uint32_t* __restrict__ rec, uint32_t* parent,
                                                          uint8_t* touched, const uint32_t* __restrict__ giant,
                                                          unsigned long long* changes, uint32_t shift,
                                                          unsigned int* ticket) {
    constexpr uint32_t kWarps = kThreads / 32;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    __shared__ unsigned long long s_run;
    __shared__ __align__(16) uint32_t s_row[kWindowWords];
    __shared__ uint2 s_q[kWarps][64];
    uint2* q = s_q[warp];
    uint32_t qn = 0;   // warp-uniform queue length (< 32 between pushes)
    uint32_t staged = ~0u, unresolved = 0;
    auto advance = [&]() -> uint64_t {
        __syncthreads();   // every thread has read the previous draw and is done with s_row
        if (threadIdx.x == 0) s_run = atomicAdd(ticket, 1u);
        __syncthreads();
        return s_run;
    };
    auto hook_pair = [&](uint32_t a, uint32_t b) {
        if (__ldcg(parent + a) == __ldcg(parent + b)) return;   // one tree already
        if (!gsops::hook(parent, a, b)) unresolved += 1;
    };
    // warp-collective: queue (a, b) where need is set; hook 32 once 32 wait
    auto push = [&](bool need, uint32_t a, uint32_t b) {
        const uint32_t bal = __ballot_sync(kFull, need);
        if (need) q[qn + __popc(bal & lt)] = make_uint2(a, b);
        qn += __popc(bal);
        if (qn >= 32) {
            __syncwarp();
            const uint2 mine = q[lane];
            const uint2 rest = lane + 32 < qn ? q[lane + 32] : make_uint2(0, 0);
            __syncwarp();
            if (lane + 32 < qn) q[lane] = rest;
            qn -= 32;
            hook_pair(mine.x, mine.y);
            __syncwarp();
        }
    };
    for (uint64_t i = advance(); i < n_runs; i = advance()) {
        const uint32_t ub = runs[i].unit_beg, ue = runs[i].unit_end;
        if (ub >= ue) continue;
        const uint32_t row = units[ub].rc >> 16;
        if (giant && row != staged) {
            const uint4* src = reinterpret_cast<const uint4*>(giant + (uint64_t)row * kWindowWords);
            for (uint32_t k = threadIdx.x; k < kWindowWords / 4; k += kThreads)
                reinterpret_cast<uint4*>(s_row)[k] = __ldg(src + k);
            staged = row;
            __syncthreads();
        }
        const uint32_t rb = row << kTileBits;
        for (uint32_t ui = ub + warp; ui < ue; ui += kWarps) {
            const gs_unit d = units[ui];
            const uint32_t cb = (d.rc & 0xFFFFu) << kTileBits;
            const uint32_t* gcol = giant ? giant + (cb >> 5) : nullptr;
            // does record r (valid on this lane) need its parents looked at?
            auto need = [&](bool valid, uint32_t r) -> bool {
                if (!valid) return false;
                const uint32_t al = r & 0xFFFFu, bl = r >> 16;
                if (touched && al + rb == bl + cb) touched[al + rb] = 1;   // wcc.cpp:203-217 (self-loop)
                if (!giant) return true;
                return !((s_row[al >> 5] >> (al & 31)) & (__ldg(gcol + (bl >> 5)) >> (bl & 31)) & 1u);
            };
            auto visit = [&](bool valid, uint32_t r) {
                push(need(valid, r), rb + (r & 0xFFFFu), cb + (r >> 16));
            };
            const uint64_t b = d.rec_beg, e = d.rec_beg + d.n;
            uint64_t ab = (b + 3) & ~3ull;
            if (ab > e) ab = e;
            uint64_t ae = e & ~3ull;
            if (ae < ab) ae = ab;
            if (shift == 0) {
                visit(b + lane < ab, b + lane < ab ? __ldcs(rec + b + lane) : 0u);
                visit(ae + lane < e, ae + lane < e ? __ldcs(rec + ae + lane) : 0u);
            }
            const uint4* r4 = reinterpret_cast<const uint4*>(rec + ab);
            const uint32_t n4 = (uint32_t)((ae - ab) >> 2);
            const uint32_t stride = 32u << shift, off = lane << shift;
            const uint4 z = make_uint4(0, 0, 0, 0);
            uint4 g = off < n4 ? load_stream(r4 + off) : z;
            for (uint32_t k0 = 0; k0 < n4; k0 += stride) {   // warp-uniform
                const bool valid = k0 + off < n4;
                const uint32_t kn = k0 + stride + off;
                const uint4 gn = kn < n4 ? load_stream(r4 + kn) : z;   // next group in flight
                const bool n0 = need(valid, g.x), n1 = need(valid, g.y), n2 = need(valid, g.z),
                           n3 = need(valid, g.w);
                if (__any_sync(kFull, n0 | n1 | n2 | n3)) {
                    push(n0, rb + (g.x & 0xFFFFu), cb + (g.x >> 16));
                    push(n1, rb + (g.y & 0xFFFFu), cb + (g.y >> 16));
                    push(n2, rb + (g.z & 0xFFFFu), cb + (g.z >> 16));
                    push(n3, rb + (g.w & 0xFFFFu), cb + (g.w >> 16));
                }
                g = gn;
            }
        }
    }
    __syncwarp();
    if (lane < qn) {
        const uint2 mine = q[lane];
        hook_pair(mine.x, mine.y);
    }
    if (changes) warp_add_u64(changes, unresolved);
    if (threadIdx.x == 0 && atomicAdd(ticket + 1, 1u) == gridDim.x - 1) {
        atomicExch(ticket, 0u);   // every CTA has drawn its last ticket
        atomicExch(ticket + 1, 0u);
    }
}

// Sweeps the whole resident graph, or, during a streamed sweep, the runs of
// the segment the graph points at.  timed = false leaves the kernel timer to
// the caller (a phase of several launches timed as one).
template <class Op>
gs_status launch_sweep(gs_graph* g, const Op& op, int algo, uint64_t bytes, bool blocked = false,
                       bool timed = true) {
    gs_ctx* ctx = g->ctx;
    const gs_seg_run* seg = g->seg.list;
    if (blocked && !seg) GS_TRY(gs_ensure_blocked(g));
    blocked = blocked && !seg && g->d_runs_blk;
    const uint64_t n = seg ? g->seg.n : (blocked ? g->R_blk : g->R);
    const uint32_t* rec = seg ? g->seg.buf : g->d_rec;
    if (n == 0) return GS_OK;
    const uint32_t grid = (uint32_t)std::min<uint64_t>(n, gs_grid_size(ctx, 8));
    if (timed) gs_timer_begin(ctx);
    sweep_runs<Op><<<grid, kThreads, 0, ctx->stream>>>(blocked ? g->d_runs_blk : g->d_runs, n,
                                                        blocked ? g->d_units_blk : g->d_units, rec, seg, op,
                                                        ctx->d_ticket);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    if (timed) gs_timer_end(ctx, algo, seg ? 0 : bytes);
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
    uint32_t known = ~0u, first;
    for (uint64_t v = tid; v < N; v += nth) {
        const uint32_t r = find_root_known(parent, (uint32_t)v, known, &first);
        if (r != first) parent[v] = r;
    }
}

// After the sampled hooking pass: the root shared by most of 1,024 vertices
// drawn with a fixed splitmix64 stream (vertices still alone in their tree
// do not vote), written to *root_out (~0u when none has a tree yet).  One
// CTA of kGiantSamples threads.  Which root wins changes no result: it only
// picks the tree whose records the full sweep may skip.
constexpr int kGiantSamples = 1024;
__global__ void __launch_bounds__(kGiantSamples) wcc_giant_root_kernel(const uint32_t* parent, uint64_t V,
                                                                        uint32_t* root_out) {
    __shared__ uint32_t s_root[kGiantSamples];
    __shared__ unsigned long long s_best;
    const uint32_t t = threadIdx.x;
    uint64_t z = (uint64_t)(t + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const uint32_t v = (uint32_t)(z % V);
    const uint32_t r = find_root(parent, v);
    const uint32_t mine = r == v ? ~0u : r;   // a root votes for no tree (its own is rarely the largest)
    s_root[t] = mine;
    if (t == 0) s_best = 0;
    __syncthreads();
    uint32_t n = 0;
    if (mine != ~0u)
        for (int i = 0; i < kGiantSamples; ++i) n += s_root[i] == mine;
    if (n) atomicMax(&s_best, ((unsigned long long)n << 32) | mine);
    __syncthreads();
    if (t == 0) *root_out = s_best ? (uint32_t)s_best : ~0u;
}

// Pointer jumping as compress_kernel, and the bitmap of the vertices whose
// root is *root (the largest sampled tree): bit v & 31 of word v >> 5.
// Warps take whole 32-vertex words (N is a multiple of 65,536).
__global__ void wcc_compress_giant_kernel(uint32_t* parent, uint32_t* giant, const uint32_t* root, uint64_t N) {
    const uint32_t c = *root;
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t nwords = N >> 5;
    const uint64_t step = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    uint32_t known = c, first;   // c is a root: the sampled pass is over
    for (uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nwords; w += step) {
        const uint32_t v = (uint32_t)(w * 32 + lane);
        const uint32_t r = find_root_known(parent, v, known, &first);
        if (r != first) parent[v] = r;
        const uint32_t bits = __ballot_sync(kFull, r == c);
        if (lane == 0) giant[w] = bits;
    }
}

__global__ void wcc_label_kernel(const uint32_t* parent, const uint8_t* touched, uint32_t* out, uint64_t N,
                                 unsigned long long* count) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    uint64_t local = 0;
    uint32_t known = ~0u, first;
    for (uint64_t v = tid; v < N; v += nth) {
        if (!touched[v]) {
            out[v] = 0xFFFFFFFFu;  // invalid_cid, wcc.cpp:54
            continue;
        }
        const uint32_t r = find_root_known(parent, (uint32_t)v, known, &first);
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

// The sampled pass of a resident graph's first WCC sweep: one 16-byte group
// of records in every 2^shift (GS_WCC_SAMPLE_SHIFT overrides the default;
// 0 turns the pass off), on graphs of at least kWccSampleMinRecords records.
constexpr uint32_t kWccSampleShift = 4;
constexpr uint64_t kWccSampleMinRecords = 1ull << 22;

uint32_t gs_wcc_sample_shift(const gs_graph* g) {
    if (g->stream || g->seg.list || g->E < kWccSampleMinRecords) return 0;
    const char* e = std::getenv("GS_WCC_SAMPLE_SHIFT");
    if (!e || !*e) return kWccSampleShift;
    const long v = std::strtol(e, nullptr, 10);
    return v <= 0 ? 0u : (uint32_t)std::min<long>(v, 10);
}

gs_status wcc_sweep_launch(gs_state* s) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    const uint64_t bytes = 4 * g->E + 8 * g->V;
    const uint32_t shift = s->step == 0 ? gs_wcc_sample_shift(g) : 0;
    if (shift == 0) {
        // later sweeps (only after a record ran out of hooking retries) keep
        // the first sweep's bitmap: its vertices still share one tree
        if (s->step == 0) s->wcc_giant = false;
        WccOp op{s->d_parent, s->step == 0 ? s->d_touched : nullptr, (unsigned long long*)ctx->d_scalars,
                 s->wcc_giant ? s->d_giant : nullptr};
        return launch_sweep(g, op, GS_ALGO_WCC, bytes, true);
    }
    // Afforest's order (Sutton, Ben-Nun, Barak, "Optimizing Parallel Graph
    // Connectivity Computation via Subgraph Sampling", IPDPS 2018), restated
    // for the tile grid: hook a sample of the records, find the largest tree,
    // then sweep every record, skipping those with both ends in that tree.
    GS_TRY(gs_ensure_blocked(g));
    if (!s->d_giant) GS_TRY(gs_state_alloc(s, (void**)&s->d_giant, (g->N / 32 + 2) * 4));
    uint32_t* d_root = s->d_giant + g->N / 32;
    // the sampled pass walks the L2-blocked runs (its hooks land on parents
    // of a few windows at a time); the full pass walks the longest-first runs
    // of the BFS sweep (one row window staged per long run), since few of
    // its records reach the parents
    const bool blk = g->d_runs_blk != nullptr;
    const uint64_t n = blk ? g->R_blk : g->R;
    const bool lpt = g->d_runs_lpt != nullptr;
    const uint64_t n_full = lpt ? g->R_lpt : g->R;
    const uint32_t grid =
        (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(n, gs_grid_size(ctx, kWccHookCtasPerSm)));
    const uint32_t grid_full =
        (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(n_full, gs_grid_size(ctx, kWccHookCtasPerSm)));
    gs_timer_begin(ctx);
    wcc_hook_runs<<<grid, kThreads, 0, ctx->stream>>>(blk ? g->d_runs_blk : g->d_runs, n,
                                                      blk ? g->d_units_blk : g->d_units, g->d_rec, s->d_parent,
                                                      nullptr, nullptr, nullptr, shift, ctx->d_ticket);
    wcc_giant_root_kernel<<<1, kGiantSamples, 0, ctx->stream>>>(s->d_parent, g->V, d_root);
    wcc_compress_giant_kernel<<<blocks_for(g->N, ctx), kThreads, 0, ctx->stream>>>(s->d_parent, s->d_giant,
                                                                                    d_root, g->N);
    wcc_hook_runs<<<grid_full, kThreads, 0, ctx->stream>>>(lpt ? g->d_runs_lpt : g->d_runs, n_full, g->d_units,
                                                           g->d_rec, s->d_parent, s->d_touched, s->d_giant,
                                                           (unsigned long long*)ctx->d_scalars, 0, ctx->d_ticket);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches += 4;
    s->wcc_giant = true;
    gs_timer_end(ctx, GS_ALGO_WCC, bytes);
    return GS_OK;
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
