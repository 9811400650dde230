// Serving loop (sm_100a): BFS / WCC / k-core / PageRank requests against
// resident graphs, admitted by HBM footprint and batched continuously.
//
// The reference answers one query per process run (gstore.cpp:250-333).
// Here a server keeps many requests in flight:
//
//   * BFS requests on one graph share a multi-source BFS: up to 64 of them as
//     bits of 64-bit frontier words, each bit with its own level, so requests
//     join a running group at any step (bfs_onepart for all bits,
//     bfs.cpp:138-185; iteration_finalize, bfs.cpp:187-224).  A step
//
//       [ table upload | counter reset | sweep kernel | post kernel |
//         counter readback ]
//
//     is captured once as a CUDA graph and replayed; the host rewrites the
//     pinned job table between steps, the sweep kernel walks the
//     concatenated runs of every group, the post kernel their vertex words.
//   * WCC, k-core and PageRank requests run to completion on side streams
//     (lower priority), beside the steps: chunks of iterations are queued
//     without waiting, each kernel first reading the request's device-side
//     done flag, and the host polls one event per chunk.  WCC: hooking sweep
//     (wcc.cpp:177-278) + pointer jumping (wcc.cpp:372-390), done when a
//     sweep left no record unresolved; k-core: round (kcore.cpp:179-217, first) +
//     decrement sweep (kcore.cpp:63-177), done when a round removed
//     nothing; PageRank: row-slice sweep + update, `arg` iterations.
//
// Each gs_serve_step admits queued requests while their state fits the HBM
// budget and a slot is free (a request identical to one queued or running --
// same graph, algorithm and argument -- attaches to it instead), launches the
// BFS step, tends the side requests while it runs, then retires the finished
// requests: results land in pinned host buffers, listed by
// gs_serve_completed, taken with gs_serve_result (a copy) or read in place
// with gs_serve_result_view until gs_serve_release.
#include "gs_internal.cuh"
#include "gs_ops.cuh"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <new>
#include <set>
#include <unordered_map>
#include <vector>

namespace {

using namespace gsops;

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kSlots = 64;
constexpr int kMaxJobs = 256;
constexpr int kCounters = 4;
constexpr int kSideSlots = 64;
constexpr int kSideStreams = 8;
// iterations queued per chunk: one WCC sweep normally finishes (its hooks
// lose no link), so a WCC chunk is one sweep and its pointer jumping
constexpr int kWccChunk = 1;
constexpr int kKcoreChunk = 8;

typedef FvPair<unsigned long long> Fv64;

// One BFS group of the step table.
struct Job {
    const gs_tile_run* runs;
    const gs_unit* units;
    const uint32_t* rec;
    uint64_t R, words;
    uint64_t run_beg, word_beg;   // offsets in the concatenated lists
    uint32_t nw;
    int directed;
    Fv64* fv;
    unsigned long long* next;
    uint8_t* depth;               // [64][N]: one plane per slot
    uint8_t* act_cur;
    uint8_t* act_next;
    unsigned long long* cnt;      // kCounters per job
    uint8_t level[kSlots];        // frontier depth per slot (0 = slot idle)
};

struct Table {
    int n_jobs;
    int pad;
    uint64_t total_runs, total_words;
    Job jobs[kMaxJobs];
};

__device__ __forceinline__ int job_of(const Table* t, uint64_t x, bool by_words) {
    int lo = 0, hi = t->n_jobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const uint64_t b = by_words ? t->jobs[mid].word_beg : t->jobs[mid].run_beg;
        if (b <= x) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// A CTA takes the next run of the concatenated lists from `ticket` (zeroed
// by the step before the launch).
__global__ void __launch_bounds__(kThreads) serve_sweep_kernel(const Table* __restrict__ t,
                                                               unsigned long long* ticket) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n_jobs = t->n_jobs;
    // the flags the post kernel sets start empty
    for (int j = blockIdx.x; j < n_jobs; j += gridDim.x) {
        const Job& jb = t->jobs[j];
        for (uint32_t w = threadIdx.x; w < jb.nw; w += blockDim.x) jb.act_next[w] = 0;
    }
    __shared__ unsigned long long s_run;
    auto draw = [&]() -> uint64_t {
        __syncthreads();   // every thread has read the previous draw
        if (threadIdx.x == 0) s_run = atomicAdd(ticket, 1ull);
        __syncthreads();
        return s_run;
    };
    for (uint64_t x = draw(); x < t->total_runs; x = draw()) {
        const Job& jb = t->jobs[job_of(t, x, false)];
        const gs_tile_run run = jb.runs[x - jb.run_beg];
        const uint32_t row = jb.units[run.unit_beg].rc >> 16;
        const bool ar = jb.act_cur[row] != 0;
        for (uint32_t ui = run.unit_beg + warp; ui < run.unit_end; ui += kWarps) {
            const gs_unit d = jb.units[ui];
            if (!ar && (jb.directed || !jb.act_cur[d.rc & 0xFFFFu])) continue;
            ms_sweep_unit<unsigned long long>(d, jb.rec, jb.fv, jb.next, jb.directed, lane);
        }
    }
}

// Depth planes are written per warp and slot: the 32 lanes' vertices are
// consecutive, so each write of a plane is one 32-byte sector.
__global__ void __launch_bounds__(kThreads) serve_post_kernel(const Table* __restrict__ t) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t gwarp = (uint64_t)blockIdx.x * kWarps + warp;
    const uint64_t nwarps = (uint64_t)gridDim.x * kWarps;
    for (uint64_t x = gwarp; x < t->total_words; x += nwarps) {
        const Job& jb = t->jobs[job_of(t, x, true)];
        const uint64_t v = (x - jb.word_beg) * 32 + lane;
        const unsigned long long nx = jb.next[v];
        const Fv64 s = load_fv(jb.fv + v);
        unsigned long long fresh = 0;
        if (nx || s.f) {
            if (nx) jb.next[v] = 0;
            fresh = nx & ~s.vis;
            store_fv(jb.fv + v, fresh, s.vis | fresh);
        }
        unsigned long long any = fresh;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) any |= __shfl_xor_sync(kFull, any, o);
        if (!any) continue;
        const uint64_t N = jb.words * 32;
        unsigned long long over = 0, m = any;
        while (m) {
            const int q = __ffsll((long long)m) - 1;
            const int d = jb.level[q] + 1;
            if (d >= 255) over |= 1ull << q;   // bfs.cpp level limit (u8 depth_t)
            else if (fresh >> q & 1) jb.depth[(uint64_t)q * N + v] = (uint8_t)d;
            m &= m - 1;
        }
        if (lane == 0) {
            jb.act_next[v >> 16] = 1;
            atomicOr(jb.cnt + 0, any);
            if (over) atomicOr(jb.cnt + 1, over);
        }
    }
}

// ------------------------------------------------------- side requests --
// Kernels of WCC / k-core requests queued in chunks: each returns at once
// when the request's done flag is set.  Iteration `it` uses counter
// cnt[it & 1] and clears cnt[(it + 1) & 1] for the next one.

// One sweep of a request's graph; `gate` (k-core: the round's removals)
// zero means the request is done.
template <class Op>
__global__ void __launch_bounds__(kThreads) side_sweep_kernel(const gs_tile_run* __restrict__ runs, uint64_t R,
                                                              const gs_unit* __restrict__ units,
                                                              const uint32_t* __restrict__ rec, Op op, int* done,
                                                              const unsigned long long* gate) {
    if (__ldcg(done)) return;
    if (gate && __ldcg(gate) == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) *done = 1;
        return;
    }
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint64_t i = blockIdx.x; i < R; i += gridDim.x) {
        const gs_tile_run run = runs[i];
        for (uint32_t ui = run.unit_beg + warp; ui < run.unit_end; ui += kWarps) sweep_unit(units[ui], rec, op, lane);
    }
}

// WCC after sweep `it`: pointer jumping (wcc.cpp:372-390); done when the
// sweep left no record unresolved (normally after the first).
__global__ void side_wcc_post(uint32_t* parent, uint64_t N, unsigned long long* cnt, int it, int* done) {
    if (__ldcg(done)) return;
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = tid; v < N; v += nth) {
        const uint32_t r = find_root(parent, (uint32_t)v);
        if (r != v) parent[v] = r;
    }
    if (tid == 0) {
        cnt[(it + 1) & 1] = 0;
        if (__ldcg(cnt + (it & 1)) == 0) *done = 1;
    }
}

// k-core round `it` (kcore.cpp:179-217): remove 0 < (int16)deg < k; their
// windows go to act_w (cleared by the previous round); act_z is cleared for
// the next round.
__global__ void side_kcore_round(int32_t* __restrict__ deg, uint32_t* __restrict__ removed, uint8_t* act_w,
                                 uint8_t* act_z, uint32_t nw, uint64_t n_words, int k, unsigned long long* cnt,
                                 int it, int* done) {
    if (__ldcg(done)) return;
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t w = tid; w < nw; w += nth) act_z[w] = 0;
    if (tid == 0) cnt[(it + 1) & 1] = 0;
    const uint64_t warp = tid >> 5, nwarps = nth >> 5;
    uint64_t local = 0;
    for (uint64_t w = warp; w < n_words; w += nwarps) {
        const uint64_t v = w * 32 + lane;
        const int16_t m = (int16_t)deg[v];      // kcore.cpp:189
        const bool gone = m < k && m > 0;
        if (gone) deg[v] = 0;
        const uint32_t bits = __ballot_sync(kFull, gone);
        if (lane == 0) {
            removed[w] = bits;
            if (bits) act_w[w >> 11] = 1;
            local += __popc(bits);
        }
    }
    if (lane == 0 && local) atomicAdd(cnt + (it & 1), (unsigned long long)local);
}

// Admission: request q of a BFS group starts at `root` (bfs.cpp:70).
__global__ void serve_seed_bfs(Fv64* fv, uint8_t* depth, uint64_t N, uint8_t* act_cur, uint64_t root, int q) {
    fv[root].f |= 1ull << q;
    fv[root].vis |= 1ull << q;
    depth[(uint64_t)q * N + root] = 1;
    act_cur[root >> 16] = 1;
}

// Retirement of BFS slots: their frontier and visited bits cleared for the
// next requests in the slots (the depth planes are copied out and zeroed by
// the host's stream operations).
__global__ void serve_clear_slots(Fv64* fv, uint64_t N, unsigned long long keep) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = tid; v < N; v += nth) {
        const Fv64 s = load_fv(fv + v);
        if ((s.f | s.vis) & ~keep) store_fv(fv + v, s.f & keep, s.vis & keep);
    }
}

__global__ void serve_iota(uint32_t* parent, uint64_t N) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = tid; v < N; v += nth) parent[v] = (uint32_t)v;
}

__global__ void serve_pr_init(float* x, float* y, uint64_t N, uint64_t V) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    const float x0 = (float)(1.0 / (double)V);         // pr.cpp:105-110
    for (uint64_t v = tid; v < N; v += nth) {
        x[v] = v < V ? x0 : 0.f;
        y[v] = 0.f;
    }
}

__global__ void serve_wcc_labels(const uint32_t* parent, const uint8_t* touched, uint32_t* out, uint64_t V) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = tid; v < V; v += nth) {
        if (!touched[v]) {
            out[v] = 0xFFFFFFFFu;     // invalid_cid, wcc.cpp:54
            continue;
        }
        uint32_t r = parent[v];
        while (parent[r] != r) r = parent[r];
        out[v] = r;
    }
}

// ------------------------------------------------------------ host side --
enum ReqState : int { kQueued = 0, kActive = 1, kDone = 2, kFailed = 3 };

struct HostBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

}  // namespace

struct gs_server;

namespace {

struct SrvGraph {
    gs_graph* g = nullptr;
    // BFS group
    Fv64* fv = nullptr;
    unsigned long long* next = nullptr;
    uint8_t* depth = nullptr;
    uint8_t* act[2] = {nullptr, nullptr};
    int cur = 0;
    int64_t slot_req[kSlots];
    int slot_start[kSlots];           // step whose sweep sees depth 1
    unsigned long long used = 0;
    size_t group_bytes = 0;
    float* pb_val = nullptr;          // the server's value stream for this graph's PageRank requests
    bool pb_val_busy = false;         // a PageRank request is sweeping with it
};

struct Request {
    uint64_t id = 0;
    int graph = 0;
    gs_algo algo = GS_ALGO_BFS;
    int64_t arg = 0;
    int state = kQueued;
    gs_status status = GS_OK;
    double t_submit = 0, t_admit = 0, t_done = 0;
    int steps = 0;
    int slot = -1;                       // BFS slot
    int job = -1;                        // position in this step's table
    int64_t leader = -1;                 // attached to an identical request
    std::vector<uint64_t> followers;
    size_t footprint = 0;
    // device state (pool blocks)
    uint32_t* parent = nullptr;
    uint8_t* touched = nullptr;
    uint32_t* labels = nullptr;          // WCC result staging
    int32_t* deg = nullptr;
    uint32_t* removed = nullptr;
    uint8_t* act[2] = {nullptr, nullptr};
    int cur = 0;
    float* x = nullptr;
    float* y = nullptr;
    float* r = nullptr;
    float* val = nullptr;                // PageRank on the propagation-blocked layout: its value stream
    bool own_val = false;                // val is this request's (else the graph's stream in the server)
    int* flags = nullptr;                // side requests: [0] done, [1] bounded-wait error
    unsigned long long* cnt = nullptr;   // side requests: two iteration counters
    int side = -1;                       // side slot (WCC, k-core, PageRank)
    int iter = 0;                        // iterations queued so far
    bool chunk_pending = false;
    bool result_pending = false;         // result copy queued, event not yet seen
    std::shared_ptr<HostBuf> result;     // pinned host copy of the result
    uint64_t result_bytes = 0;
};

}  // namespace

struct gs_server {
    gs_ctx* ctx = nullptr;
    uint64_t budget = 0;
    uint64_t used = 0;
    cudaStream_t stream = nullptr;
    // side requests (WCC, k-core, PageRank): kSideSlots slots over
    // kSideStreams lower-priority streams, an event and a pinned flag pair
    // per slot
    cudaStream_t side_stream[kSideStreams] = {};
    int n_side = kSideStreams;           // side streams in use
    cudaEvent_t side_ev[kSideSlots] = {};
    int* h_flags = nullptr;              // pinned, kSideSlots x 2
    std::vector<int> side_free;
    cudaGraphExec_t step_exec = nullptr;
    cudaGraph_t step_graph = nullptr;
    Table* h_table = nullptr;            // pinned
    Table* d_table = nullptr;
    unsigned long long* h_cnt = nullptr; // pinned, kMaxJobs x kCounters
    unsigned long long* d_cnt = nullptr; // kMaxJobs x kCounters, then the sweep ticket
    std::vector<SrvGraph> graphs;
    std::unordered_map<uint64_t, Request> reqs;
    std::deque<uint64_t> queue;
    std::vector<uint64_t> active;
    std::deque<uint64_t> completed;      // finished since the client last asked
    uint64_t next_id = 1;
    int step = 0;
    uint64_t steps_run = 0, graph_launches = 0, kernel_launches = 0;
    // host seconds spent in gs_serve_step by phase: admission, BFS step
    // launch, side requests, BFS step finish (its wait included); then the
    // seconds and count of pinned-host and device allocations made on pool
    // misses (inside those phases)
    double phase_s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    double side_in_wait_s = 0;           // side tending inside the step wait
    std::chrono::steady_clock::time_point t0;
    // device pool: exact-size free lists over blocks drawn from the
    // context's pool, which gets them all back when the server is freed (a
    // later server, batch or query state of the context reuses them)
    std::multimap<size_t, void*> dev_free;
    std::vector<std::pair<void*, size_t>> dev_all;
    // pinned host arena for results: chunks from cudaHostAlloc, carved
    // best-fit into page-rounded blocks; a freed block merges with free
    // neighbours of the same chunk
    std::vector<std::pair<char*, size_t>> host_chunks;
    std::set<char*> chunk_starts;
    std::map<char*, size_t> host_free_at;           // free blocks by address
    std::multimap<size_t, char*> host_free_size;    // the same blocks by size
};

namespace {

inline cudaStream_t side_stream_of(const gs_server* s, const Request& r) {
    return s->side_stream[r.side % s->n_side];
}

double now_s(const gs_server* s) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - s->t0).count();
}

gs_status pool_dev(gs_server* s, size_t bytes, void** out) {
    bytes = (bytes + 255) & ~(size_t)255;
    auto it = s->dev_free.find(bytes);
    if (it != s->dev_free.end()) {
        *out = it->second;
        s->dev_free.erase(it);
        return GS_OK;
    }
    const double t = now_s(s);
    const uint64_t held = s->ctx->pool_bytes;
    GS_TRY(gs_pool_get(s->ctx, bytes, out));
    if (s->ctx->pool_bytes == held) {   // the context's pool had no such block: cudaMalloc ran
        s->phase_s[6] += now_s(s) - t;
        s->phase_s[7] += 1;
    }
    s->dev_all.emplace_back(*out, bytes);
    return GS_OK;
}

void pool_dev_put(gs_server* s, void* p, size_t bytes) {
    if (p) s->dev_free.emplace((bytes + 255) & ~(size_t)255, p);
}

constexpr size_t kHostPage = 4096;
constexpr size_t kHostChunk = 64ull << 20;   // least bytes pinned per arena miss

inline size_t host_round(size_t bytes) { return (std::max<size_t>(bytes, 1) + kHostPage - 1) & ~(kHostPage - 1); }

void arena_insert(gs_server* s, char* p, size_t n) {
    s->host_free_at.emplace(p, n);
    s->host_free_size.emplace(n, p);
}

void arena_erase(gs_server* s, std::map<char*, size_t>::iterator it) {
    auto range = s->host_free_size.equal_range(it->second);
    for (auto j = range.first; j != range.second; ++j)
        if (j->second == it->first) {
            s->host_free_size.erase(j);
            break;
        }
    s->host_free_at.erase(it);
}

// Returns a block to the arena, merged with the free blocks on either side
// that lie in the same chunk.
void arena_put(gs_server* s, char* p, size_t n) {
    auto nx = s->host_free_at.find(p + n);
    if (nx != s->host_free_at.end() && !s->chunk_starts.count(p + n)) {
        n += nx->second;
        arena_erase(s, nx);
    }
    auto pv = s->host_free_at.lower_bound(p);
    if (pv != s->host_free_at.begin() && !s->chunk_starts.count(p)) {
        --pv;
        if (pv->first + pv->second == p) {
            p = pv->first;
            n += pv->second;
            arena_erase(s, pv);
        }
    }
    arena_insert(s, p, n);
}

// Pins a new chunk of at least `bytes` and adds it to the arena; `miss`
// counts it as a pool miss (a reservation made ahead of the requests is not).
gs_status arena_grow(gs_server* s, size_t bytes, bool miss) {
    const size_t n = host_round(bytes);
    void* p = nullptr;
    const double t = now_s(s);
    GS_CHECK_CUDA(s->ctx, cudaHostAlloc(&p, n, cudaHostAllocDefault));
    if (miss) {
        s->phase_s[4] += now_s(s) - t;
        s->phase_s[5] += 1;
    }
    s->host_chunks.emplace_back((char*)p, n);
    s->chunk_starts.insert((char*)p);
    arena_insert(s, (char*)p, n);
    return GS_OK;
}

gs_status pool_host(gs_server* s, size_t bytes, void** out) {
    const size_t n = host_round(bytes);
    auto it = s->host_free_size.lower_bound(n);
    if (it == s->host_free_size.end()) {
        GS_TRY(arena_grow(s, std::max(n, kHostChunk), true));
        it = s->host_free_size.lower_bound(n);
    }
    char* p = it->second;
    const size_t have = it->first;
    arena_erase(s, s->host_free_at.find(p));
    if (have > n) arena_insert(s, p + n, have - n);
    *out = p;
    return GS_OK;
}

std::shared_ptr<HostBuf> host_buf(gs_server* s, size_t bytes, gs_status* st) {
    void* p = nullptr;
    *st = pool_host(s, bytes, &p);
    if (*st != GS_OK) return nullptr;
    HostBuf* hb = new HostBuf{p, bytes};
    return std::shared_ptr<HostBuf>(hb, [s](HostBuf* b) {
        arena_put(s, (char*)b->p, host_round(b->bytes));
        delete b;
    });
}

inline uint32_t blocks_for(uint64_t n, const gs_ctx* ctx) {
    const uint64_t b = (n + kThreads - 1) / kThreads;
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(b, gs_grid_size(ctx, 16)));
}

// Side kernels: one thread per element (one CTA per run for sweeps), so
// their CTAs are short and the step's higher-priority CTAs get SMs between
// them instead of waiting for a grid-stride kernel to drain.
inline uint32_t short_blocks(uint64_t n) {
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((n + kThreads - 1) / kThreads, 0x7FFFFFFFull));
}

size_t group_bytes(const gs_graph* g) {
    return g->N * (sizeof(Fv64) + 8 + kSlots) + 2 * (size_t)g->nw + 256;
}

// HBM bytes a request adds when admitted.
size_t footprint(const gs_server* s, const Request& r) {
    const SrvGraph& sg = s->graphs[r.graph];
    const gs_graph* g = sg.g;
    switch (r.algo) {
        case GS_ALGO_BFS: return sg.fv ? 0 : group_bytes(g);
        case GS_ALGO_WCC: return g->N * 5 + g->V * 4 + 64;
        case GS_ALGO_KCORE: return g->N * 4 + g->N / 8 + 2 * (size_t)g->nw + 64;
        default:
            // a PageRank request takes the value stream the server keeps for
            // the graph; one beside it needs a stream of its own
            return g->N * 12 + (g->pb.built && sg.pb_val_busy ? g->pb.n_entries * 4 : 0) + 64;
    }
}

gs_status open_group(gs_server* s, SrvGraph& sg) {
    gs_ctx* ctx = s->ctx;
    const gs_graph* g = sg.g;
    const uint64_t N = g->N;
    GS_TRY(pool_dev(s, N * sizeof(Fv64), (void**)&sg.fv));
    GS_TRY(pool_dev(s, N * 8, (void**)&sg.next));
    GS_TRY(pool_dev(s, N * kSlots, (void**)&sg.depth));
    GS_TRY(pool_dev(s, g->nw, (void**)&sg.act[0]));
    GS_TRY(pool_dev(s, g->nw, (void**)&sg.act[1]));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(sg.fv, 0, N * sizeof(Fv64), s->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(sg.next, 0, N * 8, s->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(sg.depth, 0, N * kSlots, s->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(sg.act[0], 0, g->nw, s->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(sg.act[1], 0, g->nw, s->stream));
    sg.cur = 0;
    sg.used = 0;
    sg.group_bytes = group_bytes(g);
    for (int q = 0; q < kSlots; ++q) sg.slot_req[q] = -1;
    return GS_OK;
}

void close_group(gs_server* s, SrvGraph& sg) {
    const gs_graph* g = sg.g;
    pool_dev_put(s, sg.fv, g->N * sizeof(Fv64));
    pool_dev_put(s, sg.next, g->N * 8);
    pool_dev_put(s, sg.depth, g->N * kSlots);
    pool_dev_put(s, sg.act[0], g->nw);
    pool_dev_put(s, sg.act[1], g->nw);
    sg.fv = nullptr;
    sg.next = nullptr;
    sg.depth = nullptr;
    sg.act[0] = sg.act[1] = nullptr;
    s->used -= sg.group_bytes;
    sg.group_bytes = 0;
}

gs_status admit(gs_server* s, Request& r) {
    gs_ctx* ctx = s->ctx;
    SrvGraph& sg = s->graphs[r.graph];
    const gs_graph* g = sg.g;
    const uint64_t N = g->N;
    r.footprint = footprint(s, r);
    if (r.algo == GS_ALGO_BFS) {
        if (!sg.fv) {
            GS_TRY(open_group(s, sg));
            s->used += sg.group_bytes;
            r.footprint = 0;
        }
        int q = 0;
        while (sg.used >> q & 1) ++q;
        sg.used |= 1ull << q;
        sg.slot_req[q] = (int64_t)r.id;
        sg.slot_start[q] = s->step;
        r.slot = q;
        serve_seed_bfs<<<1, 1, 0, s->stream>>>(sg.fv, sg.depth, N, sg.act[sg.cur], (uint64_t)r.arg, q);
        s->kernel_launches++;
    } else {
        r.side = s->side_free.back();
        s->side_free.pop_back();
        cudaStream_t st = side_stream_of(s, r);
        GS_TRY(pool_dev(s, 256, (void**)&r.flags));
        GS_TRY(pool_dev(s, 2 * sizeof(unsigned long long), (void**)&r.cnt));
        GS_CHECK_CUDA(ctx, cudaMemsetAsync(r.flags, 0, 256, st));
        GS_CHECK_CUDA(ctx, cudaMemsetAsync(r.cnt, 0, 2 * sizeof(unsigned long long), st));
        switch (r.algo) {
            case GS_ALGO_WCC:
                GS_TRY(pool_dev(s, N * 4, (void**)&r.parent));
                GS_TRY(pool_dev(s, N, (void**)&r.touched));
                GS_TRY(pool_dev(s, g->V * 4 + 16, (void**)&r.labels));
                serve_iota<<<short_blocks(N), kThreads, 0, st>>>(r.parent, N);
                s->kernel_launches++;
                GS_CHECK_CUDA(ctx, cudaMemsetAsync(r.touched, 0, N, st));
                break;
            case GS_ALGO_KCORE:
                GS_TRY(pool_dev(s, N * 4, (void**)&r.deg));
                GS_TRY(pool_dev(s, N / 8, (void**)&r.removed));
                GS_TRY(pool_dev(s, g->nw, (void**)&r.act[0]));
                GS_TRY(pool_dev(s, g->nw, (void**)&r.act[1]));
                GS_CHECK_CUDA(ctx, cudaMemcpyAsync(r.deg, g->d_degree, N * 4, cudaMemcpyDeviceToDevice, st));
                GS_CHECK_CUDA(ctx, cudaMemsetAsync(r.act[0], 0, g->nw, st));
                GS_CHECK_CUDA(ctx, cudaMemsetAsync(r.act[1], 0, g->nw, st));
                break;
            default:
                // PageRank sweeps the graph's propagation-blocked layout with
                // a value stream of its own (requests on one graph may run
                // side by side), else the row-slice layout (each built once)
                if (!g->pb.built && !g->pr.built) GS_TRY(pr_layout_build(sg.g));
                if (g->pb.built && !sg.pb_val_busy) {
                    r.val = sg.pb_val;
                    r.own_val = false;
                    sg.pb_val_busy = true;
                } else if (g->pb.built) {
                    GS_TRY(pool_dev(s, g->pb.n_entries * 4, (void**)&r.val));
                    r.own_val = true;
                }
                GS_TRY(pool_dev(s, N * 4, (void**)&r.x));
                GS_TRY(pool_dev(s, N * 4, (void**)&r.y));
                GS_TRY(pool_dev(s, N * 4, (void**)&r.r));
                serve_pr_init<<<short_blocks(N), kThreads, 0, st>>>(r.x, r.y, N, g->V);
                s->kernel_launches++;
                break;
        }
        r.iter = 0;
        r.chunk_pending = false;
    }
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    s->used += r.footprint;
    r.state = kActive;
    r.t_admit = now_s(s);
    r.steps = 0;
    return GS_OK;
}

void release(gs_server* s, Request& r) {
    const gs_graph* g = s->graphs[r.graph].g;
    const uint64_t N = g->N;
    switch (r.algo) {
        case GS_ALGO_BFS: {
            SrvGraph& sg = s->graphs[r.graph];
            sg.used &= ~(1ull << r.slot);
            sg.slot_req[r.slot] = -1;
            if (!sg.used) close_group(s, sg);
            break;
        }
        case GS_ALGO_WCC:
            pool_dev_put(s, r.parent, N * 4);
            pool_dev_put(s, r.touched, N);
            pool_dev_put(s, r.labels, g->V * 4 + 16);
            break;
        case GS_ALGO_KCORE:
            pool_dev_put(s, r.deg, N * 4);
            pool_dev_put(s, r.removed, N / 8);
            pool_dev_put(s, r.act[0], g->nw);
            pool_dev_put(s, r.act[1], g->nw);
            break;
        default:
            pool_dev_put(s, r.x, N * 4);
            pool_dev_put(s, r.y, N * 4);
            pool_dev_put(s, r.r, N * 4);
            if (r.val && r.own_val) pool_dev_put(s, r.val, g->pb.n_entries * 4);
            else if (r.val) s->graphs[r.graph].pb_val_busy = false;
            r.val = nullptr;
            break;
    }
    if (r.side >= 0) {
        pool_dev_put(s, r.flags, 256);
        pool_dev_put(s, r.cnt, 2 * sizeof(unsigned long long));
        s->side_free.push_back(r.side);
        r.side = -1;
    }
    r.flags = nullptr;
    r.cnt = nullptr;
    r.parent = nullptr;
    r.touched = nullptr;
    r.labels = nullptr;
    r.deg = nullptr;
    r.removed = nullptr;
    r.act[0] = r.act[1] = nullptr;
    r.x = r.y = r.r = nullptr;
    s->used -= r.footprint;
    r.footprint = 0;
}

void fill_graph_tables(Job& j, const gs_graph* g) {
    j.runs = g->d_runs_blk ? g->d_runs_blk : g->d_runs;
    j.units = g->d_runs_blk ? g->d_units_blk : g->d_units;
    j.rec = g->d_rec;
    j.R = g->d_runs_blk ? g->R_blk : g->R;
    j.words = g->N / 32;
    j.nw = g->nw;
    j.directed = g->directed;
}

// Enqueues the copy of a finished side request's result to pinned host
// memory on the request's stream.
gs_status take_result(gs_server* s, Request& r) {
    gs_ctx* ctx = s->ctx;
    const gs_graph* g = s->graphs[r.graph].g;
    const void* src = nullptr;
    cudaStream_t stream = side_stream_of(s, r);
    switch (r.algo) {
        case GS_ALGO_WCC:
            wcc_mark_touched<<<short_blocks(g->N), kThreads, 0, stream>>>(r.parent, r.touched, g->N);
            serve_wcc_labels<<<short_blocks(g->V), kThreads, 0, stream>>>(r.parent, r.touched, r.labels,
                                                                                 g->V);
            s->kernel_launches += 2;
            src = r.labels;
            r.result_bytes = g->V * 4;
            break;
        case GS_ALGO_KCORE:
            src = r.deg;
            r.result_bytes = g->V * 4;
            break;
        default:
            src = r.r;
            r.result_bytes = g->V * 4;
            break;
    }
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    gs_status st = GS_OK;
    r.result = host_buf(s, r.result_bytes, &st);
    if (st != GS_OK) return st;
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(r.result->p, src, r.result_bytes, cudaMemcpyDeviceToHost, stream));
    return GS_OK;
}

gs_status build_step_graph(gs_server* s) {
    gs_ctx* ctx = s->ctx;
    const int grid = (int)gs_grid_size(ctx, 8);
    GS_CHECK_CUDA(ctx, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    cudaMemcpyAsync(s->d_table, s->h_table, sizeof(Table), cudaMemcpyHostToDevice, s->stream);
    // the job counters and, after them, the sweep's run ticket
    cudaMemsetAsync(s->d_cnt, 0, sizeof(unsigned long long) * (kMaxJobs * kCounters + 1), s->stream);
    serve_sweep_kernel<<<grid, kThreads, 0, s->stream>>>(s->d_table, s->d_cnt + kMaxJobs * kCounters);
    serve_post_kernel<<<grid, kThreads, 0, s->stream>>>(s->d_table);
    cudaMemcpyAsync(s->h_cnt, s->d_cnt, sizeof(unsigned long long) * kMaxJobs * kCounters, cudaMemcpyDeviceToHost,
                    s->stream);
    GS_CHECK_CUDA(ctx, cudaStreamEndCapture(s->stream, &s->step_graph));
    GS_CHECK_CUDA(ctx, cudaGraphInstantiate(&s->step_exec, s->step_graph, 0));
    return GS_OK;
}

bool same_query(const Request& a, const Request& b) {
    return a.graph == b.graph && a.algo == b.algo && (a.algo == GS_ALGO_WCC || a.arg == b.arg);
}

// Queues the next chunk of a side request's iterations on its stream, then
// the copy of its flags and the chunk's event.
gs_status queue_chunk(gs_server* s, Request& r) {
    gs_ctx* ctx = s->ctx;
    gs_graph* g = s->graphs[r.graph].g;
    cudaStream_t st = side_stream_of(s, r);
    const gs_tile_run* runs = g->d_runs_blk ? g->d_runs_blk : g->d_runs;
    const gs_unit* units = g->d_runs_blk ? g->d_units_blk : g->d_units;
    const uint64_t R = g->d_runs_blk ? g->R_blk : g->R;
    const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(R, 0x7FFFFFFFull));
    switch (r.algo) {
        case GS_ALGO_WCC:
            for (int k = 0; k < kWccChunk; ++k, ++r.iter) {
                const WccOp op{r.parent, r.iter == 0 ? r.touched : nullptr, r.cnt + (r.iter & 1)};
                side_sweep_kernel<<<grid, kThreads, 0, st>>>(runs, R, units, g->d_rec, op, r.flags, nullptr);
                side_wcc_post<<<short_blocks(g->N), kThreads, 0, st>>>(r.parent, g->N, r.cnt, r.iter, r.flags);
                s->kernel_launches += 2;
            }
            break;
        case GS_ALGO_KCORE:
            for (int k = 0; k < kKcoreChunk; ++k, ++r.iter) {
                const int p = r.iter & 1;
                side_kcore_round<<<short_blocks(g->N), kThreads, 0, st>>>(
                    r.deg, r.removed, r.act[p], r.act[p ^ 1], g->nw, g->N / 32, (int)r.arg, r.cnt, r.iter, r.flags);
                const KcoreOp op{r.deg, r.removed, r.act[p]};
                side_sweep_kernel<<<grid, kThreads, 0, st>>>(runs, R, units, g->d_rec, op, r.flags, r.cnt + p);
                s->kernel_launches += 2;
            }
            break;
        default:
            for (; r.iter < r.arg; ++r.iter) {
                if (r.val) GS_TRY(pb_sweep_on(g, st, r.x, r.y, r.flags + 1, r.val));
                else GS_TRY(pr_slice_sweep(g, st, r.x, r.y, r.flags + 1, true));
                GS_TRY(pr_finalize_launch(ctx, st, r.x, r.y, r.r, g->d_degree, g->N, g->V, 0));
                s->kernel_launches += 2;
            }
            break;
    }
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(s->h_flags + 2 * r.side, r.flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    GS_CHECK_CUDA(ctx, cudaEventRecord(s->side_ev[r.side], st));
    r.chunk_pending = true;
    return GS_OK;
}

}  // namespace

extern "C" {

gs_status gs_serve_create(gs_ctx* ctx, uint64_t state_budget_bytes, gs_server** out) {
    if (!ctx || !out) return GS_ERR_ARG;
    *out = nullptr;
    gs_server* s = new (std::nothrow) gs_server();
    if (!s) return GS_ERR_OOM;
    s->ctx = ctx;
    s->budget = state_budget_bytes ? state_budget_bytes : (32ull << 30);
    s->t0 = std::chrono::steady_clock::now();
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    gs_status st = GS_OK;
    cudaError_t e = cudaStreamCreateWithPriority(&s->stream, cudaStreamNonBlocking, hi);
    for (int k = 0; k < kSideStreams && e == cudaSuccess; ++k)
        e = cudaStreamCreateWithPriority(&s->side_stream[k], cudaStreamNonBlocking, lo);
    for (int k = 0; k < kSideSlots && e == cudaSuccess; ++k)
        e = cudaEventCreateWithFlags(&s->side_ev[k], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&s->h_flags, 2 * sizeof(int) * kSideSlots, cudaHostAllocDefault);
    for (int k = kSideSlots - 1; k >= 0; --k) s->side_free.push_back(k);
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&s->h_table, sizeof(Table), cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&s->h_cnt, sizeof(unsigned long long) * kMaxJobs * kCounters,
                                            cudaHostAllocDefault);
    if (e != cudaSuccess) st = gs_cuda_fail(ctx, e, "server set-up");
    if (st == GS_OK) st = gs_dev_alloc(ctx, (void**)&s->d_table, sizeof(Table));
    if (st == GS_OK)
        st = gs_dev_alloc(ctx, (void**)&s->d_cnt, sizeof(unsigned long long) * (kMaxJobs * kCounters + 1));
    if (st == GS_OK) {
        std::memset(s->h_table, 0, sizeof(Table));
        st = build_step_graph(s);
    }
    if (st != GS_OK) {
        gs_serve_free(s);
        return st;
    }
    *out = s;
    return GS_OK;
}

gs_status gs_serve_add_graph(gs_server* s, gs_graph* g, int* graph_id) {
    if (!s || !g || !graph_id) return GS_ERR_ARG;
    if (g->ctx != s->ctx) return gs_fail(s->ctx, GS_ERR_ARG, "graph belongs to another context");
    if (g->stream) return gs_fail(s->ctx, GS_ERR_UNSUPPORTED, "served graphs must be resident in HBM");
    // the PageRank layout and the blocked orders are built here, at set-up,
    // not under a request: the propagation-blocked layout for a graph dense
    // enough for it (the server keeps one value stream per graph for its
    // PageRank requests; a request beside another on the same graph takes a
    // stream of its own), else the row slices
    if (!g->pb.built && !g->pr.built && g->E) {
        if (pb_layout_wanted(g)) GS_TRY(pb_layout_build(g));
        else GS_TRY(pr_layout_build(g));
    }
    GS_TRY(gs_ensure_blocked(g));
    SrvGraph sg;
    sg.g = g;
    if (g->pb.built) GS_TRY(pool_dev(s, g->pb.n_entries * 4, (void**)&sg.pb_val));
    for (int q = 0; q < kSlots; ++q) sg.slot_req[q] = -1;
    s->graphs.push_back(sg);
    *graph_id = (int)s->graphs.size() - 1;
    return GS_OK;
}

gs_status gs_serve_submit(gs_server* s, int graph_id, gs_algo algo, int64_t arg, uint64_t* request_id) {
    if (!s || !request_id || graph_id < 0 || (size_t)graph_id >= s->graphs.size()) return GS_ERR_ARG;
    gs_ctx* ctx = s->ctx;
    const gs_graph* g = s->graphs[graph_id].g;
    if (algo == GS_ALGO_BFS && (arg < 0 || (uint64_t)arg >= g->V)) return gs_fail(ctx, GS_ERR_ARG, "BFS root out of range");
    if (algo == GS_ALGO_KCORE && g->directed) return gs_fail(ctx, GS_ERR_UNSUPPORTED, "Kcore not applicable for directed graphs");
    if (algo == GS_ALGO_PAGERANK && arg < 1) return gs_fail(ctx, GS_ERR_ARG, "iterations < 1");
    if (algo != GS_ALGO_BFS && algo != GS_ALGO_WCC && algo != GS_ALGO_KCORE && algo != GS_ALGO_PAGERANK)
        return GS_ERR_ARG;
    Request r;
    r.id = s->next_id++;
    r.graph = graph_id;
    r.algo = algo;
    r.arg = arg;
    r.t_submit = now_s(s);
    // an identical request queued or running answers this one too
    auto attach = [&](uint64_t other) {
        Request& o = s->reqs[other];
        if (o.leader < 0 && (o.state == kQueued || o.state == kActive) && same_query(o, r)) {
            r.leader = (int64_t)o.id;
            o.followers.push_back(r.id);
            return true;
        }
        return false;
    };
    bool attached = false;
    for (uint64_t a : s->active)
        if (!attached && attach(a)) attached = true;
    for (uint64_t a : s->queue)
        if (!attached && attach(a)) attached = true;
    if (!attached) s->queue.push_back(r.id);
    s->reqs[r.id] = r;
    *request_id = r.id;
    return GS_OK;
}

}  // extern "C"

namespace {

// Marks finished requests done (their result copies were queued and have
// completed), hands results to attached requests and frees their state.
void retire(gs_server* s, const std::vector<uint64_t>& finished, double t) {
    for (uint64_t id : finished) {
        Request& r = s->reqs[id];
        r.state = r.status == GS_OK ? kDone : kFailed;
        r.t_done = t;
        release(s, r);
        s->completed.push_back(id);
        for (uint64_t f : r.followers) {
            s->completed.push_back(f);
            Request& fr = s->reqs[f];
            fr.state = r.state;
            fr.status = r.status;
            fr.t_admit = r.t_admit;
            fr.t_done = t;
            fr.steps = r.steps;
            fr.result = r.result;
            fr.result_bytes = r.result_bytes;
        }
        s->active.erase(std::find(s->active.begin(), s->active.end(), id));
    }
}

// One step of the BFS groups (the captured step graph), in two halves: the
// launch, and the outcomes after the step has run.  `group_job` maps a graph
// to its job in the step (-1: none); *launched says whether a step runs.
gs_status bfs_launch(gs_server* s, std::vector<int>& group_job, bool* launched) {
    gs_ctx* ctx = s->ctx;
    Table* t = s->h_table;
    int nj = 0;
    uint64_t runs = 0, words = 0;
    *launched = false;
    group_job.assign(s->graphs.size(), -1);
    for (uint64_t id : s->active) {
        Request& r = s->reqs[id];
        if (r.algo != GS_ALGO_BFS) continue;
        SrvGraph& sg = s->graphs[r.graph];
        if (group_job[r.graph] >= 0) {
            r.job = group_job[r.graph];
            continue;
        }
        Job& j = t->jobs[nj];
        std::memset(&j, 0, sizeof(Job));
        fill_graph_tables(j, sg.g);
        j.run_beg = runs;
        j.word_beg = words;
        j.cnt = s->d_cnt + (size_t)nj * kCounters;
        j.fv = sg.fv;
        j.next = sg.next;
        j.depth = sg.depth;
        j.act_cur = sg.act[sg.cur];
        j.act_next = sg.act[sg.cur ^ 1];
        for (int q = 0; q < kSlots; ++q)
            j.level[q] = (sg.used >> q & 1) ? (uint8_t)std::min(255, s->step - sg.slot_start[q] + 1) : 0;
        group_job[r.graph] = nj;
        r.job = nj;
        runs += j.R;
        words += j.words;
        ++nj;
    }
    if (nj == 0) return GS_OK;
    t->n_jobs = nj;
    t->total_runs = runs;
    t->total_words = words;
    GS_CHECK_CUDA(ctx, cudaGraphLaunch(s->step_exec, s->stream));
    *launched = true;
    return GS_OK;
}

gs_status side_step(gs_server* s);

gs_status bfs_finish(gs_server* s, const std::vector<int>& group_job) {
    gs_ctx* ctx = s->ctx;
    // the side requests are tended while the step runs: a chunk that ends
    // mid-step has its next one (or its result copy) queued at once
    gs_status side_st = GS_OK;   // a side failure is returned after the step is finished
    for (;;) {
        const cudaError_t q = cudaStreamQuery(s->stream);
        if (q == cudaSuccess) break;
        if (q != cudaErrorNotReady) return gs_cuda_fail(ctx, q, "BFS step");
        if (side_st != GS_OK) {
            GS_CHECK_CUDA(ctx, cudaStreamSynchronize(s->stream));
            break;
        }
        const double t = now_s(s);
        side_st = side_step(s);
        s->side_in_wait_s += now_s(s) - t;
    }
    s->graph_launches++;
    s->kernel_launches += 2;
    s->steps_run++;
    std::vector<uint64_t> finished;
    for (int g = 0; g < (int)s->graphs.size(); ++g)
        if (group_job[g] >= 0) s->graphs[g].cur ^= 1;
    for (uint64_t id : s->active) {
        Request& r = s->reqs[id];
        if (r.algo != GS_ALGO_BFS) continue;
        const unsigned long long* c = s->h_cnt + (size_t)r.job * kCounters;
        r.steps += 1;
        bool done;
        if (c[1] >> r.slot & 1) {
            r.status = GS_ERR_RANGE;
            done = true;
        } else {
            done = !(c[0] >> r.slot & 1);
        }
        if (done) finished.push_back(id);
    }
    s->step += 1;
    if (finished.empty()) return side_st;
    // per graph: the retiring slots' bits cleared in one pass; per request:
    // its depth plane copied to pinned host memory, then zeroed
    std::vector<unsigned long long> retiring(s->graphs.size(), 0);
    for (uint64_t id : finished) {
        Request& r = s->reqs[id];
        retiring[r.graph] |= 1ull << r.slot;
    }
    for (int g = 0; g < (int)s->graphs.size(); ++g) {
        if (!retiring[g]) continue;
        const SrvGraph& sg = s->graphs[g];
        serve_clear_slots<<<blocks_for(sg.g->N, ctx), kThreads, 0, s->stream>>>(sg.fv, sg.g->N, ~retiring[g]);
        s->kernel_launches++;
    }
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    for (uint64_t id : finished) {
        Request& r = s->reqs[id];
        const SrvGraph& sg = s->graphs[r.graph];
        uint8_t* plane = sg.depth + (size_t)r.slot * sg.g->N;
        if (r.status == GS_OK) {
            gs_status st = GS_OK;
            r.result_bytes = sg.g->V;
            r.result = host_buf(s, r.result_bytes, &st);
            if (st != GS_OK) return st;
            GS_CHECK_CUDA(ctx, cudaMemcpyAsync(r.result->p, plane, r.result_bytes, cudaMemcpyDeviceToHost, s->stream));
        }
        GS_CHECK_CUDA(ctx, cudaMemsetAsync(plane, 0, sg.g->N, s->stream));
    }
    GS_CHECK_CUDA(ctx, cudaStreamSynchronize(s->stream));
    retire(s, finished, now_s(s));
    return side_st;
}

// Progress of the side requests: queue a chunk where none is in flight,
// queue the result copy of a request whose last chunk found it done, retire
// a request whose result copy has landed.  Nothing here waits on a stream.
gs_status side_step(gs_server* s) {
    gs_ctx* ctx = s->ctx;
    std::vector<uint64_t> finished;
    for (uint64_t id : s->active) {
        Request& r = s->reqs[id];
        if (r.side < 0) continue;
        if (r.chunk_pending || r.result_pending) {
            const cudaError_t e = cudaEventQuery(s->side_ev[r.side]);
            if (e == cudaErrorNotReady) continue;
            if (e != cudaSuccess) return gs_cuda_fail(ctx, e, "side request");
        }
        if (r.result_pending) {
            r.result_pending = false;
            finished.push_back(id);
            continue;
        }
        if (r.chunk_pending) {
            r.chunk_pending = false;
            const int* f = s->h_flags + 2 * r.side;
            r.steps = r.iter;
            const bool done = r.algo == GS_ALGO_PAGERANK ? r.iter >= r.arg : f[0] != 0;
            if (f[1]) {
                r.status = GS_ERR_TIMEOUT;
                finished.push_back(id);
                continue;
            }
            if (done) {
                GS_TRY(take_result(s, r));
                GS_CHECK_CUDA(ctx, cudaEventRecord(s->side_ev[r.side], side_stream_of(s, r)));
                r.result_pending = true;
                continue;
            }
        }
        GS_TRY(queue_chunk(s, r));
    }
    if (!finished.empty()) retire(s, finished, now_s(s));
    return GS_OK;
}

}  // namespace

extern "C" {

gs_status gs_serve_step(gs_server* s, int* n_active, int* n_queued) {
    if (!s) return GS_ERR_ARG;
    double t_phase = now_s(s);
    auto phase_end = [&](int k) {
        const double t = now_s(s);
        s->phase_s[k] += t - t_phase;
        t_phase = t;
    };
    // admission in arrival order while the state fits the budget: a request
    // whose slot kind is full (its graph's BFS group, or the side slots)
    // waits in place while later requests of other kinds go ahead; the
    // first request that does not fit the budget stops the scan
    {
        std::deque<uint64_t> wait;
        while (!s->queue.empty() && (int)s->active.size() < kMaxJobs) {
            const uint64_t id = s->queue.front();
            Request& r = s->reqs[id];
            const SrvGraph& sg = s->graphs[r.graph];
            const bool full = r.algo == GS_ALGO_BFS ? (sg.fv && sg.used == ~0ull) : s->side_free.empty();
            if (full) {
                wait.push_back(id);
                s->queue.pop_front();
                continue;
            }
            const size_t need = footprint(s, r);
            if (s->used + need > s->budget && !s->active.empty()) break;
            const gs_status st = admit(s, r);
            if (st != GS_OK) {
                s->queue.insert(s->queue.begin(), wait.begin(), wait.end());
                return st;
            }
            s->active.push_back(r.id);
            s->queue.pop_front();
        }
        s->queue.insert(s->queue.begin(), wait.begin(), wait.end());
    }
    // the step runs while the host tends the side requests (their chunks run
    // beside it on the lower-priority streams)
    std::vector<int> group_job;
    bool launched = false;
    phase_end(0);
    GS_TRY(bfs_launch(s, group_job, &launched));
    phase_end(1);
    gs_status st = side_step(s);
    phase_end(2);
    if (launched) {
        const gs_status st2 = bfs_finish(s, group_job);   // a launched step is always finished
        if (st == GS_OK) st = st2;
    }
    phase_end(3);
    s->phase_s[3] -= s->side_in_wait_s;
    s->phase_s[2] += s->side_in_wait_s;
    s->side_in_wait_s = 0;
    if (st != GS_OK) return st;
    if (n_active) *n_active = (int)s->active.size();
    if (n_queued) *n_queued = (int)s->queue.size();
    return GS_OK;
}

gs_status gs_serve_completed(gs_server* s, uint64_t* ids, int max_ids, int* n) {
    if (!s || !n || max_ids < 0 || (max_ids && !ids)) return GS_ERR_ARG;
    int k = 0;
    while (k < max_ids && !s->completed.empty()) {
        ids[k++] = s->completed.front();
        s->completed.pop_front();
    }
    *n = k;
    return GS_OK;
}

gs_status gs_serve_set_side_streams(gs_server* s, int n) {
    if (!s || n < 1 || n > kSideStreams) return GS_ERR_ARG;
    for (uint64_t id : s->active)
        if (s->reqs[id].side >= 0) return gs_fail(s->ctx, GS_ERR_STATE, "side requests in flight");
    s->n_side = n;
    return GS_OK;
}

gs_status gs_serve_poll(gs_server* s, uint64_t request_id, int* state) {
    if (!s || !state) return GS_ERR_ARG;
    auto it = s->reqs.find(request_id);
    if (it == s->reqs.end()) return gs_fail(s->ctx, GS_ERR_ARG, "unknown request");
    *state = it->second.state;
    return GS_OK;
}

gs_status gs_serve_result(gs_server* s, uint64_t request_id, void* host_dst, uint64_t bytes, double* t_submit,
                          double* t_done, int64_t* steps) {
    if (!s) return GS_ERR_ARG;
    auto it = s->reqs.find(request_id);
    if (it == s->reqs.end()) return gs_fail(s->ctx, GS_ERR_ARG, "unknown request");
    Request& r = it->second;
    if (r.state == kQueued || r.state == kActive) return gs_fail(s->ctx, GS_ERR_STATE, "request not finished");
    if (t_submit) *t_submit = r.t_submit;
    if (t_done) *t_done = r.t_done;
    if (steps) *steps = r.steps;
    if (r.state == kFailed) {
        const gs_status st = r.status;
        s->reqs.erase(it);
        return gs_fail(s->ctx, st, "request failed");
    }
    if (host_dst) {
        if (bytes < r.result_bytes)
            return gs_fail(s->ctx, GS_ERR_ARG, "destination too small: need " + std::to_string(r.result_bytes));
        std::memcpy(host_dst, r.result->p, r.result_bytes);
    }
    s->reqs.erase(it);
    return GS_OK;
}

gs_status gs_serve_result_view(gs_server* s, uint64_t request_id, const void** data, uint64_t* bytes,
                               double* t_submit, double* t_done, int64_t* steps) {
    if (!s || !data || !bytes) return GS_ERR_ARG;
    auto it = s->reqs.find(request_id);
    if (it == s->reqs.end()) return gs_fail(s->ctx, GS_ERR_ARG, "unknown request");
    Request& r = it->second;
    if (r.state == kQueued || r.state == kActive) return gs_fail(s->ctx, GS_ERR_STATE, "request not finished");
    if (t_submit) *t_submit = r.t_submit;
    if (t_done) *t_done = r.t_done;
    if (steps) *steps = r.steps;
    if (r.state == kFailed) {
        const gs_status st = r.status;
        s->reqs.erase(it);
        return gs_fail(s->ctx, st, "request failed");
    }
    *data = r.result->p;
    *bytes = r.result_bytes;
    return GS_OK;
}

gs_status gs_serve_release(gs_server* s, uint64_t request_id) {
    if (!s) return GS_ERR_ARG;
    auto it = s->reqs.find(request_id);
    if (it == s->reqs.end()) return gs_fail(s->ctx, GS_ERR_ARG, "unknown request");
    if (it->second.state == kQueued || it->second.state == kActive)
        return gs_fail(s->ctx, GS_ERR_STATE, "request not finished");
    s->reqs.erase(it);   // the pinned buffer returns to the pool with its last holder
    return GS_OK;
}

gs_status gs_serve_clock(const gs_server* s, double* seconds) {
    if (!s || !seconds) return GS_ERR_ARG;
    *seconds = now_s(s);
    return GS_OK;
}

gs_status gs_serve_stats(const gs_server* s, uint64_t* steps, uint64_t* graph_launches, uint64_t* kernel_launches,
                         uint64_t* hbm_in_use) {
    if (!s) return GS_ERR_ARG;
    if (steps) *steps = s->steps_run;
    if (graph_launches) *graph_launches = s->graph_launches;
    if (kernel_launches) *kernel_launches = s->kernel_launches;
    if (hbm_in_use) *hbm_in_use = s->used;
    return GS_OK;
}

gs_status gs_serve_profile(const gs_server* s, double* seconds, int n) {
    if (!s || !seconds || n < 0) return GS_ERR_ARG;
    for (int k = 0; k < n && k < 8; ++k) seconds[k] = s->phase_s[k];
    return GS_OK;
}

gs_status gs_serve_reserve_host(gs_server* s, uint64_t bytes) {
    if (!s) return GS_ERR_ARG;
    if (bytes == 0) return GS_OK;
    return arena_grow(s, bytes, false);
}

gs_status gs_serve_free(gs_server* s) {
    if (!s) return GS_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (int k = 0; k < kSideStreams; ++k)
        if (s->side_stream[k]) cudaStreamSynchronize(s->side_stream[k]);
    s->reqs.clear();   // drops result buffers into the host pool
    if (s->step_exec) cudaGraphExecDestroy(s->step_exec);
    if (s->step_graph) cudaGraphDestroy(s->step_graph);
    for (auto& pb : s->dev_all) gs_pool_put(s->ctx, pb.first, pb.second);
    for (auto& c : s->host_chunks) cudaFreeHost(c.first);
    gs_dev_free(s->d_table);
    gs_dev_free(s->d_cnt);
    if (s->h_table) cudaFreeHost(s->h_table);
    if (s->h_cnt) cudaFreeHost(s->h_cnt);
    if (s->stream) cudaStreamDestroy(s->stream);
    for (int k = 0; k < kSideStreams; ++k)
        if (s->side_stream[k]) cudaStreamDestroy(s->side_stream[k]);
    for (int k = 0; k < kSideSlots; ++k)
        if (s->side_ev[k]) cudaEventDestroy(s->side_ev[k]);
    if (s->h_flags) cudaFreeHost(s->h_flags);
    delete s;
    return GS_OK;
}

}  // extern "C"
