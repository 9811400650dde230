// Serving loop (sm_100a): BFS / WCC / k-core / PageRank requests against
// resident graphs, admitted by HBM footprint and batched continuously.
//
// The reference answers one query per process run (gstore.cpp:250-333).
// Here a server keeps many requests in flight and advances all of them one
// iteration per step:
//
//   step = [ table upload | counter reset | sweep kernel | post kernel |
//            counter readback ]
//
// captured once as a CUDA graph and replayed every step; the host rewrites
// the job table (pinned) between steps.  The sweep kernel walks the
// concatenated run lists of every job, the post kernel the concatenated
// 32-vertex words, so requests on graphs of different sizes share each
// launch.  Jobs:
//   BFS     one job per graph: up to 64 requests as bits of 64-bit frontier
//           words (a multi-source BFS whose requests start at different
//           steps; each bit keeps its own level), sweep = bfs_onepart for
//           all bits (bfs.cpp:138-185), post = iteration_finalize
//           (bfs.cpp:187-224)
//   WCC     sweep = hooking (wcc.cpp:177-278), post = pointer jumping
//           (wcc.cpp:372-390); done when a sweep changes nothing
//   k-core  post = round (kcore.cpp:179-217; the first step is a round
//           only, as kcore_mmap starts with iteration_finalize), sweep =
//           decrements (kcore.cpp:63-177); done when a round removes nothing
//   PR      not a table job: each step runs its row-slice sweep
//           (pagerank_onepart, pr.cpp:119-154) and update (pr.cpp:229-303)
//           on a lower-priority side stream beside the step graph; done
//           after `arg` iterations
// Between steps the host retires finished requests (their results are
// copied to pinned host buffers), admits queued ones while their state fits
// the HBM budget and a slot is free, and attaches a request to an identical
// one already queued or running (same graph, algorithm and argument).
#include "gs_internal.cuh"
#include "gs_ops.cuh"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <new>
#include <unordered_map>
#include <vector>

namespace {

using namespace gsops;

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kSlots = 64;
constexpr int kMaxJobs = 256;
constexpr int kCounters = 4;

enum JobKind : int { kJobBfs = 0, kJobWcc = 1, kJobKcore = 2 };
constexpr int kFlagFirst = 1;      // WCC: first sweep (labels every end); k-core: round only

typedef FvPair<unsigned long long> Fv64;

struct Job {
    const gs_tile_run* runs;
    const gs_unit* units;
    const uint32_t* rec;
    uint64_t R, words, N, V;
    uint64_t run_beg, word_beg;   // offsets in the concatenated lists
    uint32_t nw;
    int kind, flags, k, directed;
    // BFS group
    Fv64* fv;
    unsigned long long* next;
    uint8_t* depth;               // [N][64]
    uint8_t* act_cur;
    uint8_t* act_next;
    // WCC
    uint32_t* parent;
    uint8_t* touched;
    // k-core
    int32_t* deg;
    uint32_t* removed;
    unsigned long long* cnt;      // kCounters per job
    uint8_t level[kSlots];        // BFS: frontier depth per slot (0 = slot idle)
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

__global__ void __launch_bounds__(kThreads) serve_sweep_kernel(const Table* __restrict__ t) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n_jobs = t->n_jobs;
    // the flags the post kernel sets start empty
    for (int j = blockIdx.x; j < n_jobs; j += gridDim.x) {
        const Job& jb = t->jobs[j];
        if (jb.act_next)
            for (uint32_t w = threadIdx.x; w < jb.nw; w += blockDim.x) jb.act_next[w] = 0;
    }
    for (uint64_t x = blockIdx.x; x < t->total_runs; x += gridDim.x) {
        const Job& jb = t->jobs[job_of(t, x, false)];
        const gs_tile_run run = jb.runs[x - jb.run_beg];
        switch (jb.kind) {
            case kJobBfs: {
                const uint32_t row = jb.units[run.unit_beg].rc >> 16;
                const bool ar = jb.act_cur[row] != 0;
                const MsOp<unsigned long long> op{jb.fv, jb.next, jb.directed};
                for (uint32_t ui = run.unit_beg + warp; ui < run.unit_end; ui += kWarps) {
                    const gs_unit d = jb.units[ui];
                    if (!ar && (jb.directed || !jb.act_cur[d.rc & 0xFFFFu])) continue;
                    sweep_unit(d, jb.rec, op, lane);
                }
                break;
            }
            case kJobWcc: {
                const WccOp op{jb.parent, (jb.flags & kFlagFirst) ? jb.touched : nullptr, jb.cnt};
                for (uint32_t ui = run.unit_beg + warp; ui < run.unit_end; ui += kWarps)
                    sweep_unit(jb.units[ui], jb.rec, op, lane);
                break;
            }
            case kJobKcore: {
                if (jb.flags & kFlagFirst) break;
                const KcoreOpL2 op{jb.deg, jb.removed, jb.act_cur};
                for (uint32_t ui = run.unit_beg + warp; ui < run.unit_end; ui += kWarps)
                    sweep_unit(jb.units[ui], jb.rec, op, lane);
                break;
            }
            default:
                break;
        }
    }
}

__global__ void __launch_bounds__(kThreads) serve_post_kernel(const Table* __restrict__ t) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t gwarp = (uint64_t)blockIdx.x * kWarps + warp;
    const uint64_t nwarps = (uint64_t)gridDim.x * kWarps;
    for (uint64_t x = gwarp; x < t->total_words; x += nwarps) {
        const Job& jb = t->jobs[job_of(t, x, true)];
        const uint64_t w = x - jb.word_beg;
        const uint64_t v = w * 32 + lane;
        switch (jb.kind) {
            case kJobBfs: {
                const unsigned long long nx = jb.next[v];
                const Fv64 s = load_fv(jb.fv + v);
                unsigned long long fresh = 0, over = 0;
                if (nx || s.f) {
                    if (nx) jb.next[v] = 0;
                    fresh = nx & ~s.vis;
                    store_fv(jb.fv + v, fresh, s.vis | fresh);
                    if (fresh) {
                        jb.act_next[v >> 16] = 1;
                        unsigned long long m = fresh;
                        while (m) {
                            const int q = __ffsll((long long)m) - 1;
                            const int d = jb.level[q] + 1;
                            if (d >= 255) over |= 1ull << q;   // bfs.cpp level limit (u8 depth_t)
                            else jb.depth[v * kSlots + q] = (uint8_t)d;
                            m &= m - 1;
                        }
                    }
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    fresh |= __shfl_xor_sync(kFull, fresh, o);
                    over |= __shfl_xor_sync(kFull, over, o);
                }
                if (lane == 0) {
                    if (fresh) atomicOr(jb.cnt + 0, fresh);
                    if (over) atomicOr(jb.cnt + 1, over);
                }
                break;
            }
            case kJobWcc: {
                const uint32_t r = find_root(jb.parent, (uint32_t)v);
                if (r != v) jb.parent[v] = r;
                break;
            }
            case kJobKcore: {
                const int16_t m = (int16_t)jb.deg[v];      // kcore.cpp:189
                const bool gone = m < jb.k && m > 0;
                if (gone) jb.deg[v] = 0;
                const uint32_t bits = __ballot_sync(kFull, gone);
                if (lane == 0) {
                    jb.removed[w] = bits;
                    if (bits) {
                        jb.act_next[w >> 11] = 1;
                        atomicAdd(jb.cnt, (unsigned long long)__popc(bits));
                    }
                }
                break;
            }
            default:
                break;
        }
    }
}

// Admission: request q of a BFS group starts at `root` (bfs.cpp:70).
__global__ void serve_seed_bfs(Fv64* fv, uint8_t* depth, uint8_t* act_cur, uint64_t root, int q) {
    fv[root].f |= 1ull << q;
    fv[root].vis |= 1ull << q;
    depth[root * kSlots + q] = 1;
    act_cur[root >> 16] = 1;
}

// Retirement of BFS slot q: its depth column out, column and visited bit
// cleared for the next request in the slot.
__global__ void serve_take_bfs(Fv64* fv, uint8_t* depth, int q, uint8_t* out, uint64_t V, uint64_t N) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    const unsigned long long keep = ~(1ull << q);
    for (uint64_t v = tid; v < N; v += nth) {
        const uint8_t d = depth[v * kSlots + q];
        if (v < V) out[v] = d;
        if (d) {
            depth[v * kSlots + q] = 0;
            fv[v].vis &= keep;
            fv[v].f &= keep;
        }
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
    uint8_t* out = nullptr;           // BFS result staging (V bytes)
    uint32_t* out32 = nullptr;        // WCC labels staging (4 V bytes)
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
    int* err = nullptr;                  // PageRank: bounded-wait flag of its sweeps
    unsigned long long* cnt = nullptr;
    std::shared_ptr<HostBuf> result;     // pinned host copy of the result
    uint64_t result_bytes = 0;
};

}  // namespace

struct gs_server {
    gs_ctx* ctx = nullptr;
    uint64_t budget = 0;
    uint64_t used = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t pr_stream = nullptr;    // PageRank sweeps, beside the step graph
    cudaEvent_t ev_step = nullptr, ev_pr = nullptr;
    cudaGraphExec_t step_exec = nullptr;
    cudaGraph_t step_graph = nullptr;
    Table* h_table = nullptr;            // pinned
    Table* d_table = nullptr;
    unsigned long long* h_cnt = nullptr; // pinned, kMaxJobs x kCounters
    unsigned long long* d_cnt = nullptr;
    std::vector<SrvGraph> graphs;
    std::unordered_map<uint64_t, Request> reqs;
    std::deque<uint64_t> queue;
    std::vector<uint64_t> active;
    uint64_t next_id = 1;
    int step = 0;
    uint64_t steps_run = 0, graph_launches = 0, kernel_launches = 0;
    std::chrono::steady_clock::time_point t0;
    // pools: exact-size free lists
    std::multimap<size_t, void*> dev_free, host_free;
    std::vector<void*> dev_all, host_all;
};

namespace {

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
    GS_TRY(gs_dev_alloc(s->ctx, out, bytes));
    s->dev_all.push_back(*out);
    return GS_OK;
}

void pool_dev_put(gs_server* s, void* p, size_t bytes) {
    if (p) s->dev_free.emplace((bytes + 255) & ~(size_t)255, p);
}

gs_status pool_host(gs_server* s, size_t bytes, void** out) {
    bytes = (bytes + 255) & ~(size_t)255;
    auto it = s->host_free.find(bytes);
    if (it != s->host_free.end()) {
        *out = it->second;
        s->host_free.erase(it);
        return GS_OK;
    }
    GS_CHECK_CUDA(s->ctx, cudaHostAlloc(out, bytes, cudaHostAllocDefault));
    s->host_all.push_back(*out);
    return GS_OK;
}

std::shared_ptr<HostBuf> host_buf(gs_server* s, size_t bytes, gs_status* st) {
    void* p = nullptr;
    *st = pool_host(s, bytes, &p);
    if (*st != GS_OK) return nullptr;
    HostBuf* hb = new HostBuf{p, bytes};
    return std::shared_ptr<HostBuf>(hb, [s](HostBuf* b) {
        s->host_free.emplace((b->bytes + 255) & ~(size_t)255, b->p);
        delete b;
    });
}

inline uint32_t blocks_for(uint64_t n, const gs_ctx* ctx) {
    const uint64_t b = (n + kThreads - 1) / kThreads;
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(b, gs_grid_size(ctx, 16)));
}

size_t group_bytes(const gs_graph* g) {
    return g->N * (sizeof(Fv64) + 8 + kSlots) + 2 * (size_t)g->nw + g->V + 256;
}

// HBM bytes a request adds when admitted.
size_t footprint(const gs_server* s, const Request& r) {
    const SrvGraph& sg = s->graphs[r.graph];
    const gs_graph* g = sg.g;
    switch (r.algo) {
        case GS_ALGO_BFS: return sg.fv ? 0 : group_bytes(g);
        case GS_ALGO_WCC: return g->N * 5 + g->V * 4 + 64;
        case GS_ALGO_KCORE: return g->N * 4 + g->N / 8 + 2 * (size_t)g->nw + 64;
        default: return g->N * 12 + 64;
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
    GS_TRY(pool_dev(s, g->V + 16, (void**)&sg.out));
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
    pool_dev_put(s, sg.out, g->V + 16);
    sg.fv = nullptr;
    sg.next = nullptr;
    sg.depth = nullptr;
    sg.act[0] = sg.act[1] = nullptr;
    sg.out = nullptr;
    s->used -= sg.group_bytes;
    sg.group_bytes = 0;
}

gs_status admit(gs_server* s, Request& r) {
    gs_ctx* ctx = s->ctx;
    SrvGraph& sg = s->graphs[r.graph];
    const gs_graph* g = sg.g;
    const uint64_t N = g->N;
    r.footprint = footprint(s, r);
    switch (r.algo) {
        case GS_ALGO_BFS: {
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
            serve_seed_bfs<<<1, 1, 0, s->stream>>>(sg.fv, sg.depth, sg.act[sg.cur], (uint64_t)r.arg, q);
            s->kernel_launches++;
            break;
        }
        case GS_ALGO_WCC:
            GS_TRY(pool_dev(s, N * 4, (void**)&r.parent));
            GS_TRY(pool_dev(s, N, (void**)&r.touched));
            GS_TRY(pool_dev(s, g->V * 4 + 16, (void**)&r.labels));
            serve_iota<<<blocks_for(N, ctx), kThreads, 0, s->stream>>>(r.parent, N);
            s->kernel_launches++;
            GS_CHECK_CUDA(ctx, cudaMemsetAsync(r.touched, 0, N, s->stream));
            break;
        case GS_ALGO_KCORE:
            GS_TRY(pool_dev(s, N * 4, (void**)&r.deg));
            GS_TRY(pool_dev(s, N / 8, (void**)&r.removed));
            GS_TRY(pool_dev(s, g->nw, (void**)&r.act[0]));
            GS_TRY(pool_dev(s, g->nw, (void**)&r.act[1]));
            GS_CHECK_CUDA(ctx, cudaMemcpyAsync(r.deg, g->d_degree, N * 4, cudaMemcpyDeviceToDevice, s->stream));
            GS_CHECK_CUDA(ctx, cudaMemsetAsync(r.act[0], 0, g->nw, s->stream));
            GS_CHECK_CUDA(ctx, cudaMemsetAsync(r.act[1], 0, g->nw, s->stream));
            break;
        default:
            // PageRank sweeps the graph's row-slice layout (built once)
            if (!g->pr.built) GS_TRY(pr_layout_build(sg.g));
            GS_TRY(pool_dev(s, N * 4, (void**)&r.x));
            GS_TRY(pool_dev(s, N * 4, (void**)&r.y));
            GS_TRY(pool_dev(s, N * 4, (void**)&r.r));
            GS_TRY(pool_dev(s, 256, (void**)&r.err));
            GS_CHECK_CUDA(ctx, cudaMemsetAsync(r.err, 0, 256, s->stream));
            serve_pr_init<<<blocks_for(N, ctx), kThreads, 0, s->stream>>>(r.x, r.y, N, g->V);
            s->kernel_launches++;
            break;
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
            pool_dev_put(s, r.err, 256);
            break;
    }
    r.parent = nullptr;
    r.touched = nullptr;
    r.labels = nullptr;
    r.deg = nullptr;
    r.removed = nullptr;
    r.act[0] = r.act[1] = nullptr;
    r.x = r.y = r.r = nullptr;
    r.err = nullptr;
    s->used -= r.footprint;
    r.footprint = 0;
}

void fill_graph_tables(Job& j, const gs_graph* g) {
    j.runs = g->d_runs_blk ? g->d_runs_blk : g->d_runs;
    j.units = g->d_runs_blk ? g->d_units_blk : g->d_units;
    j.rec = g->d_rec;
    j.R = g->d_runs_blk ? g->R_blk : g->R;
    j.words = g->N / 32;
    j.N = g->N;
    j.V = g->V;
    j.nw = g->nw;
    j.directed = g->directed;
}

// Enqueues the copy of a finished request's result to pinned host memory.
gs_status take_result(gs_server* s, Request& r) {
    gs_ctx* ctx = s->ctx;
    SrvGraph& sg = s->graphs[r.graph];
    const gs_graph* g = sg.g;
    const void* src = nullptr;
    switch (r.algo) {
        case GS_ALGO_BFS:
            serve_take_bfs<<<blocks_for(g->N, ctx), kThreads, 0, s->stream>>>(sg.fv, sg.depth, r.slot, sg.out, g->V,
                                                                                g->N);
            s->kernel_launches++;
            src = sg.out;
            r.result_bytes = g->V;
            break;
        case GS_ALGO_WCC:
            serve_wcc_labels<<<blocks_for(g->V, ctx), kThreads, 0, s->stream>>>(r.parent, r.touched, r.labels,
                                                                                 g->V);
            s->kernel_launches++;
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
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(r.result->p, src, r.result_bytes, cudaMemcpyDeviceToHost, s->stream));
    return GS_OK;
}

gs_status build_step_graph(gs_server* s) {
    gs_ctx* ctx = s->ctx;
    const int grid = (int)gs_grid_size(ctx, 8);
    GS_CHECK_CUDA(ctx, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    cudaMemcpyAsync(s->d_table, s->h_table, sizeof(Table), cudaMemcpyHostToDevice, s->stream);
    cudaMemsetAsync(s->d_cnt, 0, sizeof(unsigned long long) * kMaxJobs * kCounters, s->stream);
    serve_sweep_kernel<<<grid, kThreads, 0, s->stream>>>(s->d_table);
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
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&s->pr_stream, cudaStreamNonBlocking, lo);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_step, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_pr, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&s->h_table, sizeof(Table), cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&s->h_cnt, sizeof(unsigned long long) * kMaxJobs * kCounters,
                                            cudaHostAllocDefault);
    if (e != cudaSuccess) st = gs_cuda_fail(ctx, e, "server set-up");
    if (st == GS_OK) st = gs_dev_alloc(ctx, (void**)&s->d_table, sizeof(Table));
    if (st == GS_OK) st = gs_dev_alloc(ctx, (void**)&s->d_cnt, sizeof(unsigned long long) * kMaxJobs * kCounters);
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
    // the PageRank layout is built here, at set-up, not under a request
    if (!g->pr.built && g->E) GS_TRY(pr_layout_build(g));
    SrvGraph sg;
    sg.g = g;
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

gs_status gs_serve_step(gs_server* s, int* n_active, int* n_queued) {
    if (!s) return GS_ERR_ARG;
    gs_ctx* ctx = s->ctx;
    // admission: FIFO while the state fits the budget and a slot is free
    while (!s->queue.empty() && (int)s->active.size() < kMaxJobs) {
        Request& r = s->reqs[s->queue.front()];
        const SrvGraph& sg = s->graphs[r.graph];
        if (r.algo == GS_ALGO_BFS && sg.fv && sg.used == ~0ull) break;
        const size_t need = footprint(s, r);
        if (s->used + need > s->budget && !s->active.empty()) break;
        GS_TRY(admit(s, r));
        s->active.push_back(r.id);
        s->queue.pop_front();
    }
    if (!s->active.empty()) {
        // one job per BFS group, one per other request
        Table* t = s->h_table;
        int nj = 0;
        uint64_t runs = 0, words = 0;
        std::vector<int> group_job(s->graphs.size(), -1);
        // PageRank requests: one row-slice sweep and one update each, on the
        // side stream, overlapping the step graph
        bool any_pr = false;
        for (uint64_t id : s->active) {
            Request& r = s->reqs[id];
            if (r.algo != GS_ALGO_PAGERANK) continue;
            if (!any_pr) {   // after this step's admissions (their init kernels)
                GS_CHECK_CUDA(ctx, cudaEventRecord(s->ev_step, s->stream));
                GS_CHECK_CUDA(ctx, cudaStreamWaitEvent(s->pr_stream, s->ev_step, 0));
            }
            any_pr = true;
            gs_graph* g = s->graphs[r.graph].g;
            GS_TRY(pr_slice_sweep(g, s->pr_stream, r.x, r.y, r.err));
            GS_TRY(pr_finalize_launch(ctx, s->pr_stream, r.x, r.y, r.r, g->d_degree, g->N, g->V, 0));
            s->kernel_launches += 2;
            r.job = -1;
        }
        if (any_pr) GS_CHECK_CUDA(ctx, cudaEventRecord(s->ev_pr, s->pr_stream));
        for (uint64_t id : s->active) {
            Request& r = s->reqs[id];
            SrvGraph& sg = s->graphs[r.graph];
            if (r.algo == GS_ALGO_PAGERANK) continue;
            if (r.algo == GS_ALGO_BFS && group_job[r.graph] >= 0) {
                r.job = group_job[r.graph];
                continue;
            }
            Job& j = t->jobs[nj];
            std::memset(&j, 0, sizeof(Job));
            fill_graph_tables(j, sg.g);
            j.run_beg = runs;
            j.word_beg = words;
            j.cnt = s->d_cnt + (size_t)nj * kCounters;
            switch (r.algo) {
                case GS_ALGO_BFS:
                    j.kind = kJobBfs;
                    j.fv = sg.fv;
                    j.next = sg.next;
                    j.depth = sg.depth;
                    j.act_cur = sg.act[sg.cur];
                    j.act_next = sg.act[sg.cur ^ 1];
                    for (int q = 0; q < kSlots; ++q)
                        j.level[q] = (sg.used >> q & 1) ? (uint8_t)std::min(255, s->step - sg.slot_start[q] + 1) : 0;
                    group_job[r.graph] = nj;
                    break;
                case GS_ALGO_WCC:
                    j.kind = kJobWcc;
                    j.flags = r.steps == 0 ? kFlagFirst : 0;
                    j.parent = r.parent;
                    j.touched = r.touched;
                    break;
                case GS_ALGO_KCORE:
                    j.kind = kJobKcore;
                    j.flags = r.steps == 0 ? kFlagFirst : 0;
                    j.k = (int)r.arg;
                    j.deg = r.deg;
                    j.removed = r.removed;
                    j.act_cur = r.act[r.cur];
                    j.act_next = r.act[r.cur ^ 1];
                    break;
                default:
                    break;
            }
            r.job = nj;
            runs += j.R;
            words += j.words;
            ++nj;
        }
        t->n_jobs = nj;
        t->total_runs = runs;
        t->total_words = words;
        GS_CHECK_CUDA(ctx, cudaGraphLaunch(s->step_exec, s->stream));
        if (any_pr) GS_CHECK_CUDA(ctx, cudaStreamWaitEvent(s->stream, s->ev_pr, 0));
        GS_CHECK_CUDA(ctx, cudaStreamSynchronize(s->stream));
        s->graph_launches++;
        s->kernel_launches += 2;
        s->steps_run++;
        // outcomes
        std::vector<uint64_t> finished;
        std::vector<bool> group_swapped(s->graphs.size(), false);
        for (uint64_t id : s->active) {
            Request& r = s->reqs[id];
            SrvGraph& sg = s->graphs[r.graph];
            const unsigned long long* c = s->h_cnt + (size_t)std::max(r.job, 0) * kCounters;
            r.steps += 1;
            bool done = false;
            switch (r.algo) {
                case GS_ALGO_BFS:
                    if (c[1] >> r.slot & 1) {
                        r.status = GS_ERR_RANGE;
                        done = true;
                    } else {
                        done = !(c[0] >> r.slot & 1);
                    }
                    if (!group_swapped[r.graph]) {
                        sg.cur ^= 1;
                        group_swapped[r.graph] = true;
                    }
                    break;
                case GS_ALGO_WCC: done = c[0] == 0; break;
                case GS_ALGO_KCORE:
                    done = c[0] == 0;
                    r.cur ^= 1;
                    break;
                default: done = r.steps >= r.arg; break;
            }
            if (done) finished.push_back(id);
        }
        s->step += 1;
        if (!finished.empty()) {
            for (uint64_t id : finished) {
                Request& r = s->reqs[id];
                if (r.algo == GS_ALGO_PAGERANK) {
                    int h_err = 0;
                    GS_CHECK_CUDA(ctx, cudaMemcpy(&h_err, r.err, sizeof(int), cudaMemcpyDeviceToHost));
                    if (h_err) r.status = GS_ERR_TIMEOUT;
                }
                if (r.status == GS_OK) GS_TRY(take_result(s, r));
                else if (r.algo == GS_ALGO_BFS) {
                    // clear the slot for its next request (result discarded)
                    SrvGraph& sg = s->graphs[r.graph];
                    serve_take_bfs<<<blocks_for(sg.g->N, ctx), kThreads, 0, s->stream>>>(sg.fv, sg.depth, r.slot, sg.out,
                                                                                         sg.g->V, sg.g->N);
                    s->kernel_launches++;
                }
            }
            GS_CHECK_CUDA(ctx, cudaStreamSynchronize(s->stream));
            const double t = now_s(s);
            for (uint64_t id : finished) {
                Request& r = s->reqs[id];
                r.state = r.status == GS_OK ? kDone : kFailed;
                r.t_done = t;
                release(s, r);
                for (uint64_t f : r.followers) {
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
    }
    if (n_active) *n_active = (int)s->active.size();
    if (n_queued) *n_queued = (int)s->queue.size();
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

gs_status gs_serve_free(gs_server* s) {
    if (!s) return GS_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->pr_stream) cudaStreamSynchronize(s->pr_stream);
    s->reqs.clear();   // drops result buffers into the host pool
    if (s->step_exec) cudaGraphExecDestroy(s->step_exec);
    if (s->step_graph) cudaGraphDestroy(s->step_graph);
    for (void* p : s->dev_all) gs_dev_free(p);
    for (void* p : s->host_all) cudaFreeHost(p);
    gs_dev_free(s->d_table);
    gs_dev_free(s->d_cnt);
    if (s->h_table) cudaFreeHost(s->h_table);
    if (s->h_cnt) cudaFreeHost(s->h_cnt);
    if (s->stream) cudaStreamDestroy(s->stream);
    if (s->pr_stream) cudaStreamDestroy(s->pr_stream);
    if (s->ev_step) cudaEventDestroy(s->ev_step);
    if (s->ev_pr) cudaEventDestroy(s->ev_pr);
    delete s;
    return GS_OK;
}

}  // extern "C"
