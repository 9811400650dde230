// BFS sweep and finalize (sm_100a): the level sweep of bfs.cpp:138-185.
//
// Per-vertex state in HBM (L2-resident for the graph sizes of interest):
//   st[v >> 4]  2 bits per vertex, frontier (depth == level) and visited
//               (depth != 0), 16 KB per 2^16-vertex window: in a word of 16
//               vertices, vertex k's frontier bit is bit k and its visited bit
//               bit k + 16 when the word index is even, and the other way
//               round when it is odd, so that one 32-bit rotation by v & 31
//               brings any vertex's frontier bit to bit 0 and its visited bit
//               to bit 16
//   next[v>>5]  discovered during this sweep
//   depth[v]    u8, written by the finalize for new vertices
//
// A CTA sweeps one run at a time (consecutive tiles of one tile row inside
// a group, <= kRunRecords records), taking the next run from an atomic
// ticket so that CTAs that drew short runs take more of them (run sizes
// range from a few records to kRunRecords).  The row window's state (16 KB) is
// brought into shared memory once per run with one cp.async.bulk copy; the
// run's units (tile slices of <= kUnitRecords records) are spread over the
// warps, each warp streaming its unit's records with 128-bit evict-first
// loads, each lane loading its next 2 x 16 bytes before it visits the
// current ones and classifying four records before it acts on any of them
// (the discovery path is one branch per four records, its reductions
// predicated rather than branched around).  Per record: the row
// end's state comes from shared memory, the
// column end's from global memory through L1 — tiles written by the device
// converter are sorted by column offset, so the 32 lookups of a warp fall
// on a few neighbouring lines.  A discovered row end sets a bit in a
// shared bitmap OR-ed into `next` once per run (its non-zero words); a
// discovered column end goes straight to `next`.  No barrier between tiles.
//
// Reference rule kept: a tile is swept when its row window (or, half grid,
// its column window) holds a frontier vertex (grid::bfs_mmap,
// gstore.cpp:2671-2698); a record discovers its unvisited end from its
// frontier end (bfs.cpp:158-177).  Depth values do not depend on the order
// in which records are visited, so the result is the reference's.
#include "gs_internal.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr uint32_t kStWords = 4096;           // 2-bit state words per window
constexpr uint32_t kStBytes = kStWords * 4;   // 16 KB
constexpr uint32_t kNxWords = 2048;           // 1-bit words per window
constexpr long long kWaitLimit = 1ll << 24;   // bounded mbarrier waits

struct __align__(128) BfsSmem {
    uint32_t strow[kStWords];
    uint32_t nx[kNxWords];
    unsigned long long bar;
    unsigned long long cur;   // the run drawn by thread 0
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Bounded wait for the phase with the given parity; false on timeout.
__device__ __forceinline__ bool bar_wait(unsigned long long* bar, uint32_t parity) {
    const uint32_t a = smem_addr(bar);
    for (long long i = 0; i < kWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Predicated reductions: the OR is issued only where cond is non-zero, with
// no branch around it.
__device__ __forceinline__ void red_or_if(uint32_t* p, uint32_t v, uint32_t cond) {
    asm volatile("{\n.reg .pred q;\nsetp.ne.u32 q, %2, 0;\n@q red.global.or.b32 [%0], %1;\n}" ::"l"(p), "r"(v),
                 "r"(cond)
                 : "memory");
}
__device__ __forceinline__ void red_or_shared_if(uint32_t* p, uint32_t v, uint32_t cond) {
    asm volatile("{\n.reg .pred q;\nsetp.ne.u32 q, %2, 0;\n@q red.shared.or.b32 [%0], %1;\n}" ::"r"(smem_addr(p)),
                 "r"(v), "r"(cond)
                 : "memory");
}

struct RunArgs {
    const gs_tile_run* runs;
    uint64_t n_runs;
    const gs_unit* units;
    const uint32_t* rec;
    const uint32_t* st;
    uint32_t* next;
    const uint8_t* act;
    uint8_t* act_next;
    int directed;
    int* error;
    const gs_seg_run* seg;   // segment sweep: entries to sweep (records at rec + delta), else null
    // [0] next run, [1] CTAs finished; zero at launch, the last CTA to
    // finish zeroes them again for the next launch on the stream
    unsigned int* ticket;
    // per unit, bit c: chunk c of the unit (its 16-byte groups 64c..64c+63,
    // chunk 0 with the unaligned head and tail records) holds no record
    // with an unvisited end, so it can discover nothing for the rest of the
    // BFS (visited bits are never cleared); null: every chunk is read
    uint8_t* dead;
    unsigned long long* read;   // kSkip: records read by the launch are added here (null: not counted)
};

// Five CTAs per SM (40 warps, a 48-register cap): with the predicated
// discovery, six CTAs at 40 registers spilled more and measured 4 % slower.
// kMark: a chunk whose records all have both ends visited at the start of
// the level is marked dead (a.dead) for the levels after it.  kSkip: dead
// chunks are not read (set once a level has marked some).  Without either,
// the unit loop is the plain one.
template <bool kMark, bool kSkip>
__global__ void __launch_bounds__(kThreads, kBfsCtasPerSm) bfs_run_kernel(RunArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    BfsSmem& m = *reinterpret_cast<BfsSmem*>(smem_raw);
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&m.bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (uint32_t w = tid; w < kNxWords; w += kThreads) m.nx[w] = 0;
    __syncthreads();
    uint32_t parity = 0;
    uint32_t nread = 0;   // kSkip, lane 0: records this warp read
    auto draw = [&]() -> uint64_t {
        // every thread has read the previous draw: a barrier lies between
        if (tid == 0) m.cur = atomicAdd(a.ticket, 1u);
        __syncthreads();
        return m.cur;
    };

    for (uint64_t i = draw(); i < a.n_runs; i = draw()) {
        uint32_t ub, ue;
        const uint32_t* rec = a.rec;
        if (a.seg) {
            const gs_seg_run e = a.seg[i];
            ub = e.unit_beg;
            ue = e.unit_end;
            rec = a.rec + e.delta;
        } else {
            ub = a.runs[i].unit_beg;
            ue = a.runs[i].unit_end;
        }
        const uint32_t row = a.units[ub].rc >> 16;
        const bool ar = a.act[row] != 0;
        // the run is swept when its row window or any column window is active
        int any = ar ? 1 : 0;
        if (!ar && !a.directed)
            for (uint32_t ui = ub + tid; ui < ue; ui += kThreads)
                any |= a.act[a.units[ui].rc & 0xFFFFu] != 0;
        if (!__syncthreads_or(any)) continue;

        if (tid == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&m.bar)),
                         "r"(kStBytes)
                         : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_addr(m.strow)),
                "l"(a.st + ((size_t)row << 12)), "r"(kStBytes), "r"(smem_addr(&m.bar))
                : "memory");
        }
        const bool got = bar_wait(&m.bar, parity);
        parity ^= 1;
        if (!__syncthreads_and(got)) {
            // the copy is late: flag it and give it one more bounded wait, so
            // that the CTA does not leave with its copy still in flight
            if (tid == 0) {
                atomicExch(a.error, 1);
                bar_wait(&m.bar, parity ^ 1);
            }
            break;   // uniform
        }
        const uint32_t mr = ar ? 1u << 16 : 0u;
        for (uint32_t ui = ub + warp; ui < ue; ui += kWarps) {
            const gs_unit d = a.units[ui];
            const uint32_t col = d.rc & 0xFFFFu;
            const uint32_t mc = (!a.directed && a.act[col]) ? 1u : 0u;
            if (!mr && !mc) continue;                       // warp-uniform
            const uint32_t* colst = a.st + ((size_t)col << 12);
            uint32_t* next_col = a.next + ((size_t)col << 11);
            uint32_t hit = 0;
            // class bit 16: the column end is discovered (row end in the
            // frontier, column end unvisited, bfs.cpp:158-164); bit 0: the
            // row end (bfs.cpp:166-172).  The rotations take their amount mod
            // 32, so the row end rotated by v0 ^ 16 has its frontier bit at
            // 16 and visited bit at 0, the column end rotated by v1 the other
            // way round, and one AND-NOT per direction gives the class.
            // allv bit 0 stays set while every record classified has both
            // ends visited (row end's visited bit 0, column end's bit 16)
            uint32_t allv = ~0u;
            auto classify = [&](uint32_t r) -> uint32_t {
                const uint32_t w0 = m.strow[(r & 0xFFFFu) >> 4];
                const uint32_t w1 = __ldg(colst + (r >> 20));
                const uint32_t s0 = __funnelshift_r(w0, w0, r ^ 16u);
                const uint32_t s1 = __funnelshift_r(w1, w1, r >> 16);
                if constexpr (kMark) allv &= s0 & (s1 >> 16);
                return (s0 & ~s1 & mr) | (s1 & ~s0 & mc);
            };
            auto discover = [&](uint32_t r, uint32_t c) {
                const uint32_t v0 = r & 0xFFFFu, v1 = r >> 16;
                red_or_if(next_col + (v1 >> 5), 1u << (v1 & 31), c >> 16);
                red_or_shared_if(m.nx + (v0 >> 5), 1u << (v0 & 31), c & 1u);
                hit |= c >> 16;
            };
            auto visit = [&](uint32_t r) {
                const uint32_t c = classify(r);
                if (c) discover(r, c);
            };
            // four records classified before any is acted on: one branch
            // per four records in a level that discovers little
            auto visit4 = [&](const uint4 q) {
                const uint32_t c0 = classify(q.x), c1 = classify(q.y), c2 = classify(q.z), c3 = classify(q.w);
                if (c0 | c1 | c2 | c3) {
                    discover(q.x, c0);
                    discover(q.y, c1);
                    discover(q.z, c2);
                    discover(q.w, c3);
                }
            };
            const uint64_t b = d.rec_beg, e = d.rec_beg + d.n;
            uint64_t ab = (b + 3) & ~3ull;
            if (ab > e) ab = e;
            uint64_t ae = e & ~3ull;
            if (ae < ab) ae = ab;
            const uint4* r4 = reinterpret_cast<const uint4*>(rec + ab);
            const uint32_t n4 = (uint32_t)((ae - ab) >> 2);
            const uint4 z = make_uint4(0, 0, 0, 0);
            if constexpr (!kMark && !kSkip) {
                if (b + lane < ab) visit(__ldcs(rec + b + lane));
                if (ae + lane < e) visit(__ldcs(rec + ae + lane));
                // the next iteration's records are loaded before this one's
                // are visited, so the loads overlap the lookups
                uint4 q0 = lane < n4 ? __ldcs(r4 + lane) : z;
                uint4 q1 = lane + 32 < n4 ? __ldcs(r4 + lane + 32) : z;
                for (uint32_t k = lane; k < n4; k += 64) {
                    const uint4 p0 = k + 64 < n4 ? __ldcs(r4 + k + 64) : z;
                    const uint4 p1 = k + 96 < n4 ? __ldcs(r4 + k + 96) : z;
                    visit4(q0);
                    if (k + 32 < n4) visit4(q1);
                    q0 = p0;
                    q1 = p1;
                }
            } else {
                // chunks of 64 16-byte groups (<= 8 per unit), chunk 0 with
                // the unaligned head and tail; the live ones are read (all of
                // them without kSkip), the next one's records loaded before
                // this one's are visited
                const uint32_t nch = n4 ? (n4 + 63) >> 6 : 1;
                const uint32_t dead = kSkip ? (uint32_t)__ldcg(a.dead + ui) : 0u;
                uint32_t todo = ((1u << nch) - 1u) & ~dead;
                if (!(dead & 1u)) {
                    if (b + lane < ab) visit(__ldcs(rec + b + lane));
                    if (ae + lane < e) visit(__ldcs(rec + ae + lane));
                    if (kSkip && lane == 0) nread += (uint32_t)((ab - b) + (e - ae));
                }
                int c = todo ? __ffs(todo) - 1 : -1;
                uint4 q0 = z, q1 = z;
                if (c >= 0) {
                    const uint32_t k = ((uint32_t)c << 6) + lane;
                    q0 = k < n4 ? __ldcs(r4 + k) : z;
                    q1 = k + 32 < n4 ? __ldcs(r4 + k + 32) : z;
                }
                uint32_t newdead = 0;
                while (c >= 0) {   // warp-uniform: todo comes from one byte read by every lane
                    todo &= todo - 1;
                    const int cn = todo ? __ffs(todo) - 1 : -1;
                    uint4 p0 = z, p1 = z;
                    if (cn >= 0) {
                        const uint32_t kn = ((uint32_t)cn << 6) + lane;
                        p0 = kn < n4 ? __ldcs(r4 + kn) : z;
                        p1 = kn + 32 < n4 ? __ldcs(r4 + kn + 32) : z;
                    }
                    const uint32_t k0 = (uint32_t)c << 6;
                    if (k0 + lane < n4) visit4(q0);
                    if (k0 + lane + 32 < n4) visit4(q1);
                    if constexpr (kMark) {
                        if (__all_sync(0xFFFFFFFFu, allv & 1u)) newdead |= 1u << c;
                        allv = ~0u;
                    }
                    if (kSkip && lane == 0) nread += 4u * min(64u, n4 - min(n4, k0));
                    q0 = p0;
                    q1 = p1;
                    c = cn;
                }
                if constexpr (kMark) {
                    if (lane == 0 && newdead)
                        atomicOr(reinterpret_cast<unsigned int*>(a.dead) + (ui >> 2), newdead << ((ui & 3u) << 3));
                }
            }
            if (__any_sync(0xFFFFFFFFu, hit != 0) && lane == 0) a.act_next[col] = 1;   // read_part_next->set_bit_atomic(j)
        }
        __syncthreads();
        // row side: OR the run's discovered words into next, clear them
        bool any_row = false;
        {
            uint32_t* dst = a.next + ((size_t)row << 11);
            for (uint32_t k = tid; k < kNxWords; k += kThreads) {
                const uint32_t x = m.nx[k];
                if (x) {
                    any_row = true;
                    atomicOr(dst + k, x);
                    m.nx[k] = 0;
                }
            }
        }
        if (__syncthreads_or(any_row) && tid == 0) a.act_next[row] = 1;        // read_part_next->set_bit_atomic(i)
    }
    if (kSkip && a.read && lane == 0 && nread) atomicAdd(a.read, (unsigned long long)nread);
    if (tid == 0 && atomicAdd(a.ticket + 1, 1u) == gridDim.x - 1) {
        // every CTA has drawn its last ticket
        atomicExch(a.ticket, 0u);
        atomicExch(a.ticket + 1, 0u);
    }
}

// Per 32 vertices: new = next & ~visited; frontier := new; visited |= new;
// depth[v] = level + 1 for new vertices; next := 0 (iteration_finalize,
// bfs.cpp:187-224 — the level count is exact here).
__global__ void bfs_finalize_kernel(uint32_t* __restrict__ st, uint32_t* __restrict__ next,
                                    uint8_t* __restrict__ depth, uint64_t n_words, uint8_t next_level,
                                    unsigned long long* count) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    uint64_t local = 0;
    for (uint64_t w = tid; w < n_words; w += nth) {
        const uint32_t nx = next[w];
        const uint2 s = reinterpret_cast<const uint2*>(st)[w];
        if (nx) next[w] = 0;
        // even word: F in bits 0-15, VIS in bits 16-31; odd word swapped
        const uint32_t vis = (s.x >> 16) | (s.y << 16);
        const uint32_t fr = (s.x & 0xFFFFu) | (s.y & 0xFFFF0000u);
        const uint32_t fresh = nx & ~vis;
        if (fresh == 0 && fr == 0) continue;
        const uint32_t nv = vis | fresh;
        reinterpret_cast<uint2*>(st)[w] = make_uint2((fresh & 0xFFFFu) | (nv << 16), (nv >> 16) | (fresh & 0xFFFF0000u));
        uint32_t x = fresh;
        while (x) {
            const int k = __ffs(x) - 1;
            depth[w * 32 + k] = next_level;
            x &= x - 1;
        }
        local += __popc(fresh);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xFFFFFFFFu, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(count, (unsigned long long)local);
}

// Vertices with at least one record (degree > 0).
__global__ void count_nonisolated_kernel(const int32_t* __restrict__ degree, uint64_t V, unsigned long long* out) {
    unsigned long long local = 0;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x)
        local += degree[v] != 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xFFFFFFFFu, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(out, local);
}

__global__ void bfs_seed_kernel(uint8_t* depth, uint32_t* st, uint8_t* act, uint64_t root) {
    depth[root] = 1;                                 // bfs.cpp:70
    st[root >> 4] = 0x10001u << (root & 15);         // frontier + visited
    act[root >> 16] = 1;                             // calc_part_needed, bfs.cpp:324-338
}

inline uint32_t blocks_for(uint64_t n, const gs_ctx* ctx) {
    uint64_t b = (n + 255) / 256;
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(b, gs_grid_size(ctx, 16)));
}

}  // namespace

gs_status gs_graph_nonisolated(gs_graph* g) {
    if (g->nonisolated_known || !g->d_degree) return GS_OK;   // counted once per graph
    gs_ctx* ctx = g->ctx;
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_scalars, 0, sizeof(uint64_t), ctx->stream));
    count_nonisolated_kernel<<<blocks_for(g->V, ctx), 256, 0, ctx->stream>>>(g->d_degree, g->V,
                                                                             (unsigned long long*)ctx->d_scalars);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->h_scalars, ctx->d_scalars, sizeof(uint64_t), cudaMemcpyDeviceToHost,
                                       ctx->stream));
    GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    g->nonisolated = ctx->h_scalars[0];
    g->nonisolated_known = true;
    return GS_OK;
}

gs_status bfs_init(gs_state* s) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    const uint64_t words = g->N / 32;
    if (!s->d_depth) GS_TRY(gs_state_alloc(s, (void**)&s->d_depth, g->N));
    if (!s->d_front) GS_TRY(gs_state_alloc(s, (void**)&s->d_front, words * 8));    // 2-bit state
    if (!s->d_visited) GS_TRY(gs_state_alloc(s, (void**)&s->d_visited, words * 4)); // next bitmap
    if (!s->d_act) GS_TRY(gs_state_alloc(s, (void**)&s->d_act, g->nw));
    if (!s->d_act_next) GS_TRY(gs_state_alloc(s, (void**)&s->d_act_next, g->nw));
    if (!s->d_error) GS_TRY(gs_state_alloc(s, (void**)&s->d_error, sizeof(uint64_t)));
    if (!s->d_ticket) GS_TRY(gs_state_alloc(s, (void**)&s->d_ticket, 2 * sizeof(uint32_t)));
    const size_t dead_bytes = ((g->U + 3) & ~(uint64_t)3) + 4;   // whole 32-bit words
    if (!s->d_dead) GS_TRY(gs_state_alloc(s, (void**)&s->d_dead, dead_bytes));
    if (!s->d_read) GS_TRY(gs_state_alloc(s, (void**)&s->d_read, 256 * sizeof(unsigned long long)));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_ticket, 0, 2 * sizeof(uint32_t), ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_dead, 0, dead_bytes, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_read, 0, 256 * sizeof(unsigned long long), ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_depth, 0, g->N, ctx->stream));   // INFTY = 0
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_front, 0, words * 8, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_visited, 0, words * 4, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_act, 0, g->nw, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_act_next, 0, g->nw, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_error, 0, sizeof(uint64_t), ctx->stream));
    bfs_seed_kernel<<<1, 1, 0, ctx->stream>>>(s->d_depth, s->d_front, s->d_act, (uint64_t)s->arg);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    GS_TRY(gs_graph_nonisolated(g));
    s->marking = false;
    s->level_skip.clear();
    s->level = 1;
    s->level_counts.clear();
    s->n_act_hist = 0;
    return GS_OK;
}

gs_status bfs_sweep_begin(gs_state* s) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    // Window flags of this sweep, kept on the device for the swept-record
    // statistics (read back only when asked for: no host round trip here).
    if (!s->d_act_hist) GS_TRY(gs_state_alloc(s, (void**)&s->d_act_hist, (size_t)g->nw * 256));
    if (s->n_act_hist < 256)
        GS_CHECK_CUDA(ctx, cudaMemcpyAsync(s->d_act_hist + (size_t)s->n_act_hist * g->nw, s->d_act, g->nw,
                                           cudaMemcpyDeviceToDevice, ctx->stream));
    s->n_act_hist += 1;
    GS_CHECK_CUDA(ctx, (gs_smem_limit_once<bfs_run_kernel<false, false>>(ctx->device, (int)sizeof(BfsSmem))));
    GS_CHECK_CUDA(ctx, (gs_smem_limit_once<bfs_run_kernel<true, false>>(ctx->device, (int)sizeof(BfsSmem))));
    GS_CHECK_CUDA(ctx, (gs_smem_limit_once<bfs_run_kernel<true, true>>(ctx->device, (int)sizeof(BfsSmem))));
    // Dead chunks: marking starts once at most 1/64 of the vertices with
    // records are still unvisited (after the peak, when most chunks have no
    // record left with an unvisited end) and goes on at every level after
    // it, which also skips the chunks marked so far (a streamed graph's
    // planner then leaves out the units whose chunks are all dead).  Only
    // speed depends on this choice: a dead chunk can discover nothing.
    uint64_t visited = 1;
    for (uint64_t c : s->level_counts) visited += c;
    const uint64_t unvisited = g->nonisolated > visited ? g->nonisolated - visited : 0;
    const bool on = g->nonisolated_known && s->d_dead;
    s->sweep_skip = on && s->marking;
    s->sweep_mark = on && (s->marking || unvisited * 64 <= g->nonisolated);
    if (s->sweep_mark) s->marking = true;
    if (s->level_skip.size() < s->level) s->level_skip.resize(s->level, 0);
    s->level_skip[s->level - 1] = s->sweep_skip ? 1 : 0;
    return GS_OK;
}

gs_status bfs_sweep_launch(gs_state* s) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    // every run of the resident graph, or the entries of the current segment
    const uint64_t n_runs = g->seg.list ? g->seg.n : (g->d_runs_lpt ? g->R_lpt : g->R);
    if (n_runs == 0) return GS_OK;
    // the level's mode (bfs_sweep_begin) holds for every segment of it
    const bool mark = s->sweep_mark, skip = s->sweep_skip;
    uint8_t* dead = mark ? s->d_dead : nullptr;
    RunArgs a{g->d_runs_lpt ? g->d_runs_lpt : g->d_runs, n_runs, g->d_units, g->seg.list ? g->seg.buf : g->d_rec,
              s->d_front, s->d_visited,
              s->d_act, s->d_act_next, g->directed, (int*)s->d_error, g->seg.list, s->d_ticket, dead,
              s->d_read + std::min(s->level - 1, 255)};
    const uint32_t grid = (uint32_t)std::min<uint64_t>(n_runs, gs_grid_size(ctx, kBfsCtasPerSm));
    gs_timer_begin(ctx);
    if (skip) bfs_run_kernel<true, true><<<grid, kThreads, sizeof(BfsSmem), ctx->stream>>>(a);
    else if (mark) bfs_run_kernel<true, false><<<grid, kThreads, sizeof(BfsSmem), ctx->stream>>>(a);
    else bfs_run_kernel<false, false><<<grid, kThreads, sizeof(BfsSmem), ctx->stream>>>(a);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    gs_timer_end(ctx, GS_ALGO_BFS, 0);
    return GS_OK;
}

gs_status bfs_finalize(gs_state* s, int64_t* frontier, int* done) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_scalars, 0, sizeof(uint64_t), ctx->stream));
    const uint64_t words = g->N / 32;
    bfs_finalize_kernel<<<blocks_for(words, ctx), 256, 0, ctx->stream>>>(
        s->d_front, s->d_visited, s->d_depth, words, (uint8_t)(s->level + 1), (unsigned long long*)ctx->d_scalars);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    // swap(read_part, read_part_next); read_part_next->reset() (bfs.cpp:322-324)
    std::swap(s->d_act, s->d_act_next);
    GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_act_next, 0, g->nw, ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->h_scalars, ctx->d_scalars, sizeof(uint64_t), cudaMemcpyDeviceToHost,
                                       ctx->stream));
    GS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->h_scalars + 1, s->d_error, sizeof(uint64_t), cudaMemcpyDeviceToHost,
                                       ctx->stream));
    GS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const uint64_t count = ctx->h_scalars[0];
    if (ctx->h_scalars[1] != 0) return gs_fail(ctx, GS_ERR_TIMEOUT, "BFS sweep: a bounded wait gave up");
    s->level_counts.push_back(count);
    *frontier = (int64_t)count;
    if (count == 0) {
        *done = 1;
        return GS_OK;
    }
    if (s->level == 254) return gs_fail(ctx, GS_ERR_RANGE, "BFS exceeds 254 levels (u8 depth_t)");
    s->level += 1;
    *done = 0;
    return GS_OK;
}

// ------------------------------------------------- caller-provided buffers --
// Launchers over explicit buffers for gs_bfs_noalloc (gs_noalloc.cu): the
// same kernels as above, with the state living wherever the caller says.
gs_status bfs_seed_into(gs_ctx* ctx, uint8_t* depth, uint32_t* st, uint8_t* act, uint64_t root) {
    bfs_seed_kernel<<<1, 1, 0, ctx->stream>>>(depth, st, act, root);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    return GS_OK;
}

gs_status bfs_level_into(gs_ctx* ctx, const gs_graph* g, uint8_t* depth, uint32_t* st, uint32_t* next,
                         uint8_t* act, uint8_t* act_next, unsigned long long* count, int* error,
                         unsigned int* ticket, uint8_t next_level) {
    if (g->R) {
        GS_CHECK_CUDA(ctx, (gs_smem_limit_once<bfs_run_kernel<false, false>>(ctx->device, (int)sizeof(BfsSmem))));
        const uint64_t n_runs = g->d_runs_lpt ? g->R_lpt : g->R;
        RunArgs a{g->d_runs_lpt ? g->d_runs_lpt : g->d_runs, n_runs, g->d_units, g->d_rec, st, next, act, act_next,
                  g->directed, error, nullptr, ticket, nullptr, nullptr};
        const uint32_t grid = (uint32_t)std::min<uint64_t>(n_runs, gs_grid_size(ctx, kBfsCtasPerSm));
        bfs_run_kernel<false, false><<<grid, kThreads, sizeof(BfsSmem), ctx->stream>>>(a);
        GS_CHECK_CUDA(ctx, cudaGetLastError());
        ctx->launches++;
    }
    const uint64_t words = g->N / 32;
    bfs_finalize_kernel<<<blocks_for(words, ctx), 256, 0, ctx->stream>>>(st, next, depth, words, next_level, count);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches++;
    return GS_OK;
}
