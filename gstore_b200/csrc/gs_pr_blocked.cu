// PageRank sweep by propagation blocking (sm_100a): pagerank_onepart
// (pr.cpp:119-154) for a large resident graph.
//
// Per record (v0, v1) of tile (i, j) the reference does
//     rank[v1] += prior[v0];   rank[v0] += prior[v1]   (the second: half grid)
// i.e. every record pushes x of one end into s of the other, once per
// direction.  At Kronecker scale 26 both ends are random over 268 MB arrays,
// so a sweep that touches x and s per record pays two random L2/DRAM
// operations per record, and the L1 pipe that issues them is the limit.
//
// Here a sweep is two streaming passes over a layout built once per graph
// (Beamer, Asanovic, Patterson, "Reducing PageRank Communication via
// Propagation Blocking", IPDPS 2017, restated for the tile grid):
//
//   * entries: one per (record, direction), sorted by (source slice S =
//     src >> 14, destination bin D = dst >> 14, dst, src).  Two u16 streams
//     hold the source's offset in its slice and the destination's offset in
//     its bin; the (S, D) blocks of the stream are contiguous, each padded to
//     a multiple of 8 entries (padding points past every destination);
//   * gather (pass 1): a CTA stages x of one source slice (16,384 floats,
//     64 KB) in shared memory with one bulk copy and streams the slice's
//     entries: val[e] = x[src of e] -- a shared-memory gather, a coalesced
//     16-bit read and a coalesced 32-bit write per entry;
//   * accumulate (pass 2): a CTA owns one destination bin (16,384 floats,
//     64 KB of shared memory), walks the bin's blocks (one per source slice,
//     D-major table, each cut into chunks of at most 256 entries, a
//     half-warp per chunk) and adds val[e] into its shared-memory sums at
//     the destination offset (equal destinations, adjacent in a block, are
//     summed in registers and across lanes first: one atomic per run), then
//     writes the bin's sums to y.
//
// Both passes stream; the random accesses stay in shared memory.  DRAM bytes
// per entry and sweep: 2 (source offset) + 4 + 4 (value written and read) +
// 2 (destination offset) = 12, plus x, y and the block table.  The sums are
// re-associated per bin (FP32), which only changes rounding.
#include "gs_internal.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <vector>

namespace {

constexpr uint32_t kSrcSlice = 1u << kPbSrcBits;   // 16,384
constexpr uint32_t kDstBin = 1u << kPbDstBits;     // 16,384
constexpr int kKeyLowBits = kPbSrcBits + kPbDstBits;
constexpr int kGatherThreads = 512;
constexpr int kGatherCtas = 3;       // resident gather CTAs per SM (64 KB of x each)
constexpr int kGatherGroups = 2;     // 8-entry groups per gather thread and step (two steps in flight)
constexpr int kAccThreads = 512;
constexpr int kAccCtas = 3;          // resident accumulate CTAs per SM (the bin's sums each)
constexpr int kAccGroups = 2;        // 8-entry groups in flight per accumulate lane
constexpr long long kWaitLimit = 1ll << 24;
// Blocks are padded to a multiple of 8 entries; a padding entry points at
// offset 0 of its slice (its value is read and never added) and at
// destination kPadDst, past every offset of a bin.
constexpr uint16_t kPadDst = 0xFFFFu;
static_assert(kPbDstBits < 16, "kPadDst must lie past every destination offset");

struct __align__(128) GatherSmem {
    float xs[kSrcSlice];
    unsigned long long bar;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool wait_bar(unsigned long long* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
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

// Pass 1.  Item: entries [e0, e0 + n) of source slice `slice`.
__global__ void __launch_bounds__(kGatherThreads, kGatherCtas)
    pb_gather_kernel(const gs_pb_item1* __restrict__ items, uint64_t n_items, const uint16_t* __restrict__ src,
                     const float* __restrict__ x, float* __restrict__ val, int* error, unsigned int* ticket) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    GatherSmem& m = *reinterpret_cast<GatherSmem*>(smem_raw);
    const uint32_t tid = threadIdx.x;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&m.bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t parity = 0;
    __shared__ unsigned long long s_item;
    auto advance = [&](uint64_t i) -> uint64_t {
        if (!ticket) return i + gridDim.x;
        __syncthreads();   // every thread has read the previous draw
        if (tid == 0) s_item = atomicAdd(ticket, 1u);
        __syncthreads();
        return s_item;
    };
    for (uint64_t i = ticket ? advance(0) : blockIdx.x; i < n_items; i = advance(i)) {
        const gs_pb_item1 it = items[i];
        if (tid == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&m.bar)),
                         "r"(kSrcSlice * 4)
                         : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_u32(m.xs)),
                "l"(x + ((uint64_t)it.slice << kPbSrcBits)), "r"(kSrcSlice * 4), "r"(smem_u32(&m.bar))
                : "memory");
        }
        const bool got = wait_bar(&m.bar, parity);
        parity ^= 1;
        if (!__syncthreads_and(got)) {
            // the copy is late: flag it and give it one more bounded wait, so
            // that the CTA does not leave with its copy still in flight
            if (tid == 0) {
                atomicExch(error, 1);
                wait_bar(&m.bar, parity ^ 1);
            }
            break;   // uniform
        }
        const uint64_t e0 = it.e0, end = it.e0 + it.n;
        // head up to a multiple of 8 entries, 8-entry body (16-byte loads,
        // two 16-byte stores), tail
        const uint64_t a = ((e0 + 7) & ~7ull) < end ? ((e0 + 7) & ~7ull) : end;
        const uint64_t b = (end & ~7ull) > a ? (end & ~7ull) : a;
        for (uint64_t e = e0 + tid; e < a; e += kGatherThreads) val[e] = m.xs[src[e]];
        for (uint64_t e = b + tid; e < end; e += kGatherThreads) val[e] = m.xs[src[e]];
        const uint4* s8 = reinterpret_cast<const uint4*>(src);
        float4* v4 = reinterpret_cast<float4*>(val);
        const uint64_t c1 = b >> 3;
        auto emit = [&](const uint4 w, uint64_t ck) {
            v4[2 * ck] = make_float4(m.xs[w.x & 0xFFFFu], m.xs[w.x >> 16], m.xs[w.y & 0xFFFFu], m.xs[w.y >> 16]);
            v4[2 * ck + 1] = make_float4(m.xs[w.z & 0xFFFFu], m.xs[w.z >> 16], m.xs[w.w & 0xFFFFu], m.xs[w.w >> 16]);
        };
        // the next groups' offsets are loaded before this one's are used, so
        // the loads overlap the shared-memory gathers and the stores
        constexpr uint64_t kStride = (uint64_t)kGatherThreads * kGatherGroups;
        uint4 w[kGatherGroups];
        uint64_t c = (a >> 3) + tid;
#pragma unroll
        for (int k = 0; k < kGatherGroups; ++k) {
            const uint64_t ck = c + (uint64_t)k * kGatherThreads;
            if (ck < c1) w[k] = __ldcs(s8 + ck);
        }
        for (; c < c1; c += kStride) {
            uint4 nw[kGatherGroups];
#pragma unroll
            for (int k = 0; k < kGatherGroups; ++k) {
                const uint64_t ck = c + kStride + (uint64_t)k * kGatherThreads;
                nw[k] = ck < c1 ? __ldcs(s8 + ck) : make_uint4(0, 0, 0, 0);
            }
#pragma unroll
            for (int k = 0; k < kGatherGroups; ++k) {
                const uint64_t ck = c + (uint64_t)k * kGatherThreads;
                if (ck < c1) emit(w[k], ck);
                w[k] = nw[k];
            }
        }
        __syncthreads();   // xs is rewritten by the next item
    }
    if (ticket && tid == 0 && atomicAdd(ticket + 1, 1u) == gridDim.x - 1) {
        atomicExch(ticket, 0u);   // every CTA has drawn its last ticket
        atomicExch(ticket + 1, 0u);
    }
}

// Adds the 8 entries of every lane of a group of W lanes (lane l of the W:
// the l-th 8-entry group of a window of the bin's group list, its entries
// sorted by destination; `valid` false for a lane past the item) into the
// shared sums.  Equal destinations are adjacent inside a group, and a run may
// cross lanes (a high-degree vertex can fill many groups of a block; two
// groups of neighbouring blocks may also end and start on one destination,
// whose sum is the same either way): a lane sums its runs in registers and
// adds the ones inside it at once; its first and last runs join the
// neighbouring lanes' runs through a segmented prefix scan over the W lanes,
// and each run is added once, by the lane where it ends.  Without the
// cross-lane step all lanes of a run would hit one address in the same
// atomic instruction.  Padding entries carry kPadDst (past every offset) and
// are never added.
template <int W>
__device__ __forceinline__ void add_lane_groups(float* acc, uint32_t hl, unsigned mask, bool valid, const uint4 d,
                                                const float4 lo, const float4 hi) {
    const uint32_t o[8] = {d.x & 0xFFFFu, d.x >> 16, d.y & 0xFFFFu, d.y >> 16,
                           d.z & 0xFFFFu, d.z >> 16, d.w & 0xFFFFu, d.w >> 16};
    const float v[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
    // in-lane runs: the first (f, sf) and the last (t, run) stay open, the
    // ones between them are added here
    const uint32_t f = valid ? o[0] : 0x10000u + hl;   // past any offset: links nothing
    uint32_t t = f;
    float run = valid ? v[0] : 0.f, sf = 0.f;
    bool single = true;
#pragma unroll
    for (int j = 1; j < 8; ++j) {
        if (!valid) break;
        if (o[j] != t) {
            if (single) sf = run;
            else if (t < kDstBin) atomicAdd(acc + t, run);
            single = false;
            t = o[j];
            run = v[j];
        } else {
            run += v[j];
        }
    }
    // lane l's first run continues lane l-1's last run when their keys match
    const uint32_t t_prev = __shfl_up_sync(mask, t, 1, W);
    const bool link = hl > 0 && t_prev == f;
    // segmented prefix sums of the last runs: a segment starts at a lane
    // whose first run does not continue the previous lane's, or whose first
    // run is not its last (its last run starts a new chain)
    float c = run;
    bool head = !single || !link;
#pragma unroll
    for (int k = 1; k < W; k <<= 1) {
        const float cu = __shfl_up_sync(mask, c, k, W);
        const bool hu = __shfl_up_sync(mask, head, k, W);
        if (hl >= (uint32_t)k && !head) {
            c += cu;
            head = hu;
        }
    }
    const float carry_in = __shfl_up_sync(mask, c, 1, W);
    const bool link_next = __shfl_down_sync(mask, link, 1, W) && hl < W - 1;
    if (!valid) return;
    if (!single && f < kDstBin) atomicAdd(acc + f, sf + (link ? carry_in : 0.f));   // first run, closed here
    if (!link_next && t < kDstBin) atomicAdd(acc + t, c);                          // the last run's chain ends here
}

// Pass 2.  Item: groups [b0, b1) of the group list, all of bin `bin`;
// `whole` when the item holds every group of the bin (its sums are then
// stored, else added to y).  A warp takes windows of 32 consecutive groups
// (a lane per group: one 4-byte group index, then one 16-byte load of
// destination offsets and two of values), kAccGroups windows in flight.
__global__ void __launch_bounds__(kAccThreads, kAccCtas)
    pb_accumulate_kernel(const gs_pb_item2* __restrict__ items, uint64_t n_items, const uint32_t* __restrict__ groups,
                         const uint16_t* __restrict__ dst, const float* __restrict__ val, float* __restrict__ y,
                         unsigned int* ticket) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float* acc = reinterpret_cast<float*>(smem_raw);
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr uint32_t kWarps = kAccThreads / 32;
    constexpr uint32_t kStep = 32 * kAccGroups;
    __shared__ unsigned long long s_item;
    auto advance = [&](uint64_t i) -> uint64_t {
        if (!ticket) return i + gridDim.x;
        __syncthreads();
        if (tid == 0) s_item = atomicAdd(ticket, 1u);
        __syncthreads();
        return s_item;
    };
    float4* acc4 = reinterpret_cast<float4*>(acc);
    const uint4* d8 = reinterpret_cast<const uint4*>(dst);
    const float4* v4 = reinterpret_cast<const float4*>(val);
    for (uint64_t i = ticket ? advance(0) : blockIdx.x; i < n_items; i = advance(i)) {
        const gs_pb_item2 it = items[i];
        for (uint32_t k = tid; k < kDstBin / 4; k += kAccThreads) acc4[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        __syncthreads();
        for (uint64_t w0 = (uint64_t)it.b0 + warp * kStep; w0 < it.b1; w0 += kWarps * kStep) {   // uniform in the warp
            uint32_t gi[kAccGroups];
#pragma unroll
            for (int k = 0; k < kAccGroups; ++k) {
                const uint64_t gk = w0 + 32u * k + lane;
                gi[k] = gk < it.b1 ? __ldcs(groups + gk) : 0u;
            }
            uint4 d[kAccGroups];
            float4 lo[kAccGroups], hi[kAccGroups];
#pragma unroll
            for (int k = 0; k < kAccGroups; ++k) {
                d[k] = make_uint4(0, 0, 0, 0);
                lo[k] = hi[k] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (w0 + 32u * k + lane < it.b1) {
                    d[k] = __ldcs(d8 + gi[k]);
                    lo[k] = __ldcs(v4 + 2 * (uint64_t)gi[k]);
                    hi[k] = __ldcs(v4 + 2 * (uint64_t)gi[k] + 1);
                }
            }
#pragma unroll
            for (int k = 0; k < kAccGroups; ++k)
                add_lane_groups<32>(acc, lane, 0xFFFFFFFFu, w0 + 32u * k + lane < it.b1, d[k], lo[k], hi[k]);
        }
        __syncthreads();
        float4* y4 = reinterpret_cast<float4*>(y + ((uint64_t)it.bin << kPbDstBits));
        for (uint32_t k = tid; k < kDstBin / 4; k += kAccThreads) {
            const float4 s = acc4[k];
            if (it.whole) y4[k] = s;
            else if (s.x != 0.f || s.y != 0.f || s.z != 0.f || s.w != 0.f) atomicAdd(y4 + k, s);
        }
        __syncthreads();   // acc is cleared by the next item
    }
    if (ticket && tid == 0 && atomicAdd(ticket + 1, 1u) == gridDim.x - 1) {
        atomicExch(ticket, 0u);
        atomicExch(ticket + 1, 0u);
    }
}

// ------------------------------------------------------------------ build --
// One key per (record, direction): (S * nD + D) above kKeyLowBits, then the
// destination's and the source's offsets.
__device__ __forceinline__ uint64_t pb_key(uint32_t src, uint32_t dst, uint32_t nD) {
    const uint64_t blk = (uint64_t)(src >> kPbSrcBits) * nD + (dst >> kPbDstBits);
    return (blk << kKeyLowBits) | ((uint64_t)(dst & (kDstBin - 1)) << kPbSrcBits) | (src & (kSrcSlice - 1));
}

__global__ void pb_keys_kernel(const gs_unit* __restrict__ units, uint64_t n_units, const uint32_t* __restrict__ rec,
                               uint32_t nD, int directed, uint64_t* __restrict__ keys) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t n_warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t u = warp; u < n_units; u += n_warps) {
        const gs_unit un = units[u];
        const uint32_t rb = (un.rc >> 16) << 16, cb = (un.rc & 0xFFFFu) << 16;
        for (uint32_t k = lane; k < un.n; k += 32) {
            const uint64_t e = un.rec_beg + k;
            const uint32_t r = rec[e];
            const uint32_t a = rb + (r & 0xFFFFu), b = cb + (r >> 16);
            if (directed) {
                keys[e] = pb_key(a, b, nD);                  // push v0 -> v1 only (pr.cpp:141-146)
            } else {
                keys[2 * e] = pb_key(a, b, nD);              // rank[v1] += prior[v0]
                keys[2 * e + 1] = pb_key(b, a, nD);          // rank[v0] += prior[v1]
            }
        }
    }
}

// Block counts rounded up to 8 entries: pc[bid] (bid < n_blk), pc[n_blk] = 0.
__global__ void pb_padded_count_kernel(const uint64_t* __restrict__ start, uint64_t n_blk, uint64_t* __restrict__ pc) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t bid = tid; bid <= n_blk; bid += nth)
        pc[bid] = bid < n_blk ? (start[bid + 1] - start[bid] + 7) & ~7ull : 0;
}

// The sorted keys of block bid go to the padded streams at pstart[bid]
// (source and destination offsets), then the block's padding entries (a warp
// per block).
__global__ void pb_split_kernel(const uint64_t* __restrict__ keys, const uint64_t* __restrict__ start,
                                const uint64_t* __restrict__ pstart, uint64_t n_blk, uint16_t* __restrict__ src,
                                uint16_t* __restrict__ dst) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t n_warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t bid = warp; bid < n_blk; bid += n_warps) {
        const uint64_t s0 = start[bid], n = start[bid + 1] - s0, p0 = pstart[bid], pn = pstart[bid + 1] - p0;
        for (uint64_t k = lane; k < pn; k += 32) {
            if (k < n) {
                const uint64_t key = keys[s0 + k];
                src[p0 + k] = (uint16_t)(key & (kSrcSlice - 1));
                dst[p0 + k] = (uint16_t)((key >> kPbSrcBits) & (kDstBin - 1));
            } else {
                src[p0 + k] = 0;
                dst[p0 + k] = kPadDst;
            }
        }
    }
}

// First entry of every block id in [0, n_blk] (n_blk: one past the last):
// a binary search over the sorted keys.
__global__ void pb_block_start_kernel(const uint64_t* __restrict__ keys, uint64_t n, uint64_t n_blk,
                                      uint64_t* __restrict__ start) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t bid = tid; bid <= n_blk; bid += nth) {
        uint64_t lo = 0, hi = n;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if ((keys[mid] >> kKeyLowBits) < bid) lo = mid + 1;
            else hi = mid;
        }
        start[bid] = lo;
    }
}

// The D-major block table: blocks[D * nS + S] = block (S, D).
__global__ void pb_block_table_kernel(const uint64_t* __restrict__ start, uint32_t nS, uint32_t nD,
                                      gs_pb_block* __restrict__ blocks) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t n_blk = (uint64_t)nS * nD;
    for (uint64_t p = tid; p < n_blk; p += nth) {
        const uint64_t D = p / nS, S = p % nS, bid = S * nD + D;
        blocks[p] = gs_pb_block{start[bid], (uint32_t)(start[bid + 1] - start[bid]), 0u};
    }
}

// The group list: block p of the D-major table (entries [e0, e0 + n), n a
// multiple of 8) lists its groups e0/8 .. (e0 + n)/8 - 1 from gpos[p] on.
// A warp per block.
__global__ void pb_group_list_kernel(const gs_pb_block* __restrict__ blocks, const uint64_t* __restrict__ gpos,
                                     uint64_t n_blk, uint32_t* __restrict__ groups) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t n_warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t p = warp; p < n_blk; p += n_warps) {
        const gs_pb_block b = blocks[p];
        const uint64_t g0 = b.e0 >> 3, out = gpos[p];
        for (uint32_t k = lane; k < (b.n >> 3); k += 32) groups[out + k] = (uint32_t)(g0 + k);
    }
}

inline uint32_t grid_for(uint64_t n, const gs_ctx* ctx) {
    const uint64_t b = (n + 255) / 256;
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(b, gs_grid_size(ctx, 16)));
}

}  // namespace

void pb_layout_free(gs_graph* g) {
    gs_pb_layout& L = g->pb;
    gs_dev_free(L.d_src);
    gs_dev_free(L.d_dst);
    gs_dev_free(L.d_val);
    gs_dev_free(L.d_groups);
    gs_dev_free(L.d_items1);
    gs_dev_free(L.d_items2);
    L = gs_pb_layout();
}

bool pb_layout_wanted(const gs_graph* g) {
    if (g->stream || g->E == 0) return false;
    const uint64_t n_ent = g->directed ? g->E : 2 * g->E;
    const uint64_t nS = g->N >> kPbSrcBits, nD = g->N >> kPbDstBits;
    // the block table is dense (every (S, D) pair): worth it when blocks hold
    // many entries on average; group indices (entry / 8) are 32-bit
    if (nS * nD * 64 > n_ent || nS * nD >= (1ull << 31) || n_ent + 8 * nS * nD >= (1ull << 34)) return false;
    // under an HBM budget the layout (8 B per entry) must fit beside the records
    if (g->ctx->budget && 4 * g->E + 8 * n_ent > g->ctx->budget) return false;
    // building needs the sort's two key buffers too
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return false;
    const uint64_t need = (n_ent + 8 * nS * nD) * 8 + n_ent / 2 + n_ent * 16 + (nS * nD + 1) * 40 + (2ull << 30);
    // (idle pool blocks count as free: an allocation that fails releases them)
    return free_b + g->ctx->pool_bytes > need;
}

gs_status pb_layout_build(gs_graph* g) {
    gs_ctx* ctx = g->ctx;
    gs_pb_layout& L = g->pb;
    pb_layout_free(g);
    const uint64_t n_ent = g->directed ? g->E : 2 * g->E;
    const uint32_t nS = (uint32_t)(g->N >> kPbSrcBits), nD = (uint32_t)(g->N >> kPbDstBits);
    const uint64_t n_blk = (uint64_t)nS * nD;
    int end_bit = kKeyLowBits;
    while ((1ull << (end_bit - kKeyLowBits)) < n_blk) ++end_bit;

    uint64_t *d_k0 = nullptr, *d_k1 = nullptr, *d_start = nullptr, *d_pstart = nullptr;
    gs_pb_block* d_blocks = nullptr;   // the D-major block table (build only)
    uint64_t n_pad = 0;   // entries with every block padded to a multiple of 8
    void* d_tmp = nullptr;
    size_t tmp_bytes = 0;
    gs_status st = gs_dev_alloc(ctx, (void**)&d_k0, n_ent * 8);
    if (st == GS_OK) st = gs_dev_alloc(ctx, (void**)&d_k1, n_ent * 8);
    if (st == GS_OK) {
        pb_keys_kernel<<<gs_grid_size(ctx, 8), 256, 0, ctx->stream>>>(g->d_units, g->U, g->d_rec, nD, g->directed,
                                                                       d_k0);
        ctx->launches++;
        cudaError_t e = cudaGetLastError();
        cub::DoubleBuffer<uint64_t> keys(d_k0, d_k1);
        if (e == cudaSuccess)
            e = cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, keys, n_ent, 0, end_bit, ctx->stream);
        if (e == cudaSuccess) st = gs_dev_alloc(ctx, &d_tmp, tmp_bytes);
        if (e == cudaSuccess && st == GS_OK)
            e = cub::DeviceRadixSort::SortKeys(d_tmp, tmp_bytes, keys, n_ent, 0, end_bit, ctx->stream);
        ctx->launches++;
        if (e != cudaSuccess && st == GS_OK) st = gs_cuda_fail(ctx, e, "propagation-blocking key sort");
        const uint64_t* sorted = keys.Current();
        gs_dev_free(d_tmp);
        d_tmp = nullptr;
        if (st == GS_OK) st = gs_dev_alloc(ctx, (void**)&d_start, (n_blk + 1) * 8);
        if (st == GS_OK) st = gs_dev_alloc(ctx, (void**)&d_pstart, (n_blk + 1) * 8);
        if (st == GS_OK) {
            pb_block_start_kernel<<<grid_for(n_blk + 1, ctx), 256, 0, ctx->stream>>>(sorted, n_ent, n_blk, d_start);
            pb_padded_count_kernel<<<grid_for(n_blk + 1, ctx), 256, 0, ctx->stream>>>(d_start, n_blk, d_pstart);
            ctx->launches += 2;
            e = cudaGetLastError();
            size_t scan_bytes = 0;
            if (e == cudaSuccess)
                e = cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, d_pstart, d_pstart, n_blk + 1, ctx->stream);
            if (e == cudaSuccess) st = gs_dev_alloc(ctx, &d_tmp, scan_bytes);
            if (e == cudaSuccess && st == GS_OK)
                e = cub::DeviceScan::ExclusiveSum(d_tmp, scan_bytes, d_pstart, d_pstart, n_blk + 1, ctx->stream);
            ctx->launches++;
            if (e == cudaSuccess && st == GS_OK)
                e = cudaMemcpyAsync(&n_pad, d_pstart + n_blk, 8, cudaMemcpyDeviceToHost, ctx->stream);
            if (e == cudaSuccess && st == GS_OK) e = cudaStreamSynchronize(ctx->stream);
            gs_dev_free(d_tmp);
            d_tmp = nullptr;
            if (e != cudaSuccess && st == GS_OK) st = gs_cuda_fail(ctx, e, "propagation-blocking block starts");
        }
        if (st == GS_OK) st = gs_dev_alloc(ctx, (void**)&L.d_src, n_pad * 2);
        if (st == GS_OK) st = gs_dev_alloc(ctx, (void**)&L.d_dst, n_pad * 2);
        if (st == GS_OK) st = gs_dev_alloc(ctx, (void**)&d_blocks, std::max<uint64_t>(1, n_blk) * sizeof(gs_pb_block));
        if (st == GS_OK) {
            pb_split_kernel<<<gs_grid_size(ctx, 8), 256, 0, ctx->stream>>>(sorted, d_start, d_pstart, n_blk, L.d_src,
                                                                            L.d_dst);
            pb_block_table_kernel<<<grid_for(n_blk, ctx), 256, 0, ctx->stream>>>(d_pstart, nS, nD, d_blocks);
            ctx->launches += 2;
            e = cudaGetLastError();
            if (e != cudaSuccess) st = gs_cuda_fail(ctx, e, "propagation-blocking layout");
        }
    }
    gs_dev_free(d_k0);
    gs_dev_free(d_k1);
    std::vector<gs_pb_block> blocks(n_blk);
    std::vector<uint64_t> slice_start(nS + 1);
    if (st == GS_OK) {
        cudaError_t e = cudaMemcpyAsync(blocks.data(), d_blocks, n_blk * sizeof(gs_pb_block),
                                        cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        // entries of slice S start at block (S, 0), the first of the bin-major table
        for (uint32_t s = 0; s < nS; ++s) slice_start[s] = blocks[s].e0;
        slice_start[nS] = n_pad;
        if (e != cudaSuccess) st = gs_cuda_fail(ctx, e, "propagation-blocking tables");
    }
    gs_dev_free(d_start);
    gs_dev_free(d_pstart);
    if (st != GS_OK) {
        gs_dev_free(d_blocks);
        pb_layout_free(g);
        return st;
    }
    // The group list the accumulate pass walks: every bin's blocks in slice
    // order, as 8-entry groups, so that a bin is one flat sequence of groups
    // however its entries are spread over blocks (a lane per group).
    std::vector<uint64_t> gpos(n_blk + 1);
    gpos[0] = 0;
    for (uint64_t b = 0; b < n_blk; ++b) gpos[b + 1] = gpos[b] + (blocks[b].n >> 3);
    const uint64_t n_groups = gpos[n_blk];
    // Items: entry chunks of every slice (pass 1) and group ranges of every
    // bin (pass 2), sized so that each pass has a few items per resident CTA
    // (pass 2: ~16, so that the last wave of equal items leaves few SMs idle).
    // (item boundaries stay multiples of 8 entries: every block starts on one)
    const uint64_t per1 =
        std::clamp<uint64_t>(n_pad / ((uint64_t)ctx->num_sms * kGatherCtas * 4), 32768, 1ull << 20) & ~7ull;
    const uint64_t per2 =
        std::clamp<uint64_t>(n_groups / ((uint64_t)ctx->num_sms * kAccCtas * 16), 8192, 1ull << 19);
    std::vector<gs_pb_item1> items1;
    for (uint32_t s = 0; s < nS; ++s)
        for (uint64_t e = slice_start[s]; e < slice_start[s + 1]; e += per1)
            items1.push_back(gs_pb_item1{e, (uint32_t)std::min<uint64_t>(per1, slice_start[s + 1] - e), s});
    std::vector<gs_pb_item2> items2;
    for (uint32_t d = 0; d < nD; ++d) {
        const uint64_t g0 = gpos[(uint64_t)d * nS], g1 = gpos[(uint64_t)(d + 1) * nS];
        const uint64_t parts = (g1 - g0 + per2 - 1) / per2;
        for (uint64_t k = 0; k < parts; ++k)
            items2.push_back(gs_pb_item2{(uint32_t)(g0 + (g1 - g0) * k / parts),
                                         (uint32_t)(g0 + (g1 - g0) * (k + 1) / parts), d, parts == 1 ? 1u : 0u});
    }
    L.n_entries = n_pad;
    L.n_groups = n_groups;
    L.n_items1 = items1.size();
    L.n_items2 = items2.size();
    uint64_t* d_gpos = nullptr;
    st = gs_dev_alloc(ctx, (void**)&L.d_val, n_pad * 4);
    if (st == GS_OK) st = gs_dev_alloc(ctx, (void**)&L.d_groups, std::max<uint64_t>(1, n_groups) * 4);
    if (st == GS_OK) st = gs_dev_alloc(ctx, (void**)&d_gpos, (n_blk + 1) * 8);
    if (st == GS_OK) st = gs_dev_alloc(ctx, (void**)&L.d_items1, std::max<size_t>(1, items1.size()) * sizeof(gs_pb_item1));
    if (st == GS_OK) st = gs_dev_alloc(ctx, (void**)&L.d_items2, std::max<size_t>(1, items2.size()) * sizeof(gs_pb_item2));
    cudaError_t e = cudaSuccess;
    if (st == GS_OK)
        e = cudaMemcpyAsync(d_gpos, gpos.data(), (n_blk + 1) * 8, cudaMemcpyHostToDevice, ctx->stream);
    if (st == GS_OK && e == cudaSuccess) {
        pb_group_list_kernel<<<gs_grid_size(ctx, 8), 256, 0, ctx->stream>>>(d_blocks, d_gpos, n_blk, L.d_groups);
        ctx->launches++;
        e = cudaGetLastError();
    }
    if (st == GS_OK && e == cudaSuccess && !items1.empty())
        e = cudaMemcpyAsync(L.d_items1, items1.data(), items1.size() * sizeof(gs_pb_item1), cudaMemcpyHostToDevice,
                            ctx->stream);
    if (st == GS_OK && e == cudaSuccess && !items2.empty())
        e = cudaMemcpyAsync(L.d_items2, items2.data(), items2.size() * sizeof(gs_pb_item2), cudaMemcpyHostToDevice,
                            ctx->stream);
    if (st == GS_OK && e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (st == GS_OK && e != cudaSuccess) st = gs_cuda_fail(ctx, e, "propagation-blocking items");
    gs_dev_free(d_gpos);
    gs_dev_free(d_blocks);
    if (st != GS_OK) {
        pb_layout_free(g);
        return st;
    }
    L.built = true;
    return GS_OK;
}

gs_status pb_sweep(gs_graph* g, const float* x, float* y, int* error) {
    gs_ctx* ctx = g->ctx;
    const gs_pb_layout& L = g->pb;
    if (L.n_items1 == 0) return GS_OK;
    GS_CHECK_CUDA(ctx, gs_smem_limit_once<pb_gather_kernel>(ctx->device, (int)sizeof(GatherSmem)));
    GS_CHECK_CUDA(ctx, gs_smem_limit_once<pb_accumulate_kernel>(ctx->device, (int)(kDstBin * 4)));
    const uint32_t g1 = (uint32_t)std::min<uint64_t>(L.n_items1, gs_grid_size(ctx, kGatherCtas));
    pb_gather_kernel<<<g1, kGatherThreads, sizeof(GatherSmem), ctx->stream>>>(L.d_items1, L.n_items1, L.d_src, x,
                                                                             L.d_val, error, ctx->d_ticket + 4);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    const uint32_t g2 = (uint32_t)std::min<uint64_t>(L.n_items2, gs_grid_size(ctx, kAccCtas));
    pb_accumulate_kernel<<<g2, kAccThreads, kDstBin * 4, ctx->stream>>>(L.d_items2, L.n_items2, L.d_groups, L.d_dst,
                                                                       L.d_val, y, ctx->d_ticket + 6);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches += 2;
    return GS_OK;
}

gs_status pb_sweep_on(gs_graph* g, cudaStream_t stream, const float* x, float* y, int* error, float* val) {
    gs_ctx* ctx = g->ctx;
    const gs_pb_layout& L = g->pb;
    if (L.n_items1 == 0) return GS_OK;
    GS_CHECK_CUDA(ctx, gs_smem_limit_once<pb_gather_kernel>(ctx->device, (int)sizeof(GatherSmem)));
    GS_CHECK_CUDA(ctx, gs_smem_limit_once<pb_accumulate_kernel>(ctx->device, (int)(kDstBin * 4)));
    // one CTA per item and no ticket: short CTAs, so that a higher-priority
    // stream's CTAs find free SMs between them
    pb_gather_kernel<<<(uint32_t)L.n_items1, kGatherThreads, sizeof(GatherSmem), stream>>>(
        L.d_items1, L.n_items1, L.d_src, x, val, error, nullptr);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    pb_accumulate_kernel<<<(uint32_t)L.n_items2, kAccThreads, kDstBin * 4, stream>>>(
        L.d_items2, L.n_items2, L.d_groups, L.d_dst, val, y, nullptr);
    GS_CHECK_CUDA(ctx, cudaGetLastError());
    ctx->launches += 2;
    return GS_OK;
}

gs_status pb_launch(gs_state* s) {
    gs_graph* g = s->g;
    gs_ctx* ctx = g->ctx;
    if (!s->d_error) {
        GS_TRY(gs_state_alloc(s, (void**)&s->d_error, sizeof(uint64_t)));
        GS_CHECK_CUDA(ctx, cudaMemsetAsync(s->d_error, 0, sizeof(uint64_t), ctx->stream));
    }
    gs_timer_begin(ctx);
    GS_TRY(pb_sweep(g, s->d_x, s->d_y, (int*)s->d_error));
    // algorithmic bytes per iteration: 4E + 12V (records, x, s, inv)
    gs_timer_end(ctx, GS_ALGO_PAGERANK, 4 * g->E + 12 * g->V);
    return GS_OK;
}
